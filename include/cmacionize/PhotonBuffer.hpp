/*
 * PhotonBuffer (reference: PhotonBuffer.hpp:42-209): up to 200 photons bound
 * for one subgrid, entering from one TravelDirection.
 */
#ifndef CMACIONIZE_PHOTONBUFFER_HPP
#define CMACIONIZE_PHOTONBUFFER_HPP

#include "Photon.hpp"

#define PHOTONBUFFER_SIZE 200u

class PhotonBuffer {
 private:
  unsigned int _subgrid_index;
  int _direction;
  unsigned int _actual_size;
  Photon _photons[PHOTONBUFFER_SIZE];

 public:
  PhotonBuffer() : _subgrid_index(0), _direction(0), _actual_size(0) {}
  unsigned int size() const { return _actual_size; }
  void reset() { _actual_size = 0; }
  const Photon &operator[](unsigned int i) const { return _photons[i]; }
  Photon &operator[](unsigned int i) { return _photons[i]; }
  unsigned int get_next_free_photon() { return _actual_size++; }
  void grow(unsigned int size) { _actual_size = size; }
  void set_subgrid_index(unsigned int s) { _subgrid_index = s; }
  unsigned int get_subgrid_index() const { return _subgrid_index; }
  void set_direction(int d) { _direction = d; }
  int get_direction() const { return _direction; }
  Photon *data() { return _photons; }
  const Photon *data() const { return _photons; }
};

#endif
