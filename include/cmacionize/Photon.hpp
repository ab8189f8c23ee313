/*
 * Photon (reference: Photon.hpp:49-248).  Same accessors; the storage is the
 * C ABI's cmi_photon, so arrays of Photon pass to the library unchanged.
 */
#ifndef CMACIONIZE_PHOTON_HPP
#define CMACIONIZE_PHOTON_HPP

#include <cstdint>

#include "cmacionize_b200.h"

enum PhotonPacketType {
  PHOTONPACKETTYPE_DIRECT = 0,
  PHOTONPACKETTYPE_TAU,
  PHOTONPACKETTYPE_PEELOFF
};

class Photon {
 private:
  cmi_photon _p;

 public:
  Photon() : _p() {}

  const double *get_position() const { return _p.position; }
  void set_position(double x, double y, double z) {
    _p.position[0] = x;
    _p.position[1] = y;
    _p.position[2] = z;
  }
  const double *get_direction() const { return _p.direction; }
  double *get_direction() { return _p.direction; }
  void set_direction(double x, double y, double z) {
    _p.direction[0] = x;
    _p.direction[1] = y;
    _p.direction[2] = z;
  }
  double get_target_optical_depth() const { return _p.target_optical_depth; }
  void set_target_optical_depth(double t) { _p.target_optical_depth = t; }
  double get_photoionization_cross_section() const { return _p.photoionization_cross_section; }
  void set_photoionization_cross_section(double s) { _p.photoionization_cross_section = s; }
  double get_weight() const { return _p.weight; }
  void set_weight(double w) { _p.weight = w; }
  int_fast32_t get_type() const { return _p.type; }
  void set_type(int_fast32_t t) { _p.type = (int32_t)t; }

  cmi_photon *raw() { return &_p; }
  const cmi_photon *raw() const { return &_p; }
};
static_assert(sizeof(Photon) == sizeof(cmi_photon), "Photon is a cmi_photon");

#endif
