/*
 * Source (reference: Source.hpp:34-109): a point source with its ionizing
 * luminosity and the subgrid (copies) that contain it.  On the GPU path a hot
 * subgrid is shared by several CTAs instead of being copied, so the list
 * normally holds the one original subgrid.
 */
#ifndef CMACIONIZE_SOURCE_HPP
#define CMACIONIZE_SOURCE_HPP

#include <vector>

#include "RandomGenerator.hpp"

class Source {
 private:
  double _position[3];
  double _luminosity;
  std::vector<unsigned int> _subgrid_indices;

 public:
  Source() : _position{0., 0., 0.}, _luminosity(0.) {}
  Source(const double position[3], const double luminosity)
      : _position{position[0], position[1], position[2]}, _luminosity(luminosity) {}
  void add_subgrid_index(unsigned int index) { _subgrid_indices.push_back(index); }
  void get_position(double position[3]) const {
    position[0] = _position[0];
    position[1] = _position[1];
    position[2] = _position[2];
  }
  double get_luminosity() const { return _luminosity; }
  unsigned int get_subgrid_index(RandomGenerator &rng) const {
    return _subgrid_indices[static_cast<unsigned int>(rng.get_uniform_random_double() *
                                                      _subgrid_indices.size())];
  }
  unsigned int get_original_subgrid_index() const { return _subgrid_indices[0]; }
};

#endif
