/*
 * RandomGenerator (reference: RandomGenerator.hpp:36-232): the reference's
 * ranlxd stream, bit for bit.
 */
#ifndef CMACIONIZE_RANDOMGENERATOR_HPP
#define CMACIONIZE_RANDOMGENERATOR_HPP

#include <cstdint>

#include "ranlxd.h"

class RandomGenerator {
 private:
  cmi_ranlxd::Ranlxd _state;

 public:
  explicit RandomGenerator(int_fast32_t seed = 42) { set_seed(seed); }
  void set_seed(int_fast32_t seed) { _state.seed((int32_t)seed); }
  double get_uniform_random_double() { return _state.uniform(); }
  int_fast32_t get_random_integer() { return get_uniform_random_double() * 2147483648.0; }
};

#endif
