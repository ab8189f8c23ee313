// The reference driver's random density field: the mean of 10 products of
// cosines with normally distributed wave vectors (4 pi k / box side) and
// uniform phases, around n_H = 1e8 m^-3 (testDensitySubGrid_omp.cpp:1880-1934).
// The modes are drawn from the host generator in the driver's order (four
// uniforms for the wave vector, then three phases, per mode), so a generator
// seeded as the driver seeds random_generator[0] gives the same field.
#ifndef CMACIONIZE_RANDOMDENSITY_HPP
#define CMACIONIZE_RANDOMDENSITY_HPP

#include <cmath>

#include "RandomGenerator.hpp"

class CosineDensityField {
 public:
  static constexpr unsigned int number_of_modes = 10;

  CosineDensityField(RandomGenerator &rng, const double box[6]) {
    for (unsigned int i = 0; i < number_of_modes; ++i) {
      double u[4];
      for (double &x : u) x = rng.get_uniform_random_double();
      const double kx = std::sqrt(-2. * std::log(u[0])) * std::cos(2. * M_PI * u[1]);
      const double ky = std::sqrt(-2. * std::log(u[0])) * std::sin(2. * M_PI * u[1]);
      const double kz = std::sqrt(-2. * std::log(u[2])) * std::cos(2. * M_PI * u[3]);
      _k[3 * i] = 4. * M_PI * kx / box[3];
      _k[3 * i + 1] = 4. * M_PI * ky / box[4];
      _k[3 * i + 2] = 4. * M_PI * kz / box[5];
      for (int a = 0; a < 3; ++a) _phase[3 * i + a] = 2. * M_PI * rng.get_uniform_random_double();
    }
  }

  // n_H at a cell midpoint, summed mode by mode in draw order
  double operator()(const double midpoint[3]) const {
    double n = 0.;
    for (unsigned int q = 0; q < number_of_modes; ++q) {
      n += 1.e8 * (std::cos(_k[3 * q] * midpoint[0] + _phase[3 * q]) *
                       std::cos(_k[3 * q + 1] * midpoint[1] + _phase[3 * q + 1]) *
                       std::cos(_k[3 * q + 2] * midpoint[2] + _phase[3 * q + 2]) +
                   1.);
    }
    return n / number_of_modes;
  }

  // midpoint of cell (ix, iy, iz) of a subgrid box (anchor, sides) with n
  // cells per axis, as DensitySubGrid::get_cell_midpoint computes it
  // (DensitySubGrid.hpp:2046-2053, cell size = side / cells)
  static void cell_midpoint(const double box[6], const int n[3], const int i3[3],
                            double midpoint[3]) {
    for (int a = 0; a < 3; ++a) midpoint[a] = box[a] + (i3[a] + 0.5) * (box[3 + a] / n[a]);
  }

 private:
  double _k[3 * number_of_modes];
  double _phase[3 * number_of_modes];
};

#endif
