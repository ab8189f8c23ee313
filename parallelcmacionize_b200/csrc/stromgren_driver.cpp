// Stromgren-sphere driver on the GPU path, with the command line and
// params.txt of the reference's OpenMP driver (testDensitySubGrid_omp.cpp):
//
//   stromgren_driver -t THREADS -p params.txt
//
// THREADS only seeds the host generator the way the reference does
// (random_generator[0] seeded 42 + THREADS, testDensitySubGrid_omp.cpp:1786-1790),
// so a random density field and random sources come out identical to a
// reference run with the same -t.  The transport and balance run on the GPU.
// Output: the reference's two result files, subgrid after subgrid:
// neutral_fractions.dat (cell centre, x_H, n_H and zero hydro slots, 60 bytes
// per cell; output_neutral_fractions, testDensitySubGrid_omp.cpp:394-442) and
// neutral_fractions.bin (x_H only; output_neutral_fractions_binary, :507-521).
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "cmacionize/DensityGrid.hpp"
#include "cmacionize/Parameters.hpp"
#include "cmacionize/RandomDensity.hpp"
#include "cmacionize/RandomGenerator.hpp"

int main(int argc, char **argv) {
  int threads = 1;
  std::string params_file;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    if ((a == "-t" || a == "--threads") && i + 1 < argc) threads = std::atoi(argv[++i]);
    else if ((a == "-p" || a == "--params") && i + 1 < argc) params_file = argv[++i];
  }
  if (params_file.empty()) {
    std::fprintf(stderr, "usage: %s -t THREADS -p PARAMS\n", argv[0]);
    return 2;
  }
  try {
    const PlainMethodParameters p(Parameters::from_file(params_file));
    DensityGrid grid(p.box, p.ncell, p.num_subgrid);
    grid.set_reemission_probability(p.reemission_probability);
    RandomGenerator rng(42 + threads);

    if (p.random_density) {
      // 10-mode cosine field, testDensitySubGrid_omp.cpp:1880-1934
      const CosineDensityField field(rng, p.box);
      const int *n = grid.subgrid_cells();
      for (unsigned int s = 0; s < grid.number_of_subgrids(); ++s) {
        DensitySubGrid sg = grid.subgrid(s);
        double box[6];
        sg.get_grid_box(box);
        for (unsigned int c = 0; c < sg.get_number_of_cells(); ++c) {
          const int i3[3] = {(int)(c / (n[1] * n[2])), (int)((c / n[2]) % n[1]), (int)(c % n[2])};
          double mid[3];
          CosineDensityField::cell_midpoint(box, n, i3, mid);
          sg.set_number_density(c, field(mid));
        }
      }
    }

    // sources, testDensitySubGrid_omp.cpp:1944-2016
    std::vector<Source> sources;
    if (p.number_of_sources > 1) {
      for (unsigned int i = 0; i < p.number_of_sources; ++i) {
        double pos[3];
        for (int a = 0; a < 3; ++a) pos[a] = p.box[a] + rng.get_uniform_random_double() * p.box[3 + a];
        sources.emplace_back(pos, 4.26e48);
      }
    } else {
      const double origin[3] = {0., 0., 0.};
      sources.emplace_back(origin, 4.26e49);
    }
    grid.set_sources(sources);
    grid.set_num_photon(p.num_photon);

    const auto t0 = std::chrono::steady_clock::now();
    const std::vector<cmi_stats> st = grid.run_iterations((int)p.number_of_iterations, 42);
    const double mc = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    unsigned long long crossings = 0;
    for (const cmi_stats &s : st) crossings += s.cell_crossings;
    std::fprintf(stderr, "Total Monte Carlo time: %g s.\n", mc);
    std::fprintf(stderr, "Cell crossings: %llu (%.4g per second)\n", crossings, crossings / mc);

    // the reference's result files (MM_FILE and BIN_FILE outputs)
    output_neutral_fractions(grid, "neutral_fractions.dat");
    output_neutral_fractions_binary(grid, "neutral_fractions.bin");
  } catch (const std::exception &e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
