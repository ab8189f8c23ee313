/*
 * Host C++ surface of the plain photoionization method over the CUDA library.
 *
 *   DensityGrid     the reference's vector of DensitySubGrid* plus neighbour
 *                   table (testDensitySubGrid_omp.cpp:1801-1877), owned by one
 *                   library context on one GPU
 *   DensitySubGrid  a view of one subgrid with the reference's calls:
 *                   interact (DensitySubGrid.hpp:1180), compute_neutral_fraction
 *                   (:1628), the field setters (:1116-1141), get_start_index
 *                   (:428) and get_output_direction (:483)
 *   do_photon_traversal  (testDensitySubGrid_omp.cpp:607)
 *
 * Field values set through the views are kept in host arrays and copied to
 * the GPU before the next transport call; reads copy back first.  Errors
 * throw std::runtime_error with the library's message (the reference aborts).
 */
#ifndef CMACIONIZE_DENSITYGRID_HPP
#define CMACIONIZE_DENSITYGRID_HPP

#include <cstdint>
#include <fstream>
#include <ostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "Photon.hpp"
#include "PhotonBuffer.hpp"
#include "Source.hpp"
#include "TravelDirections.hpp"
#include "cmacionize_b200.h"

#define NEIGHBOUR_OUTSIDE 0xffffffff

inline void cmi_check(int rc) {
  if (rc != CMI_OK) {
    throw std::runtime_error(std::string("cmacionize_b200: ") + cmi_last_error_string());
  }
}

class DensitySubGrid;

class DensityGrid {
 private:
  cmi_context *_ctx;
  cmi_grid_desc _desc;
  int _sub_ncell[3];
  std::vector<double> _nH, _xH, _J;  // host copies, subgrid-blocked order
  bool _fields_dirty, _host_stale;
  double _total_luminosity;
  uint64_t _num_photon;

 public:
  DensityGrid(const double box[6], const int ncell[3], const int num_subgrid[3],
              const cmi_options *options = nullptr, double recombination_rate = 4.e-19,
              double cross_section = 6.3e-22)
      : _ctx(nullptr), _fields_dirty(false), _host_stale(false), _total_luminosity(0.),
        _num_photon(0) {
    for (int i = 0; i < 6; ++i) _desc.box[i] = box[i];
    for (int a = 0; a < 3; ++a) {
      _desc.ncell[a] = ncell[a];
      _desc.num_subgrid[a] = num_subgrid[a];
      _sub_ncell[a] = num_subgrid[a] > 0 ? ncell[a] / num_subgrid[a] : 0;
    }
    _desc.recombination_rate = recombination_rate;
    _desc.cross_section = cross_section;
    cmi_check(cmi_create(&_desc, 1, options, &_ctx));
    const size_t n = (size_t)ncell[0] * ncell[1] * ncell[2];
    _nH.assign(n, 1.e8);  // DensitySubGrid.hpp:546-549
    _xH.assign(n, 1.e-6);
    _J.assign(n, 0.);
  }
  ~DensityGrid() { cmi_destroy(_ctx); }
  DensityGrid(const DensityGrid &) = delete;
  DensityGrid &operator=(const DensityGrid &) = delete;

  cmi_context *context() { return _ctx; }
  unsigned int number_of_subgrids() const {
    return (unsigned int)(_desc.num_subgrid[0] * _desc.num_subgrid[1] * _desc.num_subgrid[2]);
  }
  size_t cells_per_subgrid() const {
    return (size_t)_sub_ncell[0] * _sub_ncell[1] * _sub_ncell[2];
  }
  const int *subgrid_cells() const { return _sub_ncell; }
  const cmi_grid_desc &desc() const { return _desc; }
  inline DensitySubGrid subgrid(unsigned int index);

  // ---- host <-> device field copies ----
  void push() {
    if (_fields_dirty) {
      cmi_check(cmi_set_fields(_ctx, 0, CMI_LAYOUT_BLOCKED, CMI_MEMORY_HOST, _nH.data(),
                               _xH.data()));
      _fields_dirty = false;
    }
  }
  void pull() {
    if (_host_stale) {
      cmi_check(cmi_get_fields(_ctx, 0, CMI_LAYOUT_BLOCKED, CMI_MEMORY_HOST, _xH.data(),
                               _J.data()));
      _host_stale = false;
    }
  }
  void mark_device_changed() { _host_stale = true; }
  double *host_nH() { pull(); _fields_dirty = true; return _nH.data(); }
  double *host_xH() { pull(); _fields_dirty = true; return _xH.data(); }
  const double *neutral_fractions() { pull(); return _xH.data(); }
  const double *number_densities() const { return _nH.data(); }
  const double *intensity_integrals() { pull(); return _J.data(); }

  // ---- sources and the whole iteration ----
  void set_sources(const std::vector<Source> &sources) {
    std::vector<double> pos, lum;
    _total_luminosity = 0.;
    for (const Source &s : sources) {
      double p[3];
      s.get_position(p);
      pos.insert(pos.end(), p, p + 3);
      lum.push_back(s.get_luminosity());
      _total_luminosity += s.get_luminosity();
    }
    cmi_check(cmi_set_sources(_ctx, 0, pos.data(), lum.data(), (int32_t)lum.size()));
  }
  double total_luminosity() const { return _total_luminosity; }
  void set_num_photon(uint64_t n) {
    _num_photon = n;
    cmi_check(cmi_set_packet_budget(_ctx, 0, n));
  }
  // reemission_probability (params.txt): absorbed packets are re-emitted with
  // this probability (do_reemission, testDensitySubGrid_omp.cpp:675-702)
  void set_reemission_probability(double p) {
    cmi_check(cmi_set_reemission_probability(_ctx, 0, p));
  }
  // shoot num_photon packets from the sources and solve the balance
  // (testDensitySubGrid_omp.cpp:2213-2434), `iterations` times
  std::vector<cmi_stats> run_iterations(int iterations, uint64_t seed) {
    push();
    std::vector<cmi_stats> st((size_t)iterations);
    cmi_check(cmi_run_iterations(_ctx, iterations, seed, st.data()));
    _host_stale = true;
    return st;
  }
  // iterate until the mean |delta x_H| of an iteration drops below tolerance
  // (no reference counterpart); returns the stats of the iterations run and
  // sets *converged_at (0: not within max_iterations)
  std::vector<cmi_stats> run_until_converged(double tolerance, int max_iterations, uint64_t seed,
                                             int *converged_at, int min_iterations = 2) {
    push();
    std::vector<cmi_stats> st((size_t)max_iterations);
    int32_t done = 0, at = 0;
    cmi_check(cmi_run_until_converged(_ctx, max_iterations, min_iterations, tolerance, seed,
                                      st.data(), &done, &at));
    _host_stale = true;
    st.resize((size_t)done);
    if (converged_at) *converged_at = at;
    return st;
  }
};

class DensitySubGrid {
 private:
  DensityGrid *_grid;
  unsigned int _index;

  size_t offset() const { return (size_t)_index * _grid->cells_per_subgrid(); }
  int three(int a) const {
    const int *ns = _grid->desc().num_subgrid;
    const int i3[3] = {(int)(_index / (ns[1] * ns[2])), (int)((_index / ns[2]) % ns[1]),
                       (int)(_index % ns[2])};
    return i3[a];
  }

 public:
  DensitySubGrid(DensityGrid *grid, unsigned int index) : _grid(grid), _index(index) {}

  size_t get_number_of_cells() const { return _grid->cells_per_subgrid(); }

  // DensitySubGrid.hpp:1116-1141
  void set_number_density(unsigned int index, double v) { _grid->host_nH()[offset() + index] = v; }
  void set_neutral_fraction(unsigned int index, double v) {
    _grid->host_xH()[offset() + index] = v;
  }
  const double *get_neutral_fraction() { return _grid->neutral_fractions() + offset(); }
  double get_intensity_integral(int ix, int iy, int iz) {
    const int *n = _grid->subgrid_cells();
    return _grid->intensity_integrals()[offset() + (size_t)(ix * n[1] + iy) * n[2] + iz];
  }

  // DensitySubGrid.hpp:1042-1049 (box of the subgrid)
  void get_grid_box(double box[6]) const {
    const cmi_grid_desc &d = _grid->desc();
    for (int a = 0; a < 3; ++a) {
      const double side = d.box[3 + a] / d.num_subgrid[a];
      box[a] = d.box[a] + three(a) * side;
      box[3 + a] = side;
    }
  }

  // neighbour table, testDensitySubGrid_omp.cpp:1839-1874
  unsigned int get_neighbour(int direction) const {
    int s[3];
    TravelDirections::signs(direction, s);
    const int *ns = _grid->desc().num_subgrid;
    int c[3];
    for (int a = 0; a < 3; ++a) {
      c[a] = three(a) + s[a];
      if (c[a] < 0 || c[a] >= ns[a]) return NEIGHBOUR_OUTSIDE;
    }
    return (unsigned int)((c[0] * ns[1] + c[1]) * ns[2] + c[2]);
  }

  // DensitySubGrid.hpp:428-469 (position relative to the subgrid anchor)
  int get_start_index(const double *position, int input_direction, int *three_index) const {
    double box[6];
    get_grid_box(box);
    const int *n = _grid->subgrid_cells();
    int s[3];
    TravelDirections::signs(input_direction, s);
    for (int a = 0; a < 3; ++a) {
      const double inv = n[a] / box[3 + a];
      three_index[a] = (s[a] == 0) ? (int)(position[a] * inv) : ((s[a] < 0) ? 0 : n[a] - 1);
    }
    return (three_index[0] * n[1] + three_index[1]) * n[2] + three_index[2];
  }

  // DensitySubGrid.hpp:483-506
  int get_output_direction(const int *three_index) const {
    const int *n = _grid->subgrid_cells();
    int mask = 0;
    for (int a = 0; a < 3; ++a) {
      const int low = three_index[a] < 0;
      const int high = (three_index[a] / n[a]) > 0;
      mask |= (high << (5 - 2 * a)) | (low << (4 - 2 * a));
    }
    return TravelDirections::get_output_direction(mask);
  }

  // DensitySubGrid.hpp:1180-1323, on the GPU
  int interact(Photon &photon, int input_direction) {
    _grid->push();
    int32_t steps = 0, out = -1;
    cmi_check(cmi_trace_packet(_grid->context(), 0, _index, input_direction, photon.raw(), 0,
                               nullptr, nullptr, &steps, &out));
    _grid->mark_device_changed();
    return out;
  }

  // DensitySubGrid.hpp:1333-1472 (interact without the J tally) and :1482-1604
  // (the optical depth of the crossing added to the photon's target depth), on
  // the GPU; the dust driver's per-photon calls
  int propagate(Photon &photon, int input_direction) {
    return walk(photon, input_direction, CMI_WALK_PROPAGATE);
  }
  int compute_optical_depth(Photon &photon, int input_direction) {
    return walk(photon, input_direction, CMI_WALK_OPTICAL_DEPTH);
  }

  // DensitySubGrid.hpp:1628-1658, this subgrid only
  void compute_neutral_fraction(double luminosity, unsigned int num_photon) {
    _grid->push();
    cmi_check(cmi_compute_neutral_fraction_subgrids(_grid->context(), 0, _index, 1, luminosity,
                                                    num_photon, nullptr));
    _grid->mark_device_changed();
  }

  // Result-file records (DensitySubGrid.hpp:1738-1796, NO_HYDRO build): per
  // cell in index order the centre x, y, z, x_H and n_H as FP64, then five
  // zero 4-byte hydro slots; 60 bytes per cell.
  size_t get_output_size() const { return get_number_of_cells() * (5 * sizeof(double) + 20); }
  void output_intensities(std::ostream &stream) {
    double box[6];
    get_grid_box(box);
    const int *n = _grid->subgrid_cells();
    double cs[3];
    for (int a = 0; a < 3; ++a) cs[a] = box[3 + a] / n[a];
    const double *x = _grid->neutral_fractions() + offset();
    const double *nh = _grid->number_densities() + offset();
    const char zeros[20] = {0};
    for (int ix = 0; ix < n[0]; ++ix) {
      const double px = box[0] + (ix + 0.5) * cs[0];
      for (int iy = 0; iy < n[1]; ++iy) {
        const double py = box[1] + (iy + 0.5) * cs[1];
        for (int iz = 0; iz < n[2]; ++iz) {
          const double pz = box[2] + (iz + 0.5) * cs[2];
          const size_t c = (size_t)(ix * n[1] + iy) * n[2] + iz;
          const double rec[5] = {px, py, pz, x[c], nh[c]};
          stream.write(reinterpret_cast<const char *>(rec), sizeof(rec));
          stream.write(zeros, sizeof(zeros));
        }
      }
    }
  }

  unsigned int index() const { return _index; }
  DensityGrid *grid() { return _grid; }

 private:
  int walk(Photon &photon, int input_direction, int mode) {
    _grid->push();
    const int32_t in_dir = input_direction;
    int32_t out = -1;
    cmi_check(cmi_walk_photons(_grid->context(), 0, _index, mode, photon.raw(), &in_dir, 1, &out));
    return out;
  }
};

// The reference driver's result files (testDensitySubGrid_omp.cpp:394-521):
// neutral_fractions.dat (the records above, subgrid after subgrid) and
// neutral_fractions.bin (x_H as FP64 in the same order).  Return the bytes
// written.
inline size_t output_neutral_fractions(DensityGrid &grid, const char *path) {
  std::ofstream out(path, std::ios::binary);
  size_t size = 0;
  for (unsigned int s = 0; s < grid.number_of_subgrids(); ++s) {
    DensitySubGrid sg = grid.subgrid(s);
    sg.output_intensities(out);
    size += sg.get_output_size();
  }
  if (!out) throw std::runtime_error(std::string("cannot write ") + path);
  return size;
}

inline size_t output_neutral_fractions_binary(DensityGrid &grid, const char *path) {
  std::ofstream out(path, std::ios::binary);
  const size_t n = grid.cells_per_subgrid() * grid.number_of_subgrids();
  out.write(reinterpret_cast<const char *>(grid.neutral_fractions()), sizeof(double) * n);
  if (!out) throw std::runtime_error(std::string("cannot write ") + path);
  return sizeof(double) * n;
}

inline DensitySubGrid DensityGrid::subgrid(unsigned int index) {
  if (index >= number_of_subgrids()) throw std::runtime_error("subgrid index out of range");
  return DensitySubGrid(this, index);
}

/* do_photon_traversal (testDensitySubGrid_omp.cpp:607-666): every photon of
 * the input buffer through the subgrid; results appended to the 27 output
 * buffers whose flag is set (the others' photons are done: absorbed or
 * escaped). */
inline void do_photon_traversal(PhotonBuffer &input_buffer, DensitySubGrid &subgrid,
                                PhotonBuffer *output_buffers, bool *output_buffer_flags) {
  subgrid.grid()->push();
  uint8_t enabled[TRAVELDIRECTION_NUMBER];
  for (int i = 0; i < TRAVELDIRECTION_NUMBER; ++i) enabled[i] = output_buffer_flags[i] ? 1 : 0;
  std::vector<Photon> out(input_buffer.size() > 0 ? input_buffer.size() : 1);
  uint32_t counts[TRAVELDIRECTION_NUMBER];
  uint32_t done = 0;
  cmi_check(cmi_traverse_buffer(subgrid.grid()->context(), 0, subgrid.index(),
                                input_buffer.get_direction(), input_buffer.data()->raw(),
                                input_buffer.size(), enabled, out.data()->raw(), counts, &done));
  subgrid.grid()->mark_device_changed();
  size_t k = 0;
  for (int d = 0; d < TRAVELDIRECTION_NUMBER; ++d) {
    for (uint32_t i = 0; i < counts[d]; ++i) {
      PhotonBuffer &b = output_buffers[d];
      b[b.get_next_free_photon()] = out[k++];
    }
  }
}

#endif
