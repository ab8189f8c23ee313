/*
 * Reference harness (test infrastructure).  Compiled by oracle/build_ref.sh
 * directly against the reference's own headers (DensitySubGrid.hpp,
 * Photon.hpp, RandomGenerator.hpp, TravelDirections.hpp), which stay where
 * they are; the binary goes to oracle/_ref/.  It serves two purposes:
 *
 *  1. golden vectors: runs the reference's own functions on inputs written
 *     by the test-fixture generator and writes their outputs, so the C oracle
 *     (cmi_oracle.c) and the CUDA path can be pinned to the reference;
 *  2. the timed CPU baseline: whole iterations of the plain method on all
 *     host cores, using the reference's DensitySubGrid::interact,
 *     compute_neutral_fraction and its subgrid-copy merge
 *     (update_intensities / update_neutral_fractions).
 *
 * Only get_random_direction (testDensitySubGrid_omp.cpp:529-545), the
 * luminosity split (:2199-2208) and do_reemission (:675-702) live next to
 * main() in the reference driver; they are restated below with citations.
 *
 * All binary I/O is little-endian, fixed-width.
 */
#define NO_HYDRO
int MPI_rank = 0, MPI_size = 1;

#include "DensitySubGrid.hpp"
#include "Photon.hpp"
#include "RandomGenerator.hpp"
#include "TravelDirections.hpp"

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <omp.h>

extern "C" {
#include "cmi_oracle.h"
}

namespace {

struct Reader {
  FILE *f;
  explicit Reader(const char *path) : f(std::fopen(path, "rb")) {
    if (!f) {
      std::fprintf(stderr, "cannot open %s\n", path);
      std::exit(2);
    }
  }
  ~Reader() { std::fclose(f); }
  template <class T> T get() {
    T v;
    if (std::fread(&v, sizeof(T), 1, f) != 1) {
      std::fprintf(stderr, "short read\n");
      std::exit(2);
    }
    return v;
  }
  template <class T> void get(T *dst, size_t n) {
    if (n && std::fread(dst, sizeof(T), n, f) != n) {
      std::fprintf(stderr, "short read\n");
      std::exit(2);
    }
  }
};

struct Writer {
  FILE *f;
  explicit Writer(const char *path) : f(std::fopen(path, "wb")) {
    if (!f) {
      std::fprintf(stderr, "cannot open %s\n", path);
      std::exit(2);
    }
  }
  ~Writer() { std::fclose(f); }
  template <class T> void put(const T &v) { std::fwrite(&v, sizeof(T), 1, f); }
  template <class T> void put(const T *src, size_t n) {
    if (n) std::fwrite(src, sizeof(T), n, f);
  }
};

/* 80-byte record shared with the tests (same field order as Photon). */
struct PhotonRecord {
  double position[3];
  double direction[3];
  double tau;
  double sigma;
  double weight;
  int32_t type;
  int32_t reserved;
};
static_assert(sizeof(PhotonRecord) == 80, "photon record");

void to_photon(const PhotonRecord &r, Photon &p) {
  p.set_position(r.position[0], r.position[1], r.position[2]);
  p.set_direction(r.direction[0], r.direction[1], r.direction[2]);
  p.set_target_optical_depth(r.tau);
  p.set_photoionization_cross_section(r.sigma);
  p.set_weight(r.weight);
  p.set_type(r.type);
}

PhotonRecord from_photon(const Photon &p) {
  PhotonRecord r;
  std::memset(&r, 0, sizeof(r));
  for (int a = 0; a < 3; ++a) {
    r.position[a] = p.get_position()[a];
    r.direction[a] = p.get_direction()[a];
  }
  r.tau = p.get_target_optical_depth();
  r.sigma = p.get_photoionization_cross_section();
  r.weight = p.get_weight();
  r.type = (int32_t)p.get_type();
  return r;
}

/* testDensitySubGrid_omp.cpp:529-545 (restated: it lives beside main()). */
void random_direction(RandomGenerator &rng, double *direction) {
  const double cost = 2. * rng.get_uniform_random_double() - 1.;
  const double phi = 2. * M_PI * rng.get_uniform_random_double();
  const double sint = std::sqrt(std::max(1. - cost * cost, 0.));
  direction[0] = sint * std::cos(phi);
  direction[1] = sint * std::sin(phi);
  direction[2] = cost;
}

/* testDensitySubGrid_omp.cpp:556-597 (restated), for one photon. */
void emit_photon(RandomGenerator &rng, const double *src, Photon &photon) {
  photon.set_position(src[0], src[1], src[2]);
  random_direction(rng, photon.get_direction());
  photon.set_weight(1.);
  photon.set_target_optical_depth(-std::log(rng.get_uniform_random_double()));
  photon.set_photoionization_cross_section(6.3e-22);
  photon.set_type(PHOTONPACKETTYPE_DIRECT);
}

/* do_reemission (testDensitySubGrid_omp.cpp:675-702, restated) for one
 * absorbed photon: with probability p a new isotropic direction and target
 * optical depth; returns whether it was re-emitted. */
bool reemit_photon(RandomGenerator &rng, double p, Photon &photon) {
  if (!(rng.get_uniform_random_double() < p)) return false;
  random_direction(rng, photon.get_direction());
  photon.set_target_optical_depth(-std::log(rng.get_uniform_random_double()));
  return true;
}

/* ---- directions: testDensitySubGridDirections.cpp fixtures + sweeps ---- */
int cmd_directions(const char *out_path) {
  const double testbox[6] = {0., 0., 0., 1., 1., 1.};
  const int testncell[3] = {10, 10, 10};
  DensitySubGrid grid(testbox, testncell);
  FILE *f = std::fopen(out_path, "w");
  // every in-range/out-of-range combination of a 10^3 grid
  const int probe[3] = {-1, 4, 10};
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      for (int c = 0; c < 3; ++c) {
        const int ti[3] = {probe[a], probe[b], probe[c]};
        std::fprintf(f, "output %d %d %d %d\n", ti[0], ti[1], ti[2],
                     grid.get_output_direction(ti));
      }
  // start index for every input direction on the matching face/edge/corner
  // and for off-face coordinates
  const double coords[5] = {0., 0.05, 0.5, 0.95, 1.};
  for (int dir = 0; dir < TRAVELDIRECTION_NUMBER; ++dir) {
    for (int a = 0; a < 5; ++a)
      for (int b = 0; b < 5; ++b)
        for (int c = 0; c < 5; ++c) {
          const double pos[3] = {coords[a], coords[b], coords[c]};
          int ti[3];
          // the reference asserts are off in this harness: clamped axes
          // are taken from the direction, the rest truncated
          grid.get_start_index(pos, dir, ti);
          std::fprintf(f, "start %d %.17g %.17g %.17g %d %d %d\n", dir, pos[0], pos[1],
                       pos[2], ti[0], ti[1], ti[2]);
        }
  }
  for (int dir = 0; dir < TRAVELDIRECTION_NUMBER; ++dir) {
    std::fprintf(f, "mirror %d %d\n", dir, TravelDirections::output_to_input_direction(dir));
  }
  const double dvals[3] = {-0.5, 0., 0.5};
  for (int dir = 0; dir < TRAVELDIRECTION_NUMBER; ++dir)
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        for (int c = 0; c < 3; ++c) {
          const double d[3] = {dvals[a], dvals[b], dvals[c]};
          std::fprintf(f, "compat %d %g %g %g %d %d\n", dir, d[0], d[1], d[2],
                       (int)TravelDirections::is_compatible_input_direction(d, dir),
                       (int)TravelDirections::is_compatible_output_direction(d, dir));
        }
  std::fclose(f);
  return 0;
}

/* ---- rng: RandomGenerator streams ---- */
int cmd_rng(int seed, long n, const char *out_path) {
  RandomGenerator rng(seed);
  Writer w(out_path);
  for (long i = 0; i < n; ++i) {
    w.put(rng.get_uniform_random_double());
  }
  return 0;
}

/* ---- emit: one buffer stream (seed; one copy-pick draw; n photons) ---- */
int cmd_emit(int seed, int n, double sx, double sy, double sz, const char *out_path) {
  RandomGenerator rng(seed);
  (void)rng.get_uniform_random_double();
  const double src[3] = {sx, sy, sz};
  Writer w(out_path);
  for (int i = 0; i < n; ++i) {
    Photon p;
    emit_photon(rng, src, p);
    w.put(from_photon(p));
  }
  return 0;
}

/* ---- walk: DensitySubGrid::interact on a list of photons ----
 * in:  box[6] ncell[3] pad nH[C] xH[C] n {PhotonRecord, int32 in_dir}*n
 * out: {PhotonRecord, int32 result}*n, J[C] (all packets in order), then per
 *      packet: int32 count, {int32 cell, double J}*count on a fresh grid. */
int cmd_walk(const char *in_path, const char *out_path) {
  Reader r(in_path);
  double box[6];
  r.get(box, 6);
  int ncell[3];
  r.get(ncell, 3);
  (void)r.get<int32_t>();
  const long C = (long)ncell[0] * ncell[1] * ncell[2];
  std::vector<double> nH(C), xH(C);
  r.get(nH.data(), C);
  r.get(xH.data(), C);
  const long n = r.get<int64_t>();
  std::vector<PhotonRecord> in(n);
  std::vector<int32_t> in_dir(n);
  for (long i = 0; i < n; ++i) {
    in[i] = r.get<PhotonRecord>();
    in_dir[i] = r.get<int32_t>();
  }
  DensitySubGrid grid(box, ncell), fresh(box, ncell);
  for (long c = 0; c < C; ++c) {
    grid.set_number_density(c, nH[c]);
    grid.set_neutral_fraction(c, xH[c]);
    fresh.set_number_density(c, nH[c]);
    fresh.set_neutral_fraction(c, xH[c]);
  }
  Writer w(out_path);
  for (long i = 0; i < n; ++i) {
    Photon p;
    to_photon(in[i], p);
    const int res = grid.interact(p, in_dir[i]);
    w.put(from_photon(p));
    w.put((int32_t)res);
  }
  for (int ix = 0; ix < ncell[0]; ++ix)
    for (int iy = 0; iy < ncell[1]; ++iy)
      for (int iz = 0; iz < ncell[2]; ++iz) {
        w.put(grid.get_intensity_integral(ix, iy, iz));
      }
  for (long i = 0; i < n; ++i) {
    for (long c = 0; c < C; ++c) fresh.set_intensity_integral(c, 0.);
    Photon p;
    to_photon(in[i], p);
    (void)fresh.interact(p, in_dir[i]);
    std::vector<int32_t> cells;
    std::vector<double> vals;
    for (int ix = 0; ix < ncell[0]; ++ix)
      for (int iy = 0; iy < ncell[1]; ++iy)
        for (int iz = 0; iz < ncell[2]; ++iz) {
          const double v = fresh.get_intensity_integral(ix, iy, iz);
          if (v != 0.) {
            cells.push_back((ix * ncell[1] + iy) * ncell[2] + iz);
            vals.push_back(v);
          }
        }
    w.put((int32_t)cells.size());
    for (size_t k = 0; k < cells.size(); ++k) {
      w.put(cells[k]);
      w.put(vals[k]);
    }
  }
  return 0;
}

/* ---- balance: compute_neutral_fraction ----
 * in: box[6] ncell[3] pad L N(uint32) pad nH[C] J[C];  out: xH[C] J[C] */
int cmd_balance(const char *in_path, const char *out_path) {
  Reader r(in_path);
  double box[6];
  r.get(box, 6);
  int ncell[3];
  r.get(ncell, 3);
  (void)r.get<int32_t>();
  const double L = r.get<double>();
  const unsigned int N = r.get<uint32_t>();
  (void)r.get<int32_t>();
  const long C = (long)ncell[0] * ncell[1] * ncell[2];
  std::vector<double> nH(C), J(C);
  r.get(nH.data(), C);
  r.get(J.data(), C);
  DensitySubGrid grid(box, ncell);
  for (long c = 0; c < C; ++c) {
    grid.set_number_density(c, nH[c]);
    grid.set_intensity_integral(c, J[c]);
  }
  grid.compute_neutral_fraction(L, N);
  Writer w(out_path);
  w.put(grid.get_neutral_fraction(), C);
  for (int ix = 0; ix < ncell[0]; ++ix)
    for (int iy = 0; iy < ncell[1]; ++iy)
      for (int iz = 0; iz < ncell[2]; ++iz) w.put(grid.get_intensity_integral(ix, iy, iz));
  return 0;
}

/* Subgrids + neighbour table exactly as testDensitySubGrid_omp.cpp:1801-1877,
 * fields in subgrid-blocked order. */
std::vector<DensitySubGrid *> build_lattice(const double *box, const int *ncell, const int *nsub,
                                            const std::vector<double> &nH,
                                            const std::vector<double> &xH) {
  const int sub_ncell[3] = {ncell[0] / nsub[0], ncell[1] / nsub[1], ncell[2] / nsub[2]};
  const long C = (long)sub_ncell[0] * sub_ncell[1] * sub_ncell[2];
  const long S = (long)nsub[0] * nsub[1] * nsub[2];
  const double side[3] = {box[3] / nsub[0], box[4] / nsub[1], box[5] / nsub[2]};
  std::vector<DensitySubGrid *> grid(S);
  for (long s = 0; s < S; ++s) {
    const int ix = s / (nsub[1] * nsub[2]);
    const int iy = (s - ix * nsub[1] * nsub[2]) / nsub[2];
    const int iz = s - ix * nsub[1] * nsub[2] - iy * nsub[2];
    const double sbox[6] = {box[0] + ix * side[0], box[1] + iy * side[1], box[2] + iz * side[2],
                            side[0], side[1], side[2]};
    grid[s] = new DensitySubGrid(sbox, sub_ncell);
    for (int d = 0; d < TRAVELDIRECTION_NUMBER; ++d) grid[s]->set_neighbour(d, NEIGHBOUR_OUTSIDE);
    for (int nx = -1; nx < 2; ++nx)
      for (int ny = -1; ny < 2; ++ny)
        for (int nz = -1; nz < 2; ++nz) {
          const int cx = ix + nx, cy = iy + ny, cz = iz + nz;
          if (cx >= 0 && cx < nsub[0] && cy >= 0 && cy < nsub[1] && cz >= 0 && cz < nsub[2]) {
            const int ti[3] = {nx * sub_ncell[0], ny * sub_ncell[1], nz * sub_ncell[2]};
            grid[s]->set_neighbour(grid[s]->get_output_direction(ti),
                                   (cx * nsub[1] + cy) * nsub[2] + cz);
          }
        }
    for (long c = 0; c < C; ++c) {
      grid[s]->set_number_density(c, nH[s * C + c]);
      grid[s]->set_neutral_fraction(c, xH[s * C + c]);
    }
  }
  return grid;
}

/* ---- transport: packets through the lattice (serial, in order) ----
 * in:  box[6] ncell[3] nsub[3] n(int64) nH[cells] xH[cells]
 *      {PhotonRecord, uint32 start_subgrid, int32 pad}*n
 * out: J[cells, blocked], {PhotonRecord final, int32 fate(0 absorbed,1 escaped),
 *      int32 transits}*n */
int cmd_transport(const char *in_path, const char *out_path) {
  Reader r(in_path);
  double box[6];
  r.get(box, 6);
  int ncell[3], nsub[3];
  r.get(ncell, 3);
  r.get(nsub, 3);
  const long n = r.get<int64_t>();
  const long cells = (long)ncell[0] * ncell[1] * ncell[2];
  std::vector<double> nH(cells), xH(cells);
  r.get(nH.data(), cells);
  r.get(xH.data(), cells);
  std::vector<DensitySubGrid *> grid = build_lattice(box, ncell, nsub, nH, xH);
  Writer w(out_path);
  std::vector<PhotonRecord> fin(n);
  std::vector<int32_t> fate(n), transits(n);
  for (long i = 0; i < n; ++i) {
    const PhotonRecord rec = r.get<PhotonRecord>();
    unsigned int s = r.get<uint32_t>();
    (void)r.get<int32_t>();
    Photon photon;
    to_photon(rec, photon);
    int in_dir = TRAVELDIRECTION_INSIDE;
    int tr = 0;
    for (;;) {
      const int res = grid[s]->interact(photon, in_dir);
      ++tr;
      if (res == TRAVELDIRECTION_INSIDE) {
        fate[i] = 0;
        break;
      }
      const unsigned int ngb = grid[s]->get_neighbour(res);
      if (ngb == NEIGHBOUR_OUTSIDE) {
        fate[i] = 1;
        break;
      }
      s = ngb;
      in_dir = TravelDirections::output_to_input_direction(res);
    }
    fin[i] = from_photon(photon);
    transits[i] = tr;
  }
  const int sub_ncell[3] = {ncell[0] / nsub[0], ncell[1] / nsub[1], ncell[2] / nsub[2]};
  for (size_t s = 0; s < grid.size(); ++s)
    for (int ix = 0; ix < sub_ncell[0]; ++ix)
      for (int iy = 0; iy < sub_ncell[1]; ++iy)
        for (int iz = 0; iz < sub_ncell[2]; ++iz) w.put(grid[s]->get_intensity_integral(ix, iy, iz));
  for (long i = 0; i < n; ++i) {
    w.put(fin[i]);
    w.put(fate[i]);
    w.put(transits[i]);
  }
  for (auto *g : grid) delete g;
  return 0;
}

/* ---- run: whole plain-method iterations on the host cores ----
 * in:  box[6] ncell[3] nsub[3] nsrc(int32) pad nH[cells, subgrid-blocked]
 *      xH[cells] {pos[3], L}*nsrc
 * args: packets iterations threads seed count(0/1) [reemission_probability]
 * out: xH[cells] after the last iteration, then per iteration
 *      {double mc_seconds, uint64 crossings, uint64 absorbed, uint64 escaped}
 *
 * Each thread owns a copy of every subgrid (DensitySubGrid copy constructor,
 * the reference's hot-subgrid replication taken to one copy per thread);
 * the copies are merged with update_intensities and refreshed with
 * update_neutral_fractions exactly as testDensitySubGrid_omp.cpp:2403-2434.
 * Buffer b (200 packets) of an iteration draws from RandomGenerator(seed +
 * b); count=1 replays every buffer through the C oracle walk (untimed) to
 * count cell crossings, which the reference walk does not report (without
 * reemission only).  With reemission probability p > 0 an absorbed photon is
 * re-emitted in place (do_reemission, :675-702; the reemit task :1348-1395
 * walks it on through the same subgrid), drawing from its buffer's
 * generator. */
int cmd_run(const char *in_path, const char *out_path, long packets, int iterations,
            int threads, int seed, int count, double reemission) {
  if (count && reemission > 0.) {
    std::fprintf(stderr, "run: crossing counts need reemission 0\n");
    return 2;
  }
  Reader r(in_path);
  double box[6];
  r.get(box, 6);
  int ncell[3], nsub[3];
  r.get(ncell, 3);
  r.get(nsub, 3);
  const int nsrc = r.get<int32_t>();
  (void)r.get<int32_t>();
  const int sub_ncell[3] = {ncell[0] / nsub[0], ncell[1] / nsub[1], ncell[2] / nsub[2]};
  const long C = (long)sub_ncell[0] * sub_ncell[1] * sub_ncell[2];
  const long S = (long)nsub[0] * nsub[1] * nsub[2];
  std::vector<double> nH(C * S), xH(C * S);
  r.get(nH.data(), C * S);
  r.get(xH.data(), C * S);
  std::vector<double> src_pos(3 * nsrc), src_lum(nsrc);
  for (int i = 0; i < nsrc; ++i) {
    r.get(&src_pos[3 * i], 3);
    src_lum[i] = r.get<double>();
  }
  if (threads <= 0) threads = omp_get_max_threads();
  omp_set_num_threads(threads);

  std::vector<DensitySubGrid *> grid = build_lattice(box, ncell, nsub, nH, xH);
  std::vector<std::vector<DensitySubGrid *>> copies(threads);
  for (int t = 0; t < threads; ++t) {
    copies[t].resize(S);
    for (long s = 0; s < S; ++s) copies[t][s] = new DensitySubGrid(*grid[s]);
    for (long s = 0; s < S; ++s)
      for (int d = 0; d < TRAVELDIRECTION_NUMBER; ++d)
        copies[t][s]->set_neighbour(d, grid[s]->get_neighbour(d));
  }
  // sources: subgrid containing each source (:1983-1996) and the
  // luminosity split (:2199-2208); the remainder goes to the first sources
  std::vector<unsigned int> src_sub(nsrc);
  double total_lum = 0.;
  for (int i = 0; i < nsrc; ++i) {
    unsigned int si[3];
    for (int a = 0; a < 3; ++a) {
      long v = (long)((src_pos[3 * i + a] - box[a]) / box[3 + a] * nsub[a]);
      si[a] = (unsigned int)std::min<long>(std::max<long>(v, 0), nsub[a] - 1);
    }
    src_sub[i] = (si[0] * nsub[1] + si[1]) * nsub[2] + si[2];
    total_lum += src_lum[i];
  }
  std::vector<long> src_num(nsrc);
  long assigned = 0;
  for (int i = 0; i < nsrc; ++i) {
    src_num[i] = (long)(unsigned int)(src_lum[i] / total_lum * packets);
    assigned += src_num[i];
  }
  for (long k = 0; k < packets - assigned; ++k) src_num[k % nsrc] += 1;
  // buffers of 200 packets (PHOTONBUFFER_SIZE, PhotonBuffer.hpp:42)
  struct Buf { int src; int n; };
  std::vector<Buf> bufs;
  for (int i = 0; i < nsrc; ++i)
    for (long done = 0; done < src_num[i]; done += 200)
      bufs.push_back({i, (int)std::min<long>(200, src_num[i] - done)});
  const long nbuf = (long)bufs.size();

  // oracle lattice for crossing counts
  cmio_lattice lat;
  const int32_t nc32[3] = {ncell[0], ncell[1], ncell[2]}, ns32[3] = {nsub[0], nsub[1], nsub[2]};
  cmio_lattice_init(&lat, box, nc32, ns32);

  Writer w(out_path);
  std::vector<double> times;
  std::vector<uint64_t> crossings, absorbed, escaped;
  for (int it = 0; it < iterations; ++it) {
    const auto t0 = std::chrono::steady_clock::now();
    uint64_t n_abs = 0, n_esc = 0;
#pragma omp parallel reduction(+ : n_abs, n_esc)
    {
      const int t = omp_get_thread_num();
      std::vector<DensitySubGrid *> &mine = copies[t];
#pragma omp for schedule(dynamic, 1)
      for (long b = 0; b < nbuf; ++b) {
        RandomGenerator rng(seed + (int)b + it * (int)nbuf);
        (void)rng.get_uniform_random_double();
        const double *src = &src_pos[3 * bufs[b].src];
        for (int k = 0; k < bufs[b].n; ++k) {
          Photon photon;
          emit_photon(rng, src, photon);
          unsigned int s = src_sub[bufs[b].src];
          int in_dir = TRAVELDIRECTION_INSIDE;
          for (;;) {
            const int res = mine[s]->interact(photon, in_dir);
            if (res == TRAVELDIRECTION_INSIDE) {
              if (reemission > 0. && reemit_photon(rng, reemission, photon)) {
                in_dir = TRAVELDIRECTION_INSIDE;
                continue;
              }
              ++n_abs;
              break;
            }
            const unsigned int ngb = mine[s]->get_neighbour(res);
            if (ngb == NEIGHBOUR_OUTSIDE) {
              ++n_esc;
              break;
            }
            s = ngb;
            in_dir = TravelDirections::output_to_input_direction(res);
          }
        }
      }
    }
    // merge the copies and solve the balance (:2403-2434)
#pragma omp parallel for schedule(static)
    for (long s = 0; s < S; ++s) {
      for (int t = 0; t < threads; ++t) grid[s]->update_intensities(*copies[t][s]);
      grid[s]->compute_neutral_fraction(total_lum, (unsigned int)packets);
      for (int t = 0; t < threads; ++t) copies[t][s]->update_neutral_fractions(*grid[s]);
    }
    const auto t1 = std::chrono::steady_clock::now();
    times.push_back(std::chrono::duration<double>(t1 - t0).count());
    absorbed.push_back(n_abs);
    escaped.push_back(n_esc);
    uint64_t n_cross = 0;
    if (count) {
      // replay the same packets through the oracle walk on the field this
      // iteration's transport saw (xH is refreshed only below), untimed
#pragma omp parallel reduction(+ : n_cross)
      {
        std::vector<double> Jt(C * S, 0.);
#pragma omp for schedule(dynamic, 1)
        for (long b = 0; b < nbuf; ++b) {
          RandomGenerator rng(seed + (int)b + it * (int)nbuf);
          (void)rng.get_uniform_random_double();
          const double *src = &src_pos[3 * bufs[b].src];
          for (int k = 0; k < bufs[b].n; ++k) {
            Photon photon;
            emit_photon(rng, src, photon);
            const PhotonRecord rec = from_photon(photon);
            cmio_photon op;
            std::memcpy(&op, &rec, sizeof(op));
            cmio_counts cc = {0, 0, 0, 0};
            const uint32_t s0 = src_sub[bufs[b].src];
            cmio_transport(&lat, nH.data(), xH.data(), Jt.data(), &op, &s0, 1, &cc);
            n_cross += cc.crossings;
          }
        }
      }
    }
    crossings.push_back(n_cross);
    // field seen by the next iteration's transport (for the replay count)
    for (long s = 0; s < S; ++s) {
      const double *x = grid[s]->get_neutral_fraction();
      std::memcpy(&xH[s * C], x, sizeof(double) * C);
    }
  }
  w.put(xH.data(), C * S);
  for (int it = 0; it < iterations; ++it) {
    w.put(times[it]);
    w.put(crossings[it]);
    w.put(absorbed[it]);
    w.put(escaped[it]);
  }
  cmio_lattice_free(&lat);
  for (int t = 0; t < threads; ++t)
    for (long s = 0; s < S; ++s) delete copies[t][s];
  for (long s = 0; s < S; ++s) delete grid[s];
  return 0;
}

}  // namespace

/* ---- dust walks: DensitySubGrid::propagate (DensitySubGrid.hpp:1333) or
 * DensitySubGrid::compute_optical_depth (:1482) on a list of photons, each on
 * the same grid ----
 * in:  as cmd_walk
 * out: {PhotonRecord, int32 result}*n */
int cmd_dust_walk(const char *in_path, const char *out_path, bool depth) {
  Reader r(in_path);
  double box[6];
  r.get(box, 6);
  int ncell[3];
  r.get(ncell, 3);
  (void)r.get<int32_t>();
  const long C = (long)ncell[0] * ncell[1] * ncell[2];
  std::vector<double> nH(C), xH(C);
  r.get(nH.data(), C);
  r.get(xH.data(), C);
  const long n = r.get<int64_t>();
  DensitySubGrid grid(box, ncell);
  for (long c = 0; c < C; ++c) {
    grid.set_number_density(c, nH[c]);
    grid.set_neutral_fraction(c, xH[c]);
  }
  Writer w(out_path);
  for (long i = 0; i < n; ++i) {
    const PhotonRecord rec = r.get<PhotonRecord>();
    const int32_t in_dir = r.get<int32_t>();
    Photon p;
    to_photon(rec, p);
    const int res = depth ? grid.compute_optical_depth(p, in_dir) : grid.propagate(p, in_dir);
    w.put(from_photon(p));
    w.put((int32_t)res);
  }
  return 0;
}

int main(int argc, char **argv) {
  if (argc < 2) {
    std::fprintf(stderr,
                 "usage: ref_harness directions OUT | rng SEED N OUT | emit SEED N X Y Z OUT |\n"
                 "       walk IN OUT | balance IN OUT | transport IN OUT |\n"
                 "       run IN OUT PACKETS ITERS THREADS SEED "
                 "COUNT\n");
    return 2;
  }
  const std::string cmd = argv[1];
  if (cmd == "directions" && argc == 3) return cmd_directions(argv[2]);
  if (cmd == "rng" && argc == 5) return cmd_rng(std::atoi(argv[2]), std::atol(argv[3]), argv[4]);
  if (cmd == "emit" && argc == 8)
    return cmd_emit(std::atoi(argv[2]), std::atoi(argv[3]), std::atof(argv[4]),
                    std::atof(argv[5]), std::atof(argv[6]), argv[7]);
  if (cmd == "walk" && argc == 4) return cmd_walk(argv[2], argv[3]);
  if (cmd == "propagate" && argc == 4) return cmd_dust_walk(argv[2], argv[3], false);
  if (cmd == "depth" && argc == 4) return cmd_dust_walk(argv[2], argv[3], true);
  if (cmd == "balance" && argc == 4) return cmd_balance(argv[2], argv[3]);
  if (cmd == "transport" && argc == 4) return cmd_transport(argv[2], argv[3]);
  if (cmd == "run" && (argc == 9 || argc == 10))
    return cmd_run(argv[2], argv[3], std::atol(argv[4]), std::atoi(argv[5]), std::atoi(argv[6]),
                   std::atoi(argv[7]), std::atoi(argv[8]), argc == 10 ? std::atof(argv[9]) : 0.);
  std::fprintf(stderr, "bad arguments\n");
  return 2;
}
