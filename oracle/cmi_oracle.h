/*
 * CPU oracle for the photon-packet transport + ionization-balance path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithm (bwvdnbro/ParallelCMacIonize) used to check the CUDA product
 * path.  Only tests/, the smoke check and the CPU-baseline leg of bench.py
 * may load it; the product library never links or calls it.
 *
 * Pinning: every function here is checked against golden vectors produced by
 * the reference's own headers compiled from source (oracle/ref_harness.cpp,
 * built by oracle/build_ref.sh) and against the 54 known answers of
 * testDensitySubGridDirections.cpp:105-167.
 */
#ifndef CMI_ORACLE_H
#define CMI_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* TravelDirection numbering, TravelDirections.hpp:46-75. */
enum {
  CMIO_INSIDE = 0,
  CMIO_CORNER_PPP, CMIO_CORNER_PPN, CMIO_CORNER_PNP, CMIO_CORNER_PNN,
  CMIO_CORNER_NPP, CMIO_CORNER_NPN, CMIO_CORNER_NNP, CMIO_CORNER_NNN,
  CMIO_EDGE_X_PP, CMIO_EDGE_X_PN, CMIO_EDGE_X_NP, CMIO_EDGE_X_NN,
  CMIO_EDGE_Y_PP, CMIO_EDGE_Y_PN, CMIO_EDGE_Y_NP, CMIO_EDGE_Y_NN,
  CMIO_EDGE_Z_PP, CMIO_EDGE_Z_PN, CMIO_EDGE_Z_NP, CMIO_EDGE_Z_NN,
  CMIO_FACE_X_P, CMIO_FACE_X_N, CMIO_FACE_Y_P, CMIO_FACE_Y_N,
  CMIO_FACE_Z_P, CMIO_FACE_Z_N,
  CMIO_NUM_DIRECTIONS
};

#define CMIO_NEIGHBOUR_OUTSIDE 0xffffffffu

/* Same 80-byte layout as the reference Photon (Photon.hpp:49-68). */
typedef struct {
  double position[3];
  double direction[3];
  double target_optical_depth;
  double cross_section;
  double weight;
  int32_t type;
  int32_t reserved;
} cmio_photon;

/* Geometry of one subgrid (DensitySubGrid.hpp:97-160, photoionization part). */
typedef struct {
  double anchor[3];
  double cell_size[3];
  double inv_cell_size[3];
  int32_t ncell[4]; /* nx, ny, nz, ny*nz */
} cmio_subgrid;

/* ---- TravelDirections.hpp ---- */
int cmio_output_to_input_direction(int output_direction);
int cmio_direction_from_mask(int mask);
int cmio_is_compatible_input_direction(const double *direction, int input_direction);
int cmio_is_compatible_output_direction(const double *direction, int output_direction);

/* ---- DensitySubGrid.hpp geometry ---- */
void cmio_subgrid_init(cmio_subgrid *sg, const double box[6], const int32_t ncell[3]);
int cmio_get_start_index(const cmio_subgrid *sg, const double position[3],
                         int input_direction, int32_t three_index[3]);
int cmio_get_output_direction(const cmio_subgrid *sg, const int32_t three_index[3]);

/* FP64 cell walk, DensitySubGrid::interact (DensitySubGrid.hpp:1180-1323).
 * Optional trace: cells/lengths receive the visited cell index and the path
 * length lmin (m) of every loop iteration (at most max_steps entries). */
int cmio_interact(const cmio_subgrid *sg, const double *nH, const double *xH,
                  double *J, cmio_photon *photon, int input_direction,
                  int32_t *trace_cells, double *trace_lengths, int32_t max_steps,
                  int32_t *nsteps);

/* DensitySubGrid::propagate (DensitySubGrid.hpp:1333-1472: interact without the J
 * tally) and DensitySubGrid::compute_optical_depth (:1482-1604: no target; the depth
 * of the crossing is added to target_optical_depth). */
int cmio_propagate(const cmio_subgrid *sg, const double *nH, const double *xH,
                   cmio_photon *photon, int input_direction, int32_t *nsteps);
int cmio_compute_optical_depth(const cmio_subgrid *sg, const double *nH, const double *xH,
                               cmio_photon *photon, int input_direction, int32_t *nsteps);

/* FP32 cell-unit walk used by the CUDA single-precision transport (the
 * project's own formulation; restated here so the GPU kernel can be checked
 * bit for bit).  pos is in cell units relative to the subgrid; kappa is
 * sigma*n*x per cell (1/m) in float.  Tally receives path lengths (m). */
typedef struct {
  float pos[3];
  float dir[3];
  float tau_left;
  uint32_t meta; /* low 5 bits: input TravelDirection */
} cmio_packet32;

/* tally (may be NULL): double sum of the FP32 path lengths.  fixed (may be
 * NULL): the fixed-point tally of the GPU kernels, sum of
 * round_half_even(lmin * scale) clamped at 0, with scale = 2^22 / lref. */
int cmio_interact32(const int32_t ncell[3], const float cell_size[3],
                    const float inv_cell_size[3], const float *kappa, double *tally,
                    uint64_t *fixed, float scale, cmio_packet32 *packet,
                    int32_t *trace_cells, float *trace_lengths, int32_t max_steps,
                    int32_t *nsteps);

/* Mixed-precision walk of the CUDA default transport (the project's own
 * formulation, restated so the GPU kernel can be checked bit for bit).  The
 * geometry is interact's (DensitySubGrid.hpp:1186-1305) in FP64 with the
 * reference's operations in the reference's order: position relative to the
 * anchor, faces idx * cs and (idx + 1.) * cs, l = (face - pos) * (1. / d),
 * crossed coordinates snapped to their face, pos + lmin * d for the others.
 * So every cell crossed and every path length up to the last one equal the
 * reference's.  The opacity kappa = (float)(sigma n x), the optical depths
 * and the tallies are FP32: tau = (float)lmin * kappa, accumulated in FP32;
 * the absorbed cell's fraction min(1, (tau_target - tau_before) / tau) (FP32,
 * tau_before the depth before the cell; the reference's 1 - (tau_done -
 * tau_target) / tau without its cancellation) scales the last length in
 * FP64.  pos is absolute (m), as in Photon. */
typedef struct {
  double pos[3];
  double dir[3];
  float tau_left;
  uint32_t meta; /* low 5 bits: input TravelDirection */
  uint32_t pad[2];
} cmio_packetm;

/* tally / fixed as for cmio_interact32 (FP32 lengths (float)lmin);
 * trace_lengths receives the FP64 lengths. */
int cmio_interact_mixed(const cmio_subgrid *sg, const float *kappa, double *tally,
                        uint64_t *fixed, float scale, cmio_packetm *packet,
                        int32_t *trace_cells, double *trace_lengths, int32_t max_steps,
                        int32_t *nsteps);

/* compute_neutral_fraction (DensitySubGrid.hpp:1628-1658).
 * form 0: the reference expression 1 + a(1 - sqrt(2/a + 1));
 * form 1: the cancellation-free equivalent 1/(1 + a + sqrt(a(a+2))). */
double cmio_jfac(double luminosity, double num_photon, const double inv_cell_size[3]);
void cmio_compute_neutral_fraction(int64_t ncell, const double *nH, double *xH,
                                   double *J, double jfac, double alpha_H, int form);

/* ---- RandomGenerator.hpp (ranlxd, luxury 397) ---- */
typedef struct {
  double x[12];
  double carry;
  uint32_t ir, jr, ir_old, pr;
} cmio_ranlux;
void cmio_ranlux_seed(cmio_ranlux *rng, int32_t seed);
double cmio_ranlux_uniform(cmio_ranlux *rng);

/* Emission (testDensitySubGrid_omp.cpp:529-597). */
void cmio_random_direction(cmio_ranlux *rng, double direction[3]);
void cmio_fill_packets(cmio_ranlux *rng, const double source_position[3],
                       cmio_photon *out, int32_t n, double cross_section);
/* Per-buffer replay streams: buffer b of the iteration is drawn from
 * ranlux(seed + b); the first draw of each buffer picks the subgrid copy
 * (Source.hpp:94-99) and is consumed, then the packets follow. */
void cmio_fill_buffer_stream(int32_t seed, const double source_position[3],
                             cmio_photon *out, int32_t n, double cross_section);

/* Correctly rounded sin / cos (x in [0, 8)) and -log (u in [0, 1)) of the
 * CUDA library's replay of the reference emission streams, and that replay:
 * cmio_fill_buffer_stream with them in place of the C library's cos, sin
 * and log. */
void cmio_cr_sincos(double x, double *sn, double *cs);
double cmio_cr_neg_log(double u);
void cmio_fill_buffer_stream_cr(int32_t seed, const double source_position[3],
                                cmio_photon *out, int32_t n, double cross_section);

/* Photon split over sources (testDensitySubGrid_omp.cpp:2199-2208, 1650-1677). */
void cmio_source_numbers(int32_t nsrc, const double *luminosity, uint32_t num_photon,
                         uint32_t *numbers);
void cmio_distribute(int32_t total_number, int32_t distribute_number,
                     cmio_ranlux *rng, uint32_t *result);

/* Philox4x32-10 (Salmon et al., SC'11), the device production generator. */
void cmio_philox4x32(const uint32_t counter[4], const uint32_t key[2], uint32_t out[4]);
/* Packet p of an emission stream: FP64 direction + optical depth. */
void cmio_philox_packet(uint64_t seed, uint32_t stream, uint64_t packet,
                        double direction[3], double *tau);

/* ---- lattice of subgrids + full serial transport ---- */
typedef struct {
  int32_t num_subgrid[3];
  int32_t sub_ncell[3];
  int64_t cells_per_subgrid;
  int64_t nsub;
  cmio_subgrid *sub;   /* nsub */
  uint32_t *ngb;       /* nsub * 27 */
} cmio_lattice;

int cmio_lattice_init(cmio_lattice *lat, const double box[6], const int32_t ncell[3],
                      const int32_t num_subgrid[3]);
void cmio_lattice_free(cmio_lattice *lat);
/* Subgrid index containing a position (testDensitySubGrid_omp.cpp:1983-1996). */
uint32_t cmio_lattice_locate(const cmio_lattice *lat, const double box[6],
                             const double position[3]);

typedef struct {
  uint64_t absorbed, escaped, crossings, transits, reemitted;
} cmio_counts;

/* Reemission (do_reemission, testDensitySubGrid_omp.cpp:675-702) with the
 * GPU's draws: Philox4x32-10, key {seed_lo, seed_hi + instance}, counter
 * {h0, h1, h2 ^ iteration, 0x434D4952 + (count << 4) + attempt}, count = the
 * packet's earlier reemissions in this subgrid visit (at most 1024); w0 of
 * attempt 0 decides (u < p), w1, w2 a point of the unit disc (Marsaglia's
 * isotropic direction), w3 the optical depth (series logarithm).  Returns 1
 * and fills direction / tau when the packet is re-emitted. */
typedef struct {
  double probability;
  uint64_t seed;
  uint32_t instance, iteration;
} cmio_reemission;
int cmio_reemit_draw(const cmio_reemission *r, uint32_t h0, uint32_t h1, uint32_t h2,
                     uint32_t count, double direction[3], double *tau);
/* hash of an FP64 coordinate for the counter: low ^ high word */
uint32_t cmio_reemit_hash(double x);

/* Transport packets to absorption/escape (fields in subgrid-blocked order). */
void cmio_transport(const cmio_lattice *lat, const double *nH, const double *xH,
                    double *J, cmio_photon *packets, const uint32_t *start_subgrid,
                    int64_t n, cmio_counts *counts);

/* FP32 counterpart of cmio_transport (same routing, cell-unit walk). */
void cmio_transport32(const cmio_lattice *lat, const float *kappa, double *tally,
                      uint64_t *fixed, cmio_packet32 *packets, const uint32_t *start_subgrid,
                      int64_t n, cmio_counts *counts);
/* The same with reemission (r may be NULL).  FP64: counter from the absolute
 * absorption position (cmio_reemit_hash per axis).  FP32: counter from the
 * cell-unit position bits mixed with the subgrid index s: {bits(x) ^ s,
 * bits(y) ^ (s * 0x9E3779B9), bits(z)}; draws in FP64, rounded to FP32. */
void cmio_transport_r(const cmio_lattice *lat, const double *nH, const double *xH, double *J,
                      cmio_photon *packets, const uint32_t *start_subgrid, int64_t n,
                      cmio_counts *counts, const cmio_reemission *r);
void cmio_transport32_r(const cmio_lattice *lat, const float *kappa, double *tally,
                        uint64_t *fixed, cmio_packet32 *packets, const uint32_t *start_subgrid,
                        int64_t n, cmio_counts *counts, const cmio_reemission *r);
/* Mixed-precision counterpart (cmio_interact_mixed): same routing; the
 * reemission counter is the FP64 one (cmio_reemit_hash of the absolute
 * absorption position per axis), the drawn optical depth rounded to FP32. */
void cmio_transportm_r(const cmio_lattice *lat, const float *kappa, double *tally,
                       uint64_t *fixed, cmio_packetm *packets, const uint32_t *start_subgrid,
                       int64_t n, cmio_counts *counts, const cmio_reemission *r);
/* scale of the fixed-point tally of a subgrid: 2^24 / max float cell size */
float cmio_fixed_scale(const cmio_subgrid *sg);

/* Packets per source for one iteration: the reference split
 * (uint)(L_i/L_tot*N), with the remainder going to the sources holding the
 * smallest Philox draws of this (seed, iteration) -- the counter-based
 * stand-in for distribute() (testDensitySubGrid_omp.cpp:1650-1677). */
void cmio_split_packets(int32_t nsrc, const double *luminosity, uint64_t num_photon,
                        uint64_t seed, uint32_t iteration, uint64_t *numbers);

/* FP32 kappa field: (float)(sigma * nH * xH). */
void cmio_kappa32(int64_t ncell, const double *nH, const double *xH, double sigma,
                  float *kappa);

/* Whole iteration on the host cores with OpenMP (CPU baseline "port"). */
void cmio_iteration_omp(const cmio_lattice *lat, const double box[6], const double *nH,
                        double *xH, double *J, int32_t nsrc, const double *src_pos,
                        const double *src_lum, uint64_t num_photon, uint64_t seed,
                        uint32_t iteration, double alpha_H, double cross_section,
                        int balance_form, int threads, cmio_counts *counts);

/* Dust scattering with forced first scattering and a peel-off image (the photon loop
 * of testDensitySubGrid_omp_dust.cpp), restating cmi_dust_run of the CUDA library with
 * the same counter-based draws. */
typedef struct {
  uint64_t emitted, scatterings, absorbed, escaped, cell_crossings, subgrid_transits,
      peeloffs_off_image;
  uint32_t generations, error_flags;
} cmio_dust_stats;
double cmio_dust_exp(double x);
void cmio_dust_run(const cmio_lattice *lat, const double box[6], const double *nH,
                   const double *xH, uint32_t num_photon, uint64_t seed, uint32_t instance,
                   uint32_t iteration, double albedo, const double source[3],
                   uint32_t source_subgrid, int32_t npix_x, int32_t npix_y, double *image,
                   cmio_dust_stats *st);

#ifdef __cplusplus
}
#endif

#endif
