/*
 * cmacionize_b200.h -- C ABI of the B200 photon-packet transport and
 * ionization-balance library (libcmacionize_b200.so).
 *
 * This is the drop-in boundary for the plain photoionization method of
 * ParallelCMacIonize.  The reference has no plugin or FFI layer; its de-facto
 * boundary is three C++ calls, each mapped here:
 *
 *   DensitySubGrid::interact(Photon&, int)          DensitySubGrid.hpp:1180
 *       -> cmi_trace_packet (one packet, with its cell sequence)
 *   do_photon_traversal(PhotonBuffer&, DensitySubGrid&, PhotonBuffer*, bool*)
 *                                                  testDensitySubGrid_omp.cpp:607
 *       -> cmi_traverse_buffer
 *   DensitySubGrid::compute_neutral_fraction(double, unsigned int)
 *                                                  DensitySubGrid.hpp:1628
 *       -> cmi_compute_neutral_fraction
 *
 * plus the whole shoot-packets -> solve-balance iteration of the driver's
 * main loop (testDensitySubGrid_omp.cpp:2213-2434) as cmi_run_iterations.
 *
 * Conventions: every entry point returns an int status (CMI_OK = 0); no
 * exception crosses the ABI; cmi_last_error_string() describes the last
 * failure of the calling thread.  A context owns all of its device memory and
 * is used by one host thread at a time.  Field arrays are FP64, one value per
 * cell, in one of two orders (cmi_layout).  All pointers are host pointers
 * unless a function says otherwise.
 */
#ifndef CMACIONIZE_B200_H
#define CMACIONIZE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CMI_ABI_VERSION 2
#define CMI_NUM_DIRECTIONS 27           /* TRAVELDIRECTION_NUMBER, TravelDirections.hpp:74 */
#define CMI_NEIGHBOUR_OUTSIDE 0xffffffffu /* NEIGHBOUR_OUTSIDE, DensitySubGrid.hpp:53 */
#define CMI_PHOTONBUFFER_SIZE 200       /* PHOTONBUFFER_SIZE, PhotonBuffer.hpp:42 */

/* status codes */
enum cmi_status {
  CMI_OK = 0,
  CMI_ERR_INVALID_ARGUMENT = 1,
  CMI_ERR_CUDA = 2,
  CMI_ERR_OUT_OF_MEMORY = 3,
  CMI_ERR_CAPACITY = 4,       /* a device queue or buffer would overflow */
  CMI_ERR_DEVICE_TIMEOUT = 5, /* a bounded device-side wait gave up */
  CMI_ERR_INVARIANT = 6,      /* a device-side invariant check failed */
  CMI_ERR_NOT_SUPPORTED = 7
};

/* One photon packet.  Same 80-byte layout and field order as the reference
 * Photon (Photon.hpp:49-68): position (m), unit direction, target optical
 * depth, photoionization cross section (m^2), weight, packet type. */
typedef struct {
  double position[3];
  double direction[3];
  double target_optical_depth;
  double photoionization_cross_section;
  double weight;
  int32_t type;
  int32_t reserved;
} cmi_photon;

/* One grid instance: a box cut into num_subgrid[0..2] subgrids of equal size
 * (testDensitySubGrid_omp.cpp:1801-1877).  ncell must be a multiple of
 * num_subgrid on every axis. */
typedef struct {
  double box[6];              /* anchor x y z, side lengths x y z (m) */
  int32_t ncell[3];           /* cells per axis, whole grid */
  int32_t num_subgrid[3];     /* subgrids per axis */
  double recombination_rate;  /* alpha_H (m^3/s); reference: 4e-19 (DensitySubGrid.hpp:1637) */
  double cross_section;       /* sigma (m^2); reference: 6.3e-22 (testDensitySubGrid_omp.cpp:589) */
} cmi_grid_desc;

enum cmi_precision {
  CMI_TRANSPORT_FP64 = 0, /* the reference's FP64 walk, operation for operation */
  CMI_TRANSPORT_FP32 = 1, /* FP32 cell-unit walk, shared-memory tallies (cmi_tally) merged into FP64 */
  CMI_TRANSPORT_MIXED = 2 /* the reference's FP64 geometry operation for operation (cell
                             sequences and path lengths equal DensitySubGrid::interact's),
                             FP32 opacity sigma*n*x, optical depths and tallies (cmi_tally);
                             the target optical depth is held in FP32 */
};
enum cmi_balance_form {
  CMI_BALANCE_REFERENCE = 0, /* x = 1 + a(1 - sqrt(2/a + 1)), DensitySubGrid.hpp:1650 */
  CMI_BALANCE_STABLE = 1     /* x = 1 / (1 + a + sqrt(a(a + 2))), same value, no cancellation */
};
enum cmi_tally {
  CMI_TALLY_FP32 = 0,              /* FP32 shared-memory atomics */
  CMI_TALLY_FP32_COMPENSATED = 1,  /* FP32 atomics + TwoSum rounding error in a second FP32 word */
  CMI_TALLY_FIXED64 = 2,           /* fixed point (lref/2^22 units), 32-bit integer atomics, carries to FP64 J */
  CMI_TALLY_FIXED64_ATOMIC64 = 3   /* 64-bit fixed point, 64-bit integer atomics */
};
enum cmi_rng {
  CMI_RNG_PHILOX = 0, /* counter-based Philox4x32-10 per packet */
  CMI_RNG_RANLUX = 1  /* the reference's ranlxd, one stream per 200-packet buffer: buffer b
                         (counted over all sources of the context, 0-based) of iteration i
                         draws from ranlxd(seed + b + i * buffers), first one draw for the
                         subgrid-copy pick (Source.hpp:94-99), then per packet cos(theta),
                         phi and the optical depth (testDensitySubGrid_omp.cpp:529-597);
                         sin, cos and log are correctly rounded */
};
enum cmi_layout {
  CMI_LAYOUT_BLOCKED = 0, /* subgrid after subgrid, each in DensitySubGrid order (reference output order) */
  CMI_LAYOUT_CUBE = 1     /* whole grid, index (ix * ny + iy) * nz + iz */
};
enum cmi_memory {
  CMI_MEMORY_HOST = 0,
  CMI_MEMORY_DEVICE = 1
};

typedef struct {
  int32_t transport_precision; /* cmi_precision */
  int32_t balance_form;        /* cmi_balance_form */
  int32_t rng;                 /* cmi_rng */
  int32_t device;              /* CUDA device ordinal */
  int32_t threads_per_cta;     /* 0 = library default (256) */
  int32_t ctas_per_sm;         /* 0 = as many as fit */
  int32_t packets_per_chunk;   /* 0 = library default (128; 256 when subgrids have <= 1024
                                  cells); power of two in [32, 4096] */
  int32_t tally_mode;          /* FP32 and mixed transports: cmi_tally (default CMI_TALLY_FIXED64) */
  int32_t use_graph;           /* 1 = capture each iteration as a CUDA graph (default) */
  int32_t max_run_chunks;      /* most chunks a CTA claims at once (0 = 64): how long a CTA
                                  stays on one subgrid before flushing its tallies */
  int32_t refill_lanes;        /* FP32 and mixed walks: a warp routes finished packets and refills its
                                  lanes once this many lanes are not walking (0 = 16; 1..32) */
  int32_t reserved[5];
} cmi_options;

/* Per-instance counters of one iteration. */
typedef struct {
  uint64_t packets_emitted;
  uint64_t packets_absorbed;
  uint64_t packets_escaped;
  uint64_t cell_crossings;   /* iterations of the interact loop, DensitySubGrid.hpp:1221 */
  uint64_t subgrid_transits; /* calls of interact */
  double mean_abs_dx;        /* mean |x_new - x_old| over the cells of the instance */
  uint32_t error_flags;      /* CMI_FLAG_* bits raised on the device */
  uint32_t rounds;           /* wavefront rounds that carried packets */
  uint64_t packets_reemitted; /* absorptions followed by a reemission */
} cmi_stats;

#define CMI_FLAG_ARENA_OVERFLOW 1u
#define CMI_FLAG_STAGE_TIMEOUT 2u
#define CMI_FLAG_WALK_LIMIT 4u     /* a transit exceeded its step bound (NaN direction, ...) */
#define CMI_FLAG_LEFTOVER 8u       /* packets left after the last round */
#define CMI_FLAG_BAD_INPUT 16u

typedef struct cmi_context cmi_context;

void cmi_default_options(cmi_options *options);
const char *cmi_last_error_string(void);
int cmi_abi_version(void);

/* Create a context holding num_instances independent grids (a batch of one
 * is the plain method).  Fields start as n_H = 1e8 m^-3 and x_H = 1e-6, the
 * reference's initial state (DensitySubGrid.hpp:544-551). */
int cmi_create(const cmi_grid_desc *grids, int32_t num_instances, const cmi_options *options,
               cmi_context **context);
int cmi_destroy(cmi_context *context);

/* Copy n_H (m^-3) and/or x_H into an instance; either pointer may be NULL. */
int cmi_set_fields(cmi_context *context, int32_t instance, int32_t layout, int32_t memory,
                   const double *number_density, const double *neutral_fraction);
/* Overlapped input for callers that send fields every iteration: the n_H
 * copy from pinned host memory runs on a side stream, so it can proceed while
 * the previous iteration's x_H comes back (cmi_get_fields), and
 * cmi_set_fields_prefetched then takes it together with x_H (host or device,
 * `memory`) in the prefetch's layout.  cmi_set_fields_prefetched returns
 * without waiting: its copies run on the side stream while the next
 * iteration emits its packets, and the iteration's first transport round
 * waits for them.  Both input arrays must stay unchanged until the next
 * cmi_run_iterations, cmi_run_until_converged, cmi_shoot_packets,
 * cmi_get_fields or cmi_synchronize returns; every other entry point orders
 * its own work after the copies.  One prefetch per instance may be pending.
 * No reference counterpart (the reference keeps its fields in host memory). */
int cmi_prefetch_number_density(cmi_context *ctx, int32_t instance, int32_t layout,
                                const double *nH);
int cmi_set_fields_prefetched(cmi_context *ctx, int32_t instance, int32_t memory,
                              const double *xH);
/* Read x_H and/or the intensity integral J (m^3); either pointer may be NULL. */
int cmi_get_fields(cmi_context *context, int32_t instance, int32_t layout, int32_t memory,
                   double *neutral_fraction, double *intensity_integral);
/* Overwrite the intensity integrals (e.g. to merge tallies of other processes). */
int cmi_set_intensity(cmi_context *context, int32_t instance, int32_t layout, int32_t memory,
                      const double *intensity_integral);

/* Point sources of an instance (Source.hpp:34-109): positions (3 per source,
 * m) and ionizing luminosities (s^-1). */
int cmi_set_sources(cmi_context *context, int32_t instance, const double *positions,
                    const double *luminosities, int32_t num_sources);
/* Packets emitted per iteration by an instance (num_photon). */
int cmi_set_packet_budget(cmi_context *context, int32_t instance, uint64_t num_photon);
/* reemission_probability (params.txt; do_reemission,
 * testDensitySubGrid_omp.cpp:675-702): an absorbed packet is re-emitted from
 * its absorption point with this probability, in a new isotropic direction
 * with a new optical depth, and walks on (default 0: absorbed packets are
 * done).  The draws come from Philox keyed like the instance's emission, with
 * the absorption position as counter.  packets_absorbed counts the final
 * absorptions only. */
int cmi_set_reemission_probability(cmi_context *context, int32_t instance, double probability);

/* Run whole iterations of the plain method on every instance: emit the
 * packets, trace them to absorption or escape, solve the ionization balance
 * (testDensitySubGrid_omp.cpp:2213-2434).  stats receives num_iterations x
 * num_instances records (iteration-major) and may be NULL. */
int cmi_run_iterations(cmi_context *context, int32_t num_iterations, uint64_t seed,
                       cmi_stats *stats);
/* Run iterations until every instance has converged or max_iterations have
 * run.  No reference counterpart: the reference runs a fixed number of
 * iterations (number of iterations in params.txt).  An instance has converged
 * after iteration k (k >= min_iterations) when the mean over its cells of
 * |x_H after - x_H before| in that iteration is below tolerance; from then on
 * it is frozen for the rest of the call: it emits no packets and keeps its
 * x_H.  The Monte Carlo noise of x_H sets a floor under the mean change
 * (roughly proportional to 1/sqrt(packets per iteration)), so a tolerance
 * below that floor runs to max_iterations.  stats receives iterations_done x
 * num_instances records (iteration-major; capacity max_iterations x
 * num_instances; may be NULL), *iterations_done the number of iterations run,
 * converged_at[i] (num_instances entries, may be NULL) the 1-based iteration
 * after which instance i converged, 0 if it did not. */
int cmi_run_until_converged(cmi_context *context, int32_t max_iterations, int32_t min_iterations,
                            double tolerance, uint64_t seed, cmi_stats *stats,
                            int32_t *iterations_done, int32_t *converged_at);
/* fill_buffer (testDensitySubGrid_omp.cpp:556-597) for every source of the
 * context: the photons one iteration with this seed and iteration index
 * emits (cmi_run_iterations, cmi_shoot_packets), without transporting them,
 * in the reference Photon layout (source position, isotropic direction,
 * target optical depth, the instance's cross section, weight 1).  Order:
 * instance after instance, source after source, and within a source the
 * emission order (CMI_RNG_RANLUX: buffer after buffer of 200, each drawn from
 * the reference's ranlxd seeded as described under cmi_rng, with correctly
 * rounded sin, cos and log).  *count receives the number of photons; with
 * out NULL or capacity below it the call fails with CMI_ERR_CAPACITY after
 * setting *count. */
int cmi_emit_photons(cmi_context *context, uint64_t seed, uint32_t iteration, cmi_photon *out,
                     uint64_t capacity, uint64_t *count);
/* Transport phase only (no balance); J keeps accumulating. */
int cmi_shoot_packets(cmi_context *context, uint64_t seed, uint32_t iteration, cmi_stats *stats);

/* Trace caller-supplied packets through an instance until absorption or
 * escape (the driver's task loop for a given packet list).  start_subgrid[i]
 * is the subgrid that contains packet i; every packet starts INSIDE it. */
int cmi_transport_packets(cmi_context *context, int32_t instance, const cmi_photon *packets,
                          const uint32_t *start_subgrid, uint64_t num_packets, cmi_stats *stats);

/* do_photon_traversal (testDensitySubGrid_omp.cpp:607-666): walk every photon
 * of one buffer through one subgrid, entering from input_direction, and sort
 * the results into the 27 TravelDirection output buffers.  out receives the
 * updated photons grouped by output direction (direction-major, input order
 * inside a group), out_count[d] the size of group d.  Groups whose
 * output_enabled[d] is 0 are dropped and counted in *num_done (NULL enables
 * all 27).  The walk tallies into the subgrid's J. */
int cmi_traverse_buffer(cmi_context *context, int32_t instance, uint32_t subgrid,
                        int32_t input_direction, const cmi_photon *in, uint32_t num_photons,
                        const uint8_t *output_enabled, cmi_photon *out,
                        uint32_t out_count[CMI_NUM_DIRECTIONS], uint32_t *num_done);

/* DensitySubGrid::interact (DensitySubGrid.hpp:1180-1323) for one packet,
 * with its cell sequence: cells[k] is the subgrid-local cell index of loop
 * iteration k and lengths[k] its path length lmin (m).  *num_steps receives
 * the full count even when it exceeds max_steps.  *photon is updated and
 * *output_direction receives the exit TravelDirection. */
int cmi_trace_packet(cmi_context *context, int32_t instance, uint32_t subgrid,
                     int32_t input_direction, cmi_photon *photon, int32_t max_steps,
                     int32_t *cells, double *lengths, int32_t *num_steps,
                     int32_t *output_direction);

/* compute_neutral_fraction (DensitySubGrid.hpp:1628-1658) on every cell of
 * an instance with the given total luminosity and packet count; resets J. */
int cmi_compute_neutral_fraction(cmi_context *context, int32_t instance, double luminosity,
                                 uint64_t num_photon, double *mean_abs_dx);

/* The same for the subgrids [first_subgrid, first_subgrid + count) of an
 * instance only: DensitySubGrid::compute_neutral_fraction called per subgrid. */
int cmi_compute_neutral_fraction_subgrids(cmi_context *context, int32_t instance,
                                          uint32_t first_subgrid, uint32_t count,
                                          double luminosity, uint64_t num_photon,
                                          double *mean_abs_dx);

/* Device-side access for interop (zero-copy views, NCCL reductions): the
 * instance's J (which = 0), x_H (1) or n_H (2) array in BLOCKED layout, and
 * the CUDA stream every kernel of the context runs on.  cmi_device_field
 * returns once the context's queued work (field copies included) is done, so
 * the array may be read on any stream; work queued on the stream from
 * cmi_get_stream runs after the field copies. */
int cmi_device_field(cmi_context *context, int32_t instance, int32_t which, double **device_ptr,
                     uint64_t *count);
int cmi_get_stream(cmi_context *context, void **cuda_stream);
int cmi_synchronize(cmi_context *context);

/* Kernel launches issued by the most recent cmi_run_iterations /
 * cmi_shoot_packets call (graph replays count their kernel nodes). */
int cmi_last_launch_count(cmi_context *context, uint64_t *launches);

/* Per-kernel timing with CUDA events on the context's stream.  While enabled,
 * iterations are launched kernel by kernel (no graph) with an event pair
 * around every launch; cmi_kernel_timing returns the summed device time (ms)
 * and launch count of each kernel class since the last call:
 * [0] walk, [1] plan + scatter, [2] emission, [3] balance. */
#define CMI_KERNEL_CLASSES 4
int cmi_set_kernel_timing(cmi_context *context, int32_t enable);
int cmi_kernel_timing(cmi_context *context, double milliseconds[CMI_KERNEL_CLASSES],
                      uint64_t launches[CMI_KERNEL_CLASSES]);

/* Allocation-free variant of cmi_traverse_buffer.  No counterpart in the
 * reference: it exists for callers that cannot allocate device memory, e.g.
 * a host code whose GPU memory is owned by its own pool allocator, or a
 * plug-in running inside another application's process, where a cudaMalloc
 * or cudaFree would synchronize the whole device, fragment the host's pool or
 * fail outright.  It needs no context: the caller passes the subgrid (box,
 * cells, FP64 fields in DensitySubGrid cell order) and every input and output
 * as device pointers; the library allocates nothing.  The walk's intermediate
 * photons live in one fixed array in device global memory, the same for every
 * call, sized for CMI_NOALLOC_MAX_PHOTONS photons (about 340 KiB, held by
 * every GPU that loads the library until the process exits).
 *
 *   box, ncell        subgrid box (anchor, sides; m) and cells per axis
 *                     (at most 4096 cells)
 *   d_nH, d_xH, d_J   device fields; J receives the tallies (accumulated)
 *   d_in, n           device photons, n <= CMI_NOALLOC_MAX_PHOTONS
 *   output_enabled    host flags of the 27 output buffers (NULL: all)
 *   d_out             device output, n photons, grouped by exit direction
 *   d_out_count       device array of 27 group sizes
 *   d_num_done        device counter of the photons in disabled groups
 *   stream            cudaStream_t to run on (NULL: the default stream)
 *
 * Runs the reference FP64 walk on the calling thread's current device and
 * returns when the stream has finished it.  The first call on a device looks
 * up the array's device address (once per device), so make the first call
 * before any stream capture.  A cudaDeviceReset discards the array and makes
 * that address stale: do not call this entry point on a device after
 * resetting it in the same process.  Calls that overlap on the GPU (other
 * host threads, other streams) share the array and race: serialise them. */
#define CMI_NOALLOC_MAX_PHOTONS 4096
int cmi_traverse_buffer_noalloc(const double box[6], const int32_t ncell[3],
                                const double *d_nH, const double *d_xH, double *d_J,
                                int32_t input_direction, const cmi_photon *d_in, uint32_t n,
                                const uint8_t *output_enabled, cmi_photon *d_out,
                                uint32_t *d_out_count, uint32_t *d_num_done, void *stream);

/* ---------------------------------------------------------------------------
 * Dust scattering with forced first scattering and a peel-off image: the
 * photon loop of the reference's dust driver (testDensitySubGrid_omp_dust.cpp:
 * fill_buffer :564-620 with FORCED_SCATTERING, execute_relaunch_photon_task
 * :1200-1260, do_photon_traversal :621-722, do_reemission :730-760,
 * execute_photon_reemit_task :1484-1560) on an instance's current n_H, x_H:
 *   - num_photon packets leave `source` isotropically (weight 1, cross
 *     section 1) and add up the optical depth tau0 to the box edge
 *     (DensitySubGrid::compute_optical_depth, DensitySubGrid.hpp:1482-1604);
 *   - each restarts at the source with weight 1 - exp(-tau0) and target depth
 *     -ln(1 - u (1 - exp(-tau0))) and walks to it without tallies
 *     (DensitySubGrid::propagate, DensitySubGrid.hpp:1333-1472);
 *   - an absorbed packet scatters with probability `albedo` (the driver's
 *     reemission_probability): isotropic direction, target -ln u, weight / 4pi;
 *     a copy of it walks along +z to the box edge and adds weight * exp(-depth)
 *     to the pixel under its exit point (npix_x columns over the box's x
 *     side, npix_y rows over its y side; pixel (ix, iy) at image[ix * npix_y +
 *     iy]); repeated until no packet is left.
 * `image` (host, npix_x * npix_y) receives the sums divided by num_photon, as
 * the driver writes image.dat.  FP64 throughout, the reference's walk
 * arithmetic; counter-based draws (seed, iteration) replace the reference's
 * per-thread generators.  albedo in [0, 1); num_photon <= 2^30.  The packet
 * buffers (about 290 bytes per packet) grow to the largest call and stay with
 * the context until cmi_destroy. */
/* The dust driver's per-buffer walks through one subgrid (do_photon_traversal,
 * testDensitySubGrid_omp_dust.cpp:646-652), FP64 with the reference's
 * arithmetic, on the instance's current fields:
 *   CMI_WALK_PROPAGATE      DensitySubGrid::propagate (DensitySubGrid.hpp:
 *                           1333-1472): interact without the J tally
 *   CMI_WALK_OPTICAL_DEPTH  DensitySubGrid::compute_optical_depth (:1482-1604):
 *                           no target; the crossing's optical depth is added
 *                           to target_optical_depth
 * photons (host, n) are updated in place; output_directions[i] receives the
 * TravelDirection photon i leaves by (TRAVELDIRECTION_INSIDE: it reached its
 * target).  input_directions: one per photon. */
#define CMI_WALK_PROPAGATE 1
#define CMI_WALK_OPTICAL_DEPTH 2
int cmi_walk_photons(cmi_context *ctx, int32_t instance, uint32_t subgrid, int32_t mode,
                     cmi_photon *photons, const int32_t *input_directions, uint32_t n,
                     int32_t *output_directions);

typedef struct cmi_dust_stats {
  uint64_t emitted;            /* source packets */
  uint64_t scatterings;        /* scattered packets (= peel-off packets) */
  uint64_t absorbed;           /* absorbed and not scattered */
  uint64_t escaped;            /* relaunched or scattered packets that left the box */
  uint64_t cell_crossings;     /* every walk: TAU, DIRECT and PEELOFF */
  uint64_t subgrid_transits;
  uint64_t peeloffs_off_image; /* peel-offs whose exit point is off the image */
  uint32_t generations;        /* walk + scatter rounds run */
  uint32_t error_flags;
} cmi_dust_stats;
int cmi_dust_run(cmi_context *ctx, int32_t instance, uint64_t num_photon, uint64_t seed,
                 uint32_t iteration, double albedo, const double source[3], int32_t npix_x,
                 int32_t npix_y, double *image, cmi_dust_stats *stats);

/* ---------------------------------------------------------------------------
 * Learned warm start.  No reference counterpart: the reference starts every
 * run from x_H = 1e-6 (DensitySubGrid.hpp:544-551).  A 3-level 3D
 * convolutional U-Net maps three input channels per cell (cmi_unet_features:
 * density, unattenuated source flux and a Stromgren ratio along the rays
 * from the sources) to log10 x_H; the plain iteration then starts from that
 * field and still decides convergence.
 *
 * Layers (c1, c2, c3 channels per level; 3x3x3 convolutions, zero padding,
 * leaky ReLU; 2x2x2 average pooling down, nearest-neighbour upsampling up,
 * skip connections concatenated after the upsampled channels):
 *   level 1: conv(3 -> c1), conv(c1 -> c1)      pooled to level 2
 *   level 2: conv(c1 -> c2), conv(c2 -> c2)     pooled to level 3
 *   level 3: conv(c2 -> c3), conv(c3 -> c3)     upsampled to level 2
 *   level 2: conv(c3 + c2 -> c2), conv(c2 -> c2) upsampled to level 1
 *   level 1: conv(c2 + c1 -> c1), conv(c1 -> c1), 1x1 conv(c1 -> 1)
 * Parameters (FP32 master copy, in this order per convolution): W[co][tap][ci]
 * with tap = (dz * 3 + dy) * 3 + dx, then b[co]; last the head's w[c1], b.
 * Weights and activations are BF16, accumulation FP32; the 3x3x3
 * convolutions, their input gradients and their weight gradients run on the
 * tensor cores (tcgen05).  Training minimises the mean squared
 * error of log10 x_H with Adam.
 *
 * Tensors handed to the network live in device memory, FP32, one sample
 * after another in the engine's cube order (index (ix * ny + iy) * nz + iz):
 * features [batch][cells][3], targets and predictions [batch][cells].  Grid
 * sides must be multiples of 32, and batch x cells at most 2^27 (134217728;
 * CMI_ERR_NOT_SUPPORTED beyond).  Calls are synchronous.  Errors: the codes
 * above, message in cmi_unet_last_error_string().
 *
 * The network runs on a stream of its own.  The first forward, gradient or
 * training call for a (batch, grid) shape records the pass's kernel launches
 * in CUDA graphs on that stream (and the first call of all, the weight
 * packing) and later calls replay them; a new shape re-records.  Make such
 * first calls while no global-mode stream capture is active in the process. */
typedef struct cmi_unet cmi_unet;
typedef struct {
  int32_t channels[3];  /* c1 (<= 16), c2, c3 (<= 64); default 12, 24, 48 (~2e5 parameters) */
  float leaky_slope;    /* default 0.1 */
  int32_t device;
  int32_t reserved[8];
} cmi_unet_config;

void cmi_unet_default_config(cmi_unet_config *config);
const char *cmi_unet_last_error_string(void);
int cmi_unet_create(const cmi_unet_config *config, cmi_unet **net);
int cmi_unet_destroy(cmi_unet *net);
int cmi_unet_num_params(cmi_unet *net, int64_t *count);
/* FP32 parameters to / from host memory (set also resets the optimiser) */
int cmi_unet_get_params(cmi_unet *net, float *params);
int cmi_unet_set_params(cmi_unet *net, const float *params);
/* predictions of log10 x_H */
int cmi_unet_forward(cmi_unet *net, const float *features, float *prediction, int32_t batch,
                     const int32_t dims[3]);
/* forward + backward without an update: mean squared error and the gradient
 * of every parameter (host array, num_params entries; may be NULL) */
int cmi_unet_gradients(cmi_unet *net, const float *features, const float *target, int32_t batch,
                       const int32_t dims[3], float *loss, float *gradients);
/* one Adam step (beta 0.9, 0.999, eps 1e-8) at learning rate lr */
int cmi_unet_train_step(cmi_unet *net, const float *features, const float *target, int32_t batch,
                        const int32_t dims[3], float lr, float *loss);
/* The three input channels of one grid ([cells][3], FP32, device) from its
 * FP64 n_H (device, cube order) and sources (host, [x, y, z, L] each), each
 * channel (raw - norm[2k]) / norm[2k + 1]:
 *   0: log10 n_H
 *   1: log10 sum_i L_i / (4 pi r_i^2), r clamped to half a cell
 *   2: log10 sum_i L_i / (4 pi alpha R_i), R_i = integral of n_H^2 r^2 dr
 *      along the ray from source i to the cell centre (FP32 midpoint sum in
 *      steps of at most half the smallest cell side, n_H of the cell holding
 *      each sample), clamped to [1e-30, 1e30] */
int cmi_unet_features(cmi_unet *net, const double *nH_cube, const int32_t dims[3],
                      const double box[6], const double *sources, int32_t num_sources,
                      double recombination_rate, const float norm[6], float *features);
/* The same channels with channel 2 computed on the grid coarser by
 * ratio_factor per axis (n_H block-averaged, dims multiples of the factor) and
 * interpolated trilinearly in log10 to the cell centres: the ray march costs
 * ratio_factor^4 times less.  ratio_factor = 1 is cmi_unet_features. */
int cmi_unet_features_coarse_ratio(cmi_unet *net, const double *nH_cube, const int32_t dims[3],
                                   const double box[6], const double *sources,
                                   int32_t num_sources, double recombination_rate,
                                   const float norm[6], int32_t ratio_factor, float *features);
/* Weight of the squared error of predictions above the target (a neutral
 * fraction too high) in the loss of cmi_unet_gradients / cmi_unet_train_step;
 * 1 (the default) is the mean squared error. */
int cmi_unet_set_loss_weight(cmi_unet *net, float over_weight);
/* Resampling for grids finer than the network's training grid (cube order,
 * device): block mean of an FP64 field by `factor` per axis (dims of the
 * source, multiples of factor), nearest-neighbour upsampling of an FP32
 * field by `factor` per axis (dims of the source). */
int cmi_unet_block_mean(cmi_unet *net, const double *src, const int32_t dims[3], int32_t factor,
                        double *dst);
int cmi_unet_upsample_nearest(cmi_unet *net, const float *src, const int32_t dims[3],
                              int32_t factor, float *dst);
/* x_H = 10^clamp(prediction, log10_min, 0) as FP64 (device), n values */
int cmi_unet_to_neutral_fraction(cmi_unet *net, const float *prediction, double *xH, int64_t n,
                                 float log10_min);
/* Building blocks, exposed for testing (grids: X and Y multiples of 8, and Y a
 * multiple of 16 or Z of 2): one 3x3x3 convolution on the tensor cores (BF16
 * channels-last device tensors, channel counts multiples of 16 (the weight
 * gradient: output channels <= 128); up to 80 output channels the three x taps
 * share one MMA (tiles of 16 x 8 x KZ voxels), above that tiles of 8 x 16 x KZ or
 * 8 x 8 x 2 voxels; weights packed by cmi_unet_pack_weights for the same output
 * channel count, bias FP32 or NULL, activation 1 = leaky ReLU); packing of FP32 W[cout][27][cin] (flip = 1: the input-gradient
 * form); the weight gradient dW[cout][27][cin] (FP32, device) of a
 * convolution from its input x and output gradient dy. */
int cmi_unet_conv3(cmi_unet *net, const void *in, int32_t in_channels, const void *weights_packed,
                   const float *bias, void *out, int32_t out_channels, int32_t activation,
                   int32_t batch, const int32_t dims[3]);
int cmi_unet_pack_weights(cmi_unet *net, const float *weights, int32_t cout, int32_t cin,
                          int32_t flip, void *packed);
int cmi_unet_conv3_wgrad(cmi_unet *net, const void *x, int32_t cin, const void *dy, int32_t cout,
                         int32_t batch, const int32_t dims[3], float *dw);

#ifdef __cplusplus
}
#endif

#endif /* CMACIONIZE_B200_H */
