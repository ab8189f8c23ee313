/*
 * CPU oracle: plain-C restatement of the reference photon transport and
 * ionization balance (bwvdnbro/ParallelCMacIonize).  TEST INFRASTRUCTURE:
 * only tests/, the smoke check and bench.py's CPU-baseline leg load this.
 *
 * Build: oracle/Makefile  (-O2 -ffp-contract=off, no -ffast-math, so every
 * FP64 operation happens in the order written and is rounded once).
 *
 * Each function cites the reference file:line whose behaviour it restates.
 */
#include "cmi_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* TravelDirections (TravelDirections.hpp:46-403).                           */
/* Every direction is a triple of axis signs: +1 = upper (P) face of that    */
/* axis, -1 = lower (N) face, 0 = axis not involved.                         */
/* ------------------------------------------------------------------------ */
static const signed char kSigns[CMIO_NUM_DIRECTIONS][3] = {
    {0, 0, 0},                                                  /* INSIDE */
    {1, 1, 1},   {1, 1, -1},  {1, -1, 1},  {1, -1, -1},         /* CORNER_P.. */
    {-1, 1, 1},  {-1, 1, -1}, {-1, -1, 1}, {-1, -1, -1},        /* CORNER_N.. */
    {0, 1, 1},   {0, 1, -1},  {0, -1, 1},  {0, -1, -1},         /* EDGE_X_yz */
    {1, 0, 1},   {1, 0, -1},  {-1, 0, 1},  {-1, 0, -1},         /* EDGE_Y_xz */
    {1, 1, 0},   {1, -1, 0},  {-1, 1, 0},  {-1, -1, 0},         /* EDGE_Z_xy */
    {1, 0, 0},   {-1, 0, 0},  {0, 1, 0},   {0, -1, 0},          /* FACE_X/Y */
    {0, 0, 1},   {0, 0, -1}};                                   /* FACE_Z */

static int direction_from_signs(int sx, int sy, int sz) {
  for (int d = 0; d < CMIO_NUM_DIRECTIONS; ++d) {
    if (kSigns[d][0] == sx && kSigns[d][1] == sy && kSigns[d][2] == sz) {
      return d;
    }
  }
  return -1;
}

/* TravelDirections.hpp:89-152: swap every P for N. */
int cmio_output_to_input_direction(int output_direction) {
  if (output_direction < 0 || output_direction >= CMIO_NUM_DIRECTIONS) {
    return -1;
  }
  const signed char *s = kSigns[output_direction];
  return direction_from_signs(-s[0], -s[1], -s[2]);
}

/* TravelDirections.hpp:315-403: bits (x_high,x_low,y_high,y_low,z_high,z_low). */
int cmio_direction_from_mask(int mask) {
  if (mask < 0 || mask > 63) {
    return -1;
  }
  int s[3];
  for (int a = 0; a < 3; ++a) {
    const int high = (mask >> (5 - 2 * a)) & 1;
    const int low = (mask >> (4 - 2 * a)) & 1;
    if (high && low) {
      return -1;
    }
    s[a] = high ? 1 : (low ? -1 : 0);
  }
  return direction_from_signs(s[0], s[1], s[2]);
}

/* TravelDirections.hpp:163-224 (leaving moves along the face's sign). */
int cmio_is_compatible_output_direction(const double *direction, int output_direction) {
  if (output_direction < 0 || output_direction >= CMIO_NUM_DIRECTIONS) {
    return 0;
  }
  for (int a = 0; a < 3; ++a) {
    const int s = kSigns[output_direction][a];
    if ((s > 0 && !(direction[a] > 0.)) || (s < 0 && !(direction[a] < 0.))) {
      return 0;
    }
  }
  return 1;
}

/* TravelDirections.hpp:235-298 (entering moves against the face's sign). */
int cmio_is_compatible_input_direction(const double *direction, int input_direction) {
  if (input_direction < 0 || input_direction >= CMIO_NUM_DIRECTIONS) {
    return 0;
  }
  for (int a = 0; a < 3; ++a) {
    const int s = kSigns[input_direction][a];
    if ((s > 0 && !(direction[a] < 0.)) || (s < 0 && !(direction[a] > 0.))) {
      return 0;
    }
  }
  return 1;
}

/* ------------------------------------------------------------------------ */
/* DensitySubGrid geometry.                                                  */
/* ------------------------------------------------------------------------ */

/* DensitySubGrid.hpp:516-527 (constructor initialiser list). */
void cmio_subgrid_init(cmio_subgrid *sg, const double box[6], const int32_t ncell[3]) {
  for (int a = 0; a < 3; ++a) {
    sg->anchor[a] = box[a];
    sg->cell_size[a] = box[3 + a] / ncell[a];
    sg->inv_cell_size[a] = ncell[a] / box[3 + a];
    sg->ncell[a] = ncell[a];
  }
  sg->ncell[3] = ncell[1] * ncell[2];
}

/* DensitySubGrid.hpp:247-414: the entry axes are clamped to the face the
 * packet enters through, the other axes are computed by truncation. */
static int axis_start_index(const cmio_subgrid *sg, double x, int axis, int input_direction) {
  const int s = kSigns[input_direction][axis];
  if (s == 0) {
    return (int)(x * sg->inv_cell_size[axis]);
  }
  return (s < 0) ? 0 : sg->ncell[axis] - 1;
}

/* DensitySubGrid.hpp:428-469. */
int cmio_get_start_index(const cmio_subgrid *sg, const double position[3],
                         int input_direction, int32_t three_index[3]) {
  for (int a = 0; a < 3; ++a) {
    three_index[a] = axis_start_index(sg, position[a], a, input_direction);
  }
  return three_index[0] * sg->ncell[3] + three_index[1] * sg->ncell[2] + three_index[2];
}

/* DensitySubGrid.hpp:483-506. */
int cmio_get_output_direction(const cmio_subgrid *sg, const int32_t three_index[3]) {
  int mask = 0;
  for (int a = 0; a < 3; ++a) {
    const int low = three_index[a] < 0;
    const int high = (three_index[a] / sg->ncell[a]) > 0;
    mask |= (high << (5 - 2 * a)) | (low << (4 - 2 * a));
  }
  return cmio_direction_from_mask(mask);
}

static inline int is_inside3(const int32_t idx[3], const int32_t n[3]) {
  return idx[0] < n[0] && idx[0] >= 0 && idx[1] < n[1] && idx[1] >= 0 && idx[2] < n[2] &&
         idx[2] >= 0;
}

/* std::min semantics: min(a, b) = (b < a) ? b : a. */
static inline double min_d(double a, double b) { return (b < a) ? b : a; }
static inline float min_f(float a, float b) { return (b < a) ? b : a; }

/* DensitySubGrid::interact, DensitySubGrid.hpp:1180-1323. */
/* mode 0: DensitySubGrid::interact (DensitySubGrid.hpp:1180-1323); 1: propagate, the same
 * walk without the J tally (:1333-1472); 2: compute_optical_depth, no target, the depth of
 * the whole crossing added to the photon (:1482-1604). */
static int walk_mode(const cmio_subgrid *sg, const double *nH, const double *xH, double *J,
                     cmio_photon *photon, int input_direction, int32_t *trace_cells,
                     double *trace_lengths, int32_t max_steps, int32_t *nsteps, int mode) {
  const double *d = photon->direction;
  const double inv[3] = {1. / d[0], 1. / d[1], 1. / d[2]};
  double pos[3] = {photon->position[0] - sg->anchor[0], photon->position[1] - sg->anchor[1],
                   photon->position[2] - sg->anchor[2]};
  double tau_done = 0.;
  const double tau_target = photon->target_optical_depth;
  const double sigma = photon->cross_section;
  const double weight = photon->weight;
  int32_t idx[3];
  int cell = cmio_get_start_index(sg, pos, input_direction, idx);
  int32_t steps = 0;
  while ((mode == 2 || tau_done < tau_target) && is_inside3(idx, sg->ncell)) {
    const double lo[3] = {idx[0] * sg->cell_size[0], idx[1] * sg->cell_size[1],
                          idx[2] * sg->cell_size[2]};
    const double hi[3] = {(idx[0] + 1.) * sg->cell_size[0], (idx[1] + 1.) * sg->cell_size[1],
                          (idx[2] + 1.) * sg->cell_size[2]};
    double l[3];
    for (int a = 0; a < 3; ++a) {
      if (d[a] > 0.) {
        l[a] = (hi[a] - pos[a]) * inv[a];
      } else if (d[a] < 0.) {
        l[a] = (lo[a] - pos[a]) * inv[a];
      } else {
        l[a] = DBL_MAX;
      }
    }
    double lmin = min_d(l[0], min_d(l[1], l[2]));
    double lminsigma = lmin * sigma;
    const double tau = lminsigma * nH[cell] * xH[cell];
    tau_done += tau;
    if (mode != 2 && tau_done >= tau_target) {
      const double correction = (tau_done - tau_target) / tau;
      lmin *= (1. - correction);
      lminsigma = lmin * sigma;
    } else {
      for (int a = 0; a < 3; ++a) {
        if (l[a] == lmin) {
          idx[a] += (d[a] > 0.) ? 1 : -1;
        }
      }
    }
    if (mode == 0) J[cell] += lminsigma * weight;
    if (trace_cells != NULL && steps < max_steps) {
      trace_cells[steps] = cell;
      trace_lengths[steps] = lmin;
    }
    ++steps;
    for (int a = 0; a < 3; ++a) {
      pos[a] = (l[a] == lmin) ? ((d[a] > 0.) ? hi[a] : lo[a]) : pos[a] + lmin * d[a];
    }
    cell = idx[0] * sg->ncell[3] + idx[1] * sg->ncell[2] + idx[2];
  }
  photon->target_optical_depth = (mode == 2) ? tau_target + tau_done : tau_target - tau_done;
  for (int a = 0; a < 3; ++a) {
    photon->position[a] = pos[a] + sg->anchor[a];
  }
  if (nsteps != NULL) {
    *nsteps = steps;
  }
  if (mode != 2 && tau_done >= tau_target) {
    return CMIO_INSIDE;
  }
  return cmio_get_output_direction(sg, idx);
}

int cmio_interact(const cmio_subgrid *sg, const double *nH, const double *xH, double *J,
                  cmio_photon *photon, int input_direction, int32_t *trace_cells,
                  double *trace_lengths, int32_t max_steps, int32_t *nsteps) {
  return walk_mode(sg, nH, xH, J, photon, input_direction, trace_cells, trace_lengths,
                   max_steps, nsteps, 0);
}

int cmio_propagate(const cmio_subgrid *sg, const double *nH, const double *xH,
                   cmio_photon *photon, int input_direction, int32_t *nsteps) {
  return walk_mode(sg, nH, xH, NULL, photon, input_direction, NULL, NULL, 0, nsteps, 1);
}

int cmio_compute_optical_depth(const cmio_subgrid *sg, const double *nH, const double *xH,
                               cmio_photon *photon, int input_direction, int32_t *nsteps) {
  return walk_mode(sg, nH, xH, NULL, photon, input_direction, NULL, NULL, 0, nsteps, 2);
}

/* FP32 cell-unit walk.  Same loop as interact above, with positions in cell
 * units relative to the subgrid (cell faces are exact small integers) and
 * path lengths in metres: l = (face - p) * (cell_size / d).  On exit the
 * position is re-expressed relative to the neighbour across the exit face
 * (exact: the exit coordinate is 0 or n). */
float cmio_fixed_scale(const cmio_subgrid *sg) {
  float lref = 0.f;
  for (int a = 0; a < 3; ++a) {
    const float cs = (float)sg->cell_size[a];
    lref = (cs > lref) ? cs : lref;
  }
  return 4194304.f / lref;
}

int cmio_interact32(const int32_t ncell[3], const float cell_size[3],
                    const float inv_cell_size[3], const float *kappa, double *tally,
                    uint64_t *fixed, float scale, cmio_packet32 *packet, int32_t *trace_cells,
                    float *trace_lengths, int32_t max_steps, int32_t *nsteps) {
  const int in_dir = (int)(packet->meta & 31u);
  const float *d = packet->dir;
  float p[3] = {packet->pos[0], packet->pos[1], packet->pos[2]};
  float inv[3], dcs[3];
  int32_t idx[3];
  for (int a = 0; a < 3; ++a) {
    /* correctly rounded reciprocal and products (no divisions) */
    dcs[a] = d[a] * inv_cell_size[a];
    inv[a] = cell_size[a] * (1.f / d[a]);
    const int s = kSigns[in_dir][a];
    idx[a] = (s == 0) ? (int32_t)p[a] : ((s < 0) ? 0 : ncell[a] - 1);
  }
  const int32_t nyz = ncell[1] * ncell[2];
  int32_t cell = idx[0] * nyz + idx[1] * ncell[2] + idx[2];
  float tau_done = 0.f;
  const float tau_target = packet->tau_left;
  int32_t steps = 0;
  while (tau_done < tau_target && is_inside3(idx, ncell)) {
    float lo[3], hi[3], l[3];
    for (int a = 0; a < 3; ++a) {
      lo[a] = (float)idx[a];
      hi[a] = lo[a] + 1.f;
      if (d[a] > 0.f) {
        l[a] = (hi[a] - p[a]) * inv[a];
      } else if (d[a] < 0.f) {
        l[a] = (lo[a] - p[a]) * inv[a];
      } else {
        l[a] = FLT_MAX;
      }
    }
    float lmin = min_f(l[0], min_f(l[1], l[2]));
    const float tau = lmin * kappa[cell];
    tau_done += tau;
    if (tau_done >= tau_target) {
      const float correction = (tau_done - tau_target) / tau;
      lmin *= (1.f - correction);
    } else {
      for (int a = 0; a < 3; ++a) {
        if (l[a] == lmin) {
          idx[a] += (d[a] > 0.f) ? 1 : -1;
        }
      }
    }
    if (tally != NULL) {
      tally[cell] += (double)lmin;
    }
    if (fixed != NULL) {
      /* round half to even of lmin * scale (< 2^23), clamped at 0 */
      const float q = lmin * scale;
      fixed[cell] += (q > 0.f) ? (uint64_t)nearbyintf(q) : 0u;
    }
    if (trace_cells != NULL && steps < max_steps) {
      trace_cells[steps] = cell;
      trace_lengths[steps] = lmin;
    }
    ++steps;
    for (int a = 0; a < 3; ++a) {
      p[a] = (l[a] == lmin) ? ((d[a] > 0.f) ? hi[a] : lo[a]) : fmaf(lmin, dcs[a], p[a]);
    }
    cell = idx[0] * nyz + idx[1] * ncell[2] + idx[2];
  }
  packet->tau_left = tau_target - tau_done;
  if (nsteps != NULL) {
    *nsteps = steps;
  }
  int out = CMIO_INSIDE;
  if (!(tau_done >= tau_target)) {
    int mask = 0;
    for (int a = 0; a < 3; ++a) {
      const int low = idx[a] < 0;
      const int high = (idx[a] / ncell[a]) > 0;
      mask |= (high << (5 - 2 * a)) | (low << (4 - 2 * a));
      if (high) {
        p[a] -= (float)ncell[a];
      } else if (low) {
        p[a] += (float)ncell[a];
      }
    }
    out = cmio_direction_from_mask(mask);
  }
  packet->pos[0] = p[0];
  packet->pos[1] = p[1];
  packet->pos[2] = p[2];
  return out;
}

/* FP32 optical depth of a mixed-precision packet: round to nearest; a
 * positive depth below the FP32 range becomes the smallest subnormal. */
static float tau32(double tau) {
  const float f = (float)tau;
  return (f == 0.f && tau > 0.) ? 1.40129846e-45f : f;
}

/* Mixed-precision walk: interact's loop (DensitySubGrid.hpp:1186-1305) with
 * the geometry of walk_mode above, operation for operation, and the optical
 * depth of each crossing in FP32 from the cell's FP32 opacity. */
int cmio_interact_mixed(const cmio_subgrid *sg, const float *kappa, double *tally,
                        uint64_t *fixed, float scale, cmio_packetm *packet,
                        int32_t *trace_cells, double *trace_lengths, int32_t max_steps,
                        int32_t *nsteps) {
  const int in_dir = (int)(packet->meta & 31u);
  const double *d = packet->dir;
  const double inv[3] = {1. / d[0], 1. / d[1], 1. / d[2]};
  double pos[3] = {packet->pos[0] - sg->anchor[0], packet->pos[1] - sg->anchor[1],
                   packet->pos[2] - sg->anchor[2]};
  float tau_done = 0.f;
  const float tau_target = packet->tau_left;
  int32_t idx[3];
  int cell = cmio_get_start_index(sg, pos, in_dir, idx);
  int32_t steps = 0;
  while (tau_done < tau_target && is_inside3(idx, sg->ncell)) {
    const double lo[3] = {idx[0] * sg->cell_size[0], idx[1] * sg->cell_size[1],
                          idx[2] * sg->cell_size[2]};
    const double hi[3] = {(idx[0] + 1.) * sg->cell_size[0], (idx[1] + 1.) * sg->cell_size[1],
                          (idx[2] + 1.) * sg->cell_size[2]};
    double l[3];
    for (int a = 0; a < 3; ++a) {
      if (d[a] > 0.) {
        l[a] = (hi[a] - pos[a]) * inv[a];
      } else if (d[a] < 0.) {
        l[a] = (lo[a] - pos[a]) * inv[a];
      } else {
        l[a] = DBL_MAX;
      }
    }
    double lmin = min_d(l[0], min_d(l[1], l[2]));
    float lf = (float)lmin;
    const float tau = lf * kappa[cell];
    const float tau_before = tau_done;
    tau_done += tau;
    if (tau_done >= tau_target) {
      /* the absorbed fraction 1 - (tau_done - tau_target) / tau of the
       * reference, as (tau_target - tau_before) / tau: no cancellation when
       * the packet stops early in the cell */
      float fraction = (tau_target - tau_before) / tau;
      fraction = (fraction < 1.f) ? fraction : 1.f;
      lmin *= (double)fraction;
      lf = (float)lmin;
    } else {
      for (int a = 0; a < 3; ++a) {
        if (l[a] == lmin) {
          idx[a] += (d[a] > 0.) ? 1 : -1;
        }
      }
    }
    if (tally != NULL) {
      tally[cell] += (double)lf;
    }
    if (fixed != NULL) {
      /* round half to even of lf * scale (< 2^23), clamped at 0 */
      const float q = lf * scale;
      fixed[cell] += (q > 0.f) ? (uint64_t)nearbyintf(q) : 0u;
    }
    if (trace_cells != NULL && steps < max_steps) {
      trace_cells[steps] = cell;
      trace_lengths[steps] = lmin;
    }
    ++steps;
    for (int a = 0; a < 3; ++a) {
      pos[a] = (l[a] == lmin) ? ((d[a] > 0.) ? hi[a] : lo[a]) : pos[a] + lmin * d[a];
    }
    cell = idx[0] * sg->ncell[3] + idx[1] * sg->ncell[2] + idx[2];
  }
  packet->tau_left = tau_target - tau_done;
  for (int a = 0; a < 3; ++a) {
    packet->pos[a] = pos[a] + sg->anchor[a];
  }
  if (nsteps != NULL) {
    *nsteps = steps;
  }
  if (tau_done >= tau_target) {
    return CMIO_INSIDE;
  }
  return cmio_get_output_direction(sg, idx);
}

/* ------------------------------------------------------------------------ */
/* Ionization balance, DensitySubGrid.hpp:1628-1658.                         */
/* ------------------------------------------------------------------------ */
double cmio_jfac(double luminosity, double num_photon, const double inv_cell_size[3]) {
  return luminosity / num_photon * inv_cell_size[0] * inv_cell_size[1] * inv_cell_size[2];
}

void cmio_compute_neutral_fraction(int64_t ncell, const double *nH, double *xH, double *J,
                                   double jfac, double alpha_H, int form) {
  for (int64_t i = 0; i < ncell; ++i) {
    const double jH = jfac * J[i];
    if (jH > 0.) {
      const double ntot = nH[i];
      const double aa = 0.5 * jH / (ntot * alpha_H);
      if (form == 0) {
        const double bb = 2. / aa;
        const double cc = sqrt(bb + 1.);
        xH[i] = 1. + aa * (1. - cc);
      } else {
        xH[i] = 1. / (1. + aa + sqrt(aa * (aa + 2.)));
      }
    } else {
      xH[i] = 1.;
    }
    J[i] = 0.;
  }
}

/* ------------------------------------------------------------------------ */
/* ranlxd generator, RandomGenerator.hpp:36-232 (restating GSL ranlxd with   */
/* luxury 397; the sequence must match bit for bit).                         */
/* ------------------------------------------------------------------------ */
#define RL_ONE_BIT (1.0 / 281474976710656.0) /* 2^-48 */

/* One subtract-with-borrow step at slot ir with partner slot jr. */
static inline void rl_step(double *x, double *carry, uint32_t ir, uint32_t jr) {
  double y = x[jr] - x[ir];
  y = y - *carry;
  if (y < 0) {
    *carry = RL_ONE_BIT;
    y += 1;
  } else {
    *carry = 0;
  }
  x[ir] = y;
}

/* RandomGenerator.hpp:80-150.  Leading single steps until ir wraps to 0,
 * then 12-step blocks whose partner slot is (i+7) mod 12, then trailing
 * single steps up to pr. */
static void rl_increment(cmio_ranlux *r) {
  double *x = r->x;
  double carry = r->carry;
  uint32_t ir = r->ir;
  uint32_t jr = r->jr;
  int32_t k = 0;
  for (; ir > 0; ++k) {
    rl_step(x, &carry, ir, jr);
    ir = (ir + 1) % 12;
    jr = (jr + 1) % 12;
  }
  const int32_t kblock = (int32_t)r->pr - 12;
  for (; k <= kblock; k += 12) {
    for (uint32_t i = 0; i < 12; ++i) {
      rl_step(x, &carry, i, (i + 7) % 12);
    }
  }
  for (; k < (int32_t)r->pr; ++k) {
    rl_step(x, &carry, ir, jr);
    ir = (ir + 1) % 12;
    jr = (jr + 1) % 12;
  }
  r->ir = ir;
  r->ir_old = ir;
  r->jr = jr;
  r->carry = carry;
}

/* RandomGenerator.hpp:158-197. */
void cmio_ranlux_seed(cmio_ranlux *r, int32_t seed) {
  if (seed == 0) {
    seed = 1;
  }
  int32_t bits[31];
  int32_t v = seed & 0x7FFFFFFF;
  for (int k = 0; k < 31; ++k) {
    bits[k] = v % 2;
    v /= 2;
  }
  int ib = 0, jb = 18;
  for (int k = 0; k < 12; ++k) {
    double acc = 0;
    for (int m = 1; m <= 48; ++m) {
      const double y = (double)((bits[ib] + 1) % 2);
      acc += acc + y;
      bits[ib] = (bits[ib] + bits[jb]) % 2;
      ib = (ib + 1) % 31;
      jb = (jb + 1) % 31;
    }
    r->x[k] = RL_ONE_BIT * acc;
  }
  r->carry = 0;
  r->ir = 11;
  r->jr = 7;
  r->ir_old = 0;
  r->pr = 397;
}

/* RandomGenerator.hpp:214-222. */
double cmio_ranlux_uniform(cmio_ranlux *r) {
  r->ir = (r->ir + 1) % 12;
  if (r->ir == r->ir_old) {
    rl_increment(r);
  }
  return r->x[r->ir];
}

/* ------------------------------------------------------------------------ */
/* Emission, testDensitySubGrid_omp.cpp:529-597.                             */
/* ------------------------------------------------------------------------ */
void cmio_random_direction(cmio_ranlux *rng, double direction[3]) {
  const double cost = 2. * cmio_ranlux_uniform(rng) - 1.;
  const double phi = 2. * M_PI * cmio_ranlux_uniform(rng);
  const double s2 = 1. - cost * cost;
  const double sint = sqrt((s2 < 0.) ? 0. : s2);
  const double cosp = cos(phi);
  const double sinp = sin(phi);
  direction[0] = sint * cosp;
  direction[1] = sint * sinp;
  direction[2] = cost;
}

void cmio_fill_packets(cmio_ranlux *rng, const double source_position[3], cmio_photon *out,
                       int32_t n, double cross_section) {
  for (int32_t i = 0; i < n; ++i) {
    cmio_photon *p = &out[i];
    memset(p, 0, sizeof(*p));
    p->position[0] = source_position[0];
    p->position[1] = source_position[1];
    p->position[2] = source_position[2];
    cmio_random_direction(rng, p->direction);
    p->weight = 1.;
    p->target_optical_depth = -log(cmio_ranlux_uniform(rng));
    p->cross_section = cross_section;
  }
}

void cmio_fill_buffer_stream(int32_t seed, const double source_position[3], cmio_photon *out,
                             int32_t n, double cross_section) {
  cmio_ranlux rng;
  cmio_ranlux_seed(&rng, seed);
  (void)cmio_ranlux_uniform(&rng); /* Source::get_subgrid_index draw */
  cmio_fill_packets(&rng, source_position, out, n, cross_section);
}

/* Correctly rounded sin, cos and -log of the CUDA library's replay of the
 * reference emission streams (restated: double-double arithmetic after
 * Dekker and Knuth, Cody-Waite reduction by pi/2 in three parts, Taylor
 * series of sin and cos to x^29 / 29!, -ln u = -(e ln 2 + 2 atanh s) with the
 * atanh series to s^45 / 45).  Every operation is a correctly rounded IEEE
 * operation or an fma, so host and device give the same bits. */
typedef struct {
  double hi, lo;
} cmio_dd;
static cmio_dd dd_two_sum(double a, double b) {
  const double s = a + b, bb = s - a;
  const cmio_dd r = {s, (a - (s - bb)) + (b - bb)};
  return r;
}
static cmio_dd dd_fast_two_sum(double a, double b) {
  const double s = a + b;
  const cmio_dd r = {s, b - (s - a)};
  return r;
}
static cmio_dd dd_two_prod(double a, double b) {
  const double p = a * b;
  const cmio_dd r = {p, fma(a, b, -p)};
  return r;
}
static cmio_dd dd_add(cmio_dd a, cmio_dd b) {
  cmio_dd s = dd_two_sum(a.hi, b.hi);
  const cmio_dd t = dd_two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = dd_fast_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return dd_fast_two_sum(s.hi, s.lo);
}
static cmio_dd dd_mul(cmio_dd a, cmio_dd b) {
  cmio_dd p = dd_two_prod(a.hi, b.hi);
  p.lo += a.hi * b.lo + a.lo * b.hi;
  return dd_fast_two_sum(p.hi, p.lo);
}
static cmio_dd dd_div_d(cmio_dd a, double b) {
  const double q1 = a.hi / b;
  const cmio_dd p = dd_two_prod(q1, b);
  cmio_dd s = dd_two_sum(a.hi, -p.hi);
  s.lo = (s.lo - p.lo) + a.lo;
  return dd_fast_two_sum(q1, (s.hi + s.lo) / b);
}
static cmio_dd dd_div(cmio_dd a, cmio_dd b) {
  const double q1 = a.hi / b.hi;
  const cmio_dd m1 = {-q1, 0.};
  cmio_dd r = dd_add(a, dd_mul(m1, b));
  const double q2 = r.hi / b.hi;
  const cmio_dd m2 = {-q2, 0.};
  r = dd_add(r, dd_mul(m2, b));
  const cmio_dd q3 = {r.hi / b.hi, 0.};
  return dd_add(dd_fast_two_sum(q1, q2), q3);
}

void cmio_cr_sincos(double x, double *sn, double *cs) {
  const double P1 = 0x1.921fb54442d18p+0, P2 = 0x1.1a62633145c07p-54,
               P3 = -0x1.f1976b7ed8fbcp-110;
  const double k = nearbyint(x * (1. / P1));
  cmio_dd r = {x - k * P1, 0.};
  r = dd_add(r, dd_two_prod(-k, P2));
  const cmio_dd r3 = {-k * P3, 0.};
  r = dd_add(r, r3);
  const cmio_dd r2 = dd_mul(r, r);
  const cmio_dd one = {1., 0.};
  cmio_dd ts = one, tc = one;
  for (int n = 14; n >= 1; --n) {
    ts = dd_add(one, dd_div_d(dd_mul(r2, ts), -(double)((2 * n) * (2 * n + 1))));
    tc = dd_add(one, dd_div_d(dd_mul(r2, tc), -(double)((2 * n - 1) * (2 * n))));
  }
  const cmio_dd s = dd_mul(r, ts);
  const double sv = s.hi + s.lo, cv = tc.hi + tc.lo;
  const int q = ((int)k) & 3;
  *sn = (q == 0) ? sv : (q == 1) ? cv : (q == 2) ? -sv : -cv;
  *cs = (q == 0) ? cv : (q == 1) ? -sv : (q == 2) ? -cv : sv;
}

double cmio_cr_neg_log(double u) {
  if (u == 0.) return INFINITY;
  int e;
  double m = frexp(u, &e);
  if (m < 0.70710678118654752440) {
    m *= 2.;
    e -= 1;
  }
  const cmio_dd one = {1., 0.}, num = {m - 1., 0.}, two = {2., 0.};
  const cmio_dd s = dd_div(num, dd_two_sum(m, 1.));
  const cmio_dd s2 = dd_mul(s, s);
  cmio_dd t = {0., 0.};
  for (int k = 22; k >= 0; --k) t = dd_add(dd_div_d(one, (double)(2 * k + 1)), dd_mul(s2, t));
  const cmio_dd lm = dd_mul(dd_mul(two, s), t);
  const double L2H = 0x1.62e42fefa39efp-1, L2L = 0x1.abc9e3b39803fp-56;
  const cmio_dd el0 = {L2L * (double)e, 0.};
  const cmio_dd el = dd_add(dd_two_prod(L2H, (double)e), el0);
  const cmio_dd l = dd_add(el, lm);
  return -(l.hi + l.lo);
}

/* The reference's fill_buffer stream (testDensitySubGrid_omp.cpp:529-597)
 * with the correctly rounded functions above in place of cos, sin and log. */
void cmio_fill_buffer_stream_cr(int32_t seed, const double source_position[3],
                                cmio_photon *out, int32_t n, double cross_section) {
  cmio_ranlux rng;
  cmio_ranlux_seed(&rng, seed);
  (void)cmio_ranlux_uniform(&rng); /* Source::get_subgrid_index draw */
  for (int32_t i = 0; i < n; ++i) {
    cmio_photon *p = &out[i];
    memset(p, 0, sizeof(*p));
    for (int a = 0; a < 3; ++a) p->position[a] = source_position[a];
    const double cost = 2. * cmio_ranlux_uniform(&rng) - 1.;
    const double phi = 2. * M_PI * cmio_ranlux_uniform(&rng);
    const double s2 = 1. - cost * cost;
    const double sint = sqrt((s2 < 0.) ? 0. : s2);
    double sinp, cosp;
    cmio_cr_sincos(phi, &sinp, &cosp);
    p->direction[0] = sint * cosp;
    p->direction[1] = sint * sinp;
    p->direction[2] = cost;
    p->weight = 1.;
    p->target_optical_depth = cmio_cr_neg_log(cmio_ranlux_uniform(&rng));
    p->cross_section = cross_section;
  }
}

/* testDensitySubGrid_omp.cpp:2199-2208: packets proportional to luminosity. */
void cmio_source_numbers(int32_t nsrc, const double *luminosity, uint32_t num_photon,
                         uint32_t *numbers) {
  double total = 0.;
  for (int32_t i = 0; i < nsrc; ++i) {
    total += luminosity[i];
  }
  for (int32_t i = 0; i < nsrc; ++i) {
    numbers[i] = (uint32_t)(luminosity[i] / total * num_photon);
  }
}

/* testDensitySubGrid_omp.cpp:1650-1677: the distribute_number smallest of
 * total_number uniform draws receive one extra packet. */
typedef struct {
  double v;
  int32_t i;
} rl_pair;
static int cmp_pair(const void *a, const void *b) {
  const rl_pair *x = (const rl_pair *)a, *y = (const rl_pair *)b;
  if (x->v < y->v) return -1;
  if (y->v < x->v) return 1;
  return (x->i < y->i) ? -1 : (x->i > y->i);
}
void cmio_distribute(int32_t total_number, int32_t distribute_number, cmio_ranlux *rng,
                     uint32_t *result) {
  rl_pair *p = (rl_pair *)malloc(sizeof(rl_pair) * (size_t)(total_number > 0 ? total_number : 1));
  for (int32_t i = 0; i < total_number; ++i) {
    p[i].v = cmio_ranlux_uniform(rng);
    p[i].i = i;
    result[i] = 0;
  }
  qsort(p, (size_t)total_number, sizeof(rl_pair), cmp_pair);
  for (int32_t i = 0; i < distribute_number && i < total_number; ++i) {
    result[p[i].i] = 1;
  }
  free(p);
}

/* ------------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).                        */
/* ------------------------------------------------------------------------ */
void cmio_philox4x32(const uint32_t counter[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = counter[0], c1 = counter[1], c2 = counter[2], c3 = counter[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; ++r) {
    if (r > 0) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    const uint32_t n1 = (uint32_t)p1;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    const uint32_t n3 = (uint32_t)p0;
    c0 = n0;
    c1 = n1;
    c2 = n2;
    c3 = n3;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

void cmio_philox_packet(uint64_t seed, uint32_t stream, uint64_t packet, double direction[3],
                        double *tau) {
  const uint32_t ctr[4] = {(uint32_t)packet, (uint32_t)(packet >> 32), stream, 0x434D4901u};
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t w[4];
  cmio_philox4x32(ctr, key, w);
  const double u0 = ((double)w[0] + 0.5) * (1.0 / 4294967296.0);
  const double u1 = ((double)w[1] + 0.5) * (1.0 / 4294967296.0);
  const uint64_t k53 = ((uint64_t)w[2] << 21) ^ (uint64_t)(w[3] >> 11);
  const double u2 = ((double)k53 + 0.5) * (1.0 / 9007199254740992.0);
  const double cost = 2. * u0 - 1.;
  const double phi = 2. * M_PI * u1;
  const double s2 = 1. - cost * cost;
  const double sint = sqrt((s2 < 0.) ? 0. : s2);
  direction[0] = sint * cos(phi);
  direction[1] = sint * sin(phi);
  direction[2] = cost;
  *tau = -log(u2);
}

/* ------------------------------------------------------------------------ */
/* Lattice of subgrids (testDensitySubGrid_omp.cpp:1801-1877).               */
/* ------------------------------------------------------------------------ */
int cmio_lattice_init(cmio_lattice *lat, const double box[6], const int32_t ncell[3],
                      const int32_t num_subgrid[3]) {
  memset(lat, 0, sizeof(*lat));
  for (int a = 0; a < 3; ++a) {
    if (num_subgrid[a] <= 0 || ncell[a] % num_subgrid[a] != 0) {
      return -1;
    }
    lat->num_subgrid[a] = num_subgrid[a];
    lat->sub_ncell[a] = ncell[a] / num_subgrid[a];
  }
  lat->cells_per_subgrid = (int64_t)lat->sub_ncell[0] * lat->sub_ncell[1] * lat->sub_ncell[2];
  lat->nsub = (int64_t)num_subgrid[0] * num_subgrid[1] * num_subgrid[2];
  lat->sub = (cmio_subgrid *)calloc((size_t)lat->nsub, sizeof(cmio_subgrid));
  lat->ngb = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)lat->nsub * CMIO_NUM_DIRECTIONS);
  const double side[3] = {box[3] / num_subgrid[0], box[4] / num_subgrid[1],
                          box[5] / num_subgrid[2]};
  const int32_t ns1 = num_subgrid[1], ns2 = num_subgrid[2];
  for (int64_t s = 0; s < lat->nsub; ++s) {
    const int32_t ix = (int32_t)(s / (ns1 * ns2));
    const int32_t iy = (int32_t)((s - (int64_t)ix * ns1 * ns2) / ns2);
    const int32_t iz = (int32_t)(s - (int64_t)ix * ns1 * ns2 - (int64_t)iy * ns2);
    const double sbox[6] = {box[0] + ix * side[0], box[1] + iy * side[1], box[2] + iz * side[2],
                            side[0], side[1], side[2]};
    cmio_subgrid_init(&lat->sub[s], sbox, lat->sub_ncell);
    uint32_t *ngb = &lat->ngb[s * CMIO_NUM_DIRECTIONS];
    for (int d = 0; d < CMIO_NUM_DIRECTIONS; ++d) {
      ngb[d] = CMIO_NEIGHBOUR_OUTSIDE;
    }
    for (int nx = -1; nx < 2; ++nx) {
      for (int ny = -1; ny < 2; ++ny) {
        for (int nz = -1; nz < 2; ++nz) {
          const int cx = ix + nx, cy = iy + ny, cz = iz + nz;
          if (cx >= 0 && cx < num_subgrid[0] && cy >= 0 && cy < ns1 && cz >= 0 && cz < ns2) {
            ngb[direction_from_signs(nx, ny, nz)] = (uint32_t)((cx * ns1 + cy) * ns2 + cz);
          }
        }
      }
    }
  }
  return 0;
}

void cmio_lattice_free(cmio_lattice *lat) {
  free(lat->sub);
  free(lat->ngb);
  memset(lat, 0, sizeof(*lat));
}

uint32_t cmio_lattice_locate(const cmio_lattice *lat, const double box[6],
                             const double position[3]) {
  uint32_t i3[3];
  for (int a = 0; a < 3; ++a) {
    int64_t v = (int64_t)((position[a] - box[a]) / box[3 + a] * lat->num_subgrid[a]);
    if (v < 0) v = 0;
    if (v >= lat->num_subgrid[a]) v = lat->num_subgrid[a] - 1;
    i3[a] = (uint32_t)v;
  }
  return (i3[0] * lat->num_subgrid[1] + i3[1]) * lat->num_subgrid[2] + i3[2];
}

/* do_photon_traversal + routing (testDensitySubGrid_omp.cpp:607-666,
 * 1178-1191) applied to one packet at a time until absorption (INSIDE with
 * reemission off) or escape (neighbour NEIGHBOUR_OUTSIDE). */
uint32_t cmio_reemit_hash(double x) {
  uint64_t b;
  memcpy(&b, &x, sizeof(b));
  return (uint32_t)b ^ (uint32_t)(b >> 32);
}

static uint32_t float_bits(float x) {
  uint32_t b;
  memcpy(&b, &x, sizeof(b));
  return b;
}

/* -ln(u), the GPU's series: u = m 2^e with m in [sqrt(1/2), sqrt(2)),
 * ln m = 2 (s + s^3/3 + ... + s^31/31), s = (m - 1) / (m + 1) */
static double reemit_neg_log(double u) {
  int e;
  double m = frexp(u, &e);
  if (m < 0.70710678118654752440) {
    m *= 2.;
    e -= 1;
  }
  const double s = (m - 1.) / (m + 1.);
  const double s2 = s * s;
  double term = s, sum = s;
  for (int k = 3; k <= 31; k += 2) {
    term *= s2;
    sum += term / (double)k;
  }
  return -(2. * sum + (double)e * 0.69314718055994530942);
}

/* do_reemission (testDensitySubGrid_omp.cpp:675-702) with the GPU's
 * counter-based draws: Marsaglia's direction (attempt k uses tag + k) and the
 * series above, correctly rounded operations only, so both sides agree bit
 * for bit */
int cmio_reemit_draw(const cmio_reemission *r, uint32_t h0, uint32_t h1, uint32_t h2,
                     uint32_t count, double direction[3], double *tau) {
  const double inv32 = 1.0 / 4294967296.0;
  const uint32_t key[2] = {(uint32_t)r->seed, (uint32_t)(r->seed >> 32) + r->instance};
  if (count >= 1024u) return 0; /* the GPU's cap per subgrid visit */
  for (uint32_t k = 0; k < 16u; ++k) {
    const uint32_t ctr[4] = {h0, h1, h2 ^ r->iteration, 0x434D4952u + (count << 4) + k};
    uint32_t w[4];
    cmio_philox4x32(ctr, key, w);
    if (k == 0u && !(((double)w[0] + 0.5) * inv32 < r->probability)) return 0;
    const double x1 = 2. * (((double)w[1] + 0.5) * inv32) - 1.;
    const double x2 = 2. * (((double)w[2] + 0.5) * inv32) - 1.;
    const double s = x1 * x1 + x2 * x2;
    if (s < 1.) {
      const double f = 2. * sqrt(1. - s);
      direction[0] = x1 * f;
      direction[1] = x2 * f;
      direction[2] = 1. - 2. * s;
      *tau = reemit_neg_log(((double)w[3] + 0.5) * inv32);
      return 1;
    }
  }
  direction[0] = 0.;
  direction[1] = 0.;
  direction[2] = 1.;
  *tau = 1.;
  return 1;
}

void cmio_transport_r(const cmio_lattice *lat, const double *nH, const double *xH, double *J,
                      cmio_photon *packets, const uint32_t *start_subgrid, int64_t n,
                      cmio_counts *counts, const cmio_reemission *r) {
  const int64_t C = lat->cells_per_subgrid;
  for (int64_t i = 0; i < n; ++i) {
    uint32_t s = start_subgrid[i];
    int in_dir = CMIO_INSIDE;
    uint32_t rcount = 0; /* reemissions in this subgrid visit */
    for (;;) {
      int32_t steps = 0;
      const int out = cmio_interact(&lat->sub[s], nH + s * C, xH + s * C, J + s * C, &packets[i],
                                    in_dir, NULL, NULL, 0, &steps);
      counts->crossings += (uint64_t)steps;
      counts->transits += 1;
      if (out == CMIO_INSIDE) {
        double d[3], tau;
        cmio_photon *ph = &packets[i];
        if (r && r->probability > 0. &&
            cmio_reemit_draw(r, cmio_reemit_hash(ph->position[0]),
                             cmio_reemit_hash(ph->position[1]),
                             cmio_reemit_hash(ph->position[2]), rcount, d, &tau)) {
          counts->reemitted += 1;
          rcount += 1;
          for (int a = 0; a < 3; ++a) ph->direction[a] = d[a];
          ph->target_optical_depth = tau;
          in_dir = CMIO_INSIDE;
          continue;  /* a new traversal of the same subgrid */
        }
        counts->absorbed += 1;
        break;
      }
      const uint32_t ngb = lat->ngb[s * CMIO_NUM_DIRECTIONS + out];
      if (ngb == CMIO_NEIGHBOUR_OUTSIDE) {
        counts->escaped += 1;
        break;
      }
      s = ngb;
      in_dir = cmio_output_to_input_direction(out);
      rcount = 0;
    }
  }
}

void cmio_transport(const cmio_lattice *lat, const double *nH, const double *xH, double *J,
                    cmio_photon *packets, const uint32_t *start_subgrid, int64_t n,
                    cmio_counts *counts) {
  cmio_transport_r(lat, nH, xH, J, packets, start_subgrid, n, counts, NULL);
}

void cmio_transport32_r(const cmio_lattice *lat, const float *kappa, double *tally,
                        uint64_t *fixed, cmio_packet32 *packets, const uint32_t *start_subgrid,
                        int64_t n, cmio_counts *counts, const cmio_reemission *r) {
  const int64_t C = lat->cells_per_subgrid;
  for (int64_t i = 0; i < n; ++i) {
    uint32_t s = start_subgrid[i];
    uint32_t rcount = 0; /* reemissions in this subgrid visit */
    for (;;) {
      const cmio_subgrid *sg = &lat->sub[s];
      const float cs[3] = {(float)sg->cell_size[0], (float)sg->cell_size[1],
                           (float)sg->cell_size[2]};
      const float ics[3] = {(float)sg->inv_cell_size[0], (float)sg->inv_cell_size[1],
                            (float)sg->inv_cell_size[2]};
      int32_t steps = 0;
      const int out = cmio_interact32(lat->sub_ncell, cs, ics, kappa + s * C,
                                      tally ? tally + s * C : NULL, fixed ? fixed + s * C : NULL,
                                      cmio_fixed_scale(sg), &packets[i], NULL, NULL, 0, &steps);
      counts->crossings += (uint64_t)steps;
      counts->transits += 1;
      if (out == CMIO_INSIDE) {
        double d[3], tau;
        cmio_packet32 *pk = &packets[i];
        if (r && r->probability > 0. &&
            cmio_reemit_draw(r, float_bits(pk->pos[0]) ^ s,
                             float_bits(pk->pos[1]) ^ (s * 0x9E3779B9u), float_bits(pk->pos[2]),
                             rcount, d, &tau)) {
          counts->reemitted += 1;
          rcount += 1;
          for (int a = 0; a < 3; ++a) pk->dir[a] = (float)d[a];
          pk->tau_left = (float)tau;
          pk->meta = (pk->meta & ~31u) | (uint32_t)CMIO_INSIDE;
          continue;
        }
        counts->absorbed += 1;
        break;
      }
      const uint32_t ngb = lat->ngb[s * CMIO_NUM_DIRECTIONS + out];
      if (ngb == CMIO_NEIGHBOUR_OUTSIDE) {
        counts->escaped += 1;
        break;
      }
      s = ngb;
      packets[i].meta = (packets[i].meta & ~31u) | (uint32_t)cmio_output_to_input_direction(out);
      rcount = 0;
    }
  }
}

void cmio_transport32(const cmio_lattice *lat, const float *kappa, double *tally,
                      uint64_t *fixed, cmio_packet32 *packets, const uint32_t *start_subgrid,
                      int64_t n, cmio_counts *counts) {
  cmio_transport32_r(lat, kappa, tally, fixed, packets, start_subgrid, n, counts, NULL);
}

void cmio_transportm_r(const cmio_lattice *lat, const float *kappa, double *tally,
                       uint64_t *fixed, cmio_packetm *packets, const uint32_t *start_subgrid,
                       int64_t n, cmio_counts *counts, const cmio_reemission *r) {
  const int64_t C = lat->cells_per_subgrid;
  for (int64_t i = 0; i < n; ++i) {
    uint32_t s = start_subgrid[i];
    uint32_t rcount = 0; /* reemissions in this subgrid visit */
    for (;;) {
      const cmio_subgrid *sg = &lat->sub[s];
      int32_t steps = 0;
      const int out = cmio_interact_mixed(sg, kappa + s * C, tally ? tally + s * C : NULL,
                                          fixed ? fixed + s * C : NULL, cmio_fixed_scale(sg),
                                          &packets[i], NULL, NULL, 0, &steps);
      counts->crossings += (uint64_t)steps;
      counts->transits += 1;
      if (out == CMIO_INSIDE) {
        double d[3], tau;
        cmio_packetm *pk = &packets[i];
        if (r && r->probability > 0. &&
            cmio_reemit_draw(r, cmio_reemit_hash(pk->pos[0]), cmio_reemit_hash(pk->pos[1]),
                             cmio_reemit_hash(pk->pos[2]), rcount, d, &tau)) {
          counts->reemitted += 1;
          rcount += 1;
          for (int a = 0; a < 3; ++a) pk->dir[a] = d[a];
          pk->tau_left = tau32(tau);
          pk->meta = (pk->meta & ~31u) | (uint32_t)CMIO_INSIDE;
          continue;
        }
        counts->absorbed += 1;
        break;
      }
      const uint32_t ngb = lat->ngb[s * CMIO_NUM_DIRECTIONS + out];
      if (ngb == CMIO_NEIGHBOUR_OUTSIDE) {
        counts->escaped += 1;
        break;
      }
      s = ngb;
      packets[i].meta = (packets[i].meta & ~31u) | (uint32_t)cmio_output_to_input_direction(out);
      rcount = 0;
    }
  }
}


void cmio_kappa32(int64_t ncell, const double *nH, const double *xH, double sigma,
                  float *kappa) {
  for (int64_t i = 0; i < ncell; ++i) {
    kappa[i] = (float)(sigma * nH[i] * xH[i]);
  }
}

void cmio_split_packets(int32_t nsrc, const double *luminosity, uint64_t num_photon,
                        uint64_t seed, uint32_t iteration, uint64_t *numbers) {
  double total = 0.;
  for (int32_t i = 0; i < nsrc; ++i) {
    total += luminosity[i];
  }
  uint64_t assigned = 0;
  for (int32_t i = 0; i < nsrc; ++i) {
    numbers[i] = (uint64_t)(luminosity[i] / total * (double)num_photon);
    assigned += numbers[i];
  }
  uint64_t rem = (num_photon > assigned) ? num_photon - assigned : 0;
  /* rank sources by a Philox draw; the rem smallest get one packet each */
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t *draw = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(nsrc > 0 ? nsrc : 1));
  for (int32_t i = 0; i < nsrc; ++i) {
    const uint32_t ctr[4] = {(uint32_t)i, 0u, iteration, 0x434D4902u};
    uint32_t w[4];
    cmio_philox4x32(ctr, key, w);
    draw[i] = w[0];
  }
  while (rem > 0) {
    int32_t best = -1;
    for (int32_t i = 0; i < nsrc; ++i) {
      if (draw[i] != 0xFFFFFFFFu || best < 0) {
        if (best < 0 || draw[i] < draw[best] || (draw[i] == draw[best] && i < best)) {
          best = i;
        }
      }
    }
    numbers[best] += 1;
    draw[best] = 0xFFFFFFFFu;
    --rem;
  }
  free(draw);
}

void cmio_iteration_omp(const cmio_lattice *lat, const double box[6], const double *nH,
                        double *xH, double *J, int32_t nsrc, const double *src_pos,
                        const double *src_lum, uint64_t num_photon, uint64_t seed,
                        uint32_t iteration, double alpha_H, double cross_section,
                        int balance_form, int threads, cmio_counts *counts) {
  const int64_t C = lat->cells_per_subgrid;
  const int64_t ncell = C * lat->nsub;
  uint64_t *numbers = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)nsrc);
  uint64_t *first = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(nsrc + 1));
  uint32_t *src_sub = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)nsrc);
  cmio_split_packets(nsrc, src_lum, num_photon, seed, iteration, numbers);
  first[0] = 0;
  double total_lum = 0.;
  for (int32_t i = 0; i < nsrc; ++i) {
    first[i + 1] = first[i] + numbers[i];
    src_sub[i] = cmio_lattice_locate(lat, box, &src_pos[3 * i]);
    total_lum += src_lum[i];
  }
  if (threads <= 0) {
#ifdef _OPENMP
    threads = omp_get_max_threads();
#else
    threads = 1;
#endif
  }
  double *priv = (double *)calloc((size_t)threads * (size_t)ncell, sizeof(double));
  uint64_t c_abs = 0, c_esc = 0, c_cross = 0, c_tr = 0;
#pragma omp parallel num_threads(threads) reduction(+ : c_abs, c_esc, c_cross, c_tr)
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    double *Jt = priv + (size_t)tid * (size_t)ncell;
    cmio_counts local = {0, 0, 0, 0, 0};
#pragma omp for schedule(dynamic, 4096)
    for (int64_t p = 0; p < (int64_t)num_photon; ++p) {
      int32_t src = 0;
      while (src + 1 < nsrc && (uint64_t)p >= first[src + 1]) {
        ++src;
      }
      cmio_photon ph;
      memset(&ph, 0, sizeof(ph));
      ph.position[0] = src_pos[3 * src];
      ph.position[1] = src_pos[3 * src + 1];
      ph.position[2] = src_pos[3 * src + 2];
      cmio_philox_packet(seed, iteration, (uint64_t)p, ph.direction, &ph.target_optical_depth);
      ph.cross_section = cross_section;
      ph.weight = 1.;
      const uint32_t s0 = src_sub[src];
      cmio_transport(lat, nH, xH, Jt, &ph, &s0, 1, &local);
    }
    c_abs += local.absorbed;
    c_esc += local.escaped;
    c_cross += local.crossings;
    c_tr += local.transits;
  }
#pragma omp parallel for num_threads(threads) schedule(static)
  for (int64_t i = 0; i < ncell; ++i) {
    double acc = J[i];
    for (int t = 0; t < threads; ++t) {
      acc += priv[(size_t)t * (size_t)ncell + (size_t)i];
    }
    J[i] = acc;
  }
  const double jfac = cmio_jfac(total_lum, (double)num_photon, lat->sub[0].inv_cell_size);
#pragma omp parallel for num_threads(threads) schedule(static)
  for (int64_t s = 0; s < lat->nsub; ++s) {
    cmio_compute_neutral_fraction(C, nH + s * C, xH + s * C, J + s * C, jfac, alpha_H,
                                  balance_form);
  }
  counts->absorbed += c_abs;
  counts->escaped += c_esc;
  counts->crossings += c_cross;
  counts->transits += c_tr;
  free(priv);
  free(numbers);
  free(first);
  free(src_sub);
}

/* ------------------------------------------------------------------------ */
/* Dust scattering with forced first scattering and peel-off image: the      */
/* photon loop of testDensitySubGrid_omp_dust.cpp (fill_buffer :564-620,     */
/* relaunch :1200-1260, do_photon_traversal :621-722, do_reemission          */
/* :730-760, peel-offs :1533-1560), with counter-based draws in place of the */
/* per-thread generators: the CUDA library's cmi_dust_run draws the same     */
/* numbers with the same correctly rounded operations.                       */
/* ------------------------------------------------------------------------ */
#define DUST_TAG 0x44555354u

/* exp(x), x <= 0: Cody-Waite reduction x = k ln2 + r, Taylor series of
 * exp(r) to r^18/18!, scaled by 2^k; 0 below e^-700 */
double cmio_dust_exp(double x) {
  if (!(x >= -700.)) return 0.;
  if (x > 0.) x = 0.;
  const double k = rint(x * 0x1.71547652b82fep+0);
  const double r = (x - k * 0x1.62e42fefa3800p-1) - k * 0x1.ef35793c76730p-45;
  double term = 1., sum = 1.;
  for (int n = 1; n <= 18; ++n) {
    term = term * r / (double)n;
    sum += term;
  }
  return ldexp(sum, (int)k);
}

static double dust_uniform(uint32_t w) { return ((double)w + 0.5) * (1.0 / 4294967296.0); }

static void dust_words(uint64_t seed, uint32_t instance, uint32_t iteration, uint32_t id,
                       uint32_t gen, uint32_t purpose, uint32_t attempt, uint32_t w[4]) {
  const uint32_t ctr[4] = {id, gen, iteration, DUST_TAG + (purpose << 8) + attempt};
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32) + instance};
  cmio_philox4x32(ctr, key, w);
}

static void dust_direction(uint64_t seed, uint32_t instance, uint32_t iteration, uint32_t id,
                           uint32_t gen, uint32_t purpose, double dir[3], uint32_t *w0,
                           uint32_t *w3) {
  for (uint32_t k = 0; k < 16u; ++k) {
    uint32_t w[4];
    dust_words(seed, instance, iteration, id, gen, purpose, k, w);
    if (k == 0u && w0) *w0 = w[0];
    const double x1 = 2. * dust_uniform(w[1]) - 1.;
    const double x2 = 2. * dust_uniform(w[2]) - 1.;
    const double ss = x1 * x1 + x2 * x2;
    if (ss < 1.) {
      const double f = 2. * sqrt(1. - ss);
      dir[0] = x1 * f;
      dir[1] = x2 * f;
      dir[2] = 1. - 2. * ss;
      if (w3) *w3 = w[3];
      return;
    }
  }
  dir[0] = 0.;
  dir[1] = 0.;
  dir[2] = 1.;
  if (w3) *w3 = 0x80000000u;
}

/* one packet from subgrid to subgrid; 0: absorbed, 1: left the box */
static int dust_walk(const cmio_lattice *lat, const double *nH, const double *xH,
                     cmio_photon *ph, uint32_t *sub, int mode, cmio_dust_stats *st) {
  const int64_t C = (int64_t)lat->sub_ncell[0] * lat->sub_ncell[1] * lat->sub_ncell[2];
  int in_dir = (int)ph->reserved;
  for (;;) {
    const uint32_t s = *sub;
    int32_t steps = 0;
    const int out = walk_mode(&lat->sub[s], nH + s * C, xH + s * C, NULL, ph, in_dir, NULL,
                              NULL, 0, &steps, mode);
    st->cell_crossings += (uint64_t)steps;
    st->subgrid_transits += 1;
    if (out == CMIO_INSIDE) return 0;
    const uint32_t ngb = lat->ngb[s * CMIO_NUM_DIRECTIONS + out];
    in_dir = cmio_output_to_input_direction(out);
    ph->reserved = in_dir;
    if (ngb == CMIO_NEIGHBOUR_OUTSIDE) return 1;
    *sub = ngb;
  }
}

void cmio_dust_run(const cmio_lattice *lat, const double box[6], const double *nH,
                   const double *xH, uint32_t num_photon, uint64_t seed, uint32_t instance,
                   uint32_t iteration, double albedo, const double source[3],
                   uint32_t source_subgrid, int32_t npix_x, int32_t npix_y, double *image,
                   cmio_dust_stats *st) {
  memset(st, 0, sizeof(*st));
  st->emitted = num_photon;
  const size_t npix = (size_t)npix_x * npix_y;
  for (size_t k = 0; k < npix; ++k) image[k] = 0.;
  const size_t cap = num_photon ? num_photon : 1;
  cmio_photon *cur = (cmio_photon *)malloc(sizeof(cmio_photon) * cap);
  uint32_t *sub = (uint32_t *)malloc(sizeof(uint32_t) * cap);
  uint32_t *id = (uint32_t *)malloc(sizeof(uint32_t) * cap);
  uint32_t *gen = (uint32_t *)malloc(sizeof(uint32_t) * cap);
  /* 1. TAU packets to the box edge, 2. relaunch */
  for (uint32_t i = 0; i < num_photon; ++i) {
    cmio_photon *ph = &cur[i];
    memset(ph, 0, sizeof(*ph));
    for (int a = 0; a < 3; ++a) ph->position[a] = source[a];
    dust_direction(seed, instance, iteration, i, 0u, 0u, ph->direction, NULL, NULL);
    ph->target_optical_depth = 0.;
    ph->cross_section = 1.;
    ph->weight = 1.;
    ph->type = 1; /* TAU */
    ph->reserved = 0;
    sub[i] = source_subgrid;
    id[i] = i;
    gen[i] = 0u;
    (void)dust_walk(lat, nH, xH, ph, &sub[i], 2, st);
    const double weight = 1. - cmio_dust_exp(-ph->target_optical_depth);
    uint32_t w[4];
    dust_words(seed, instance, iteration, i, 0u, 1u, 0u, w);
    for (int a = 0; a < 3; ++a) ph->position[a] = source[a];
    ph->weight = weight;
    ph->target_optical_depth = reemit_neg_log(1. - dust_uniform(w[0]) * weight);
    ph->type = 0; /* DIRECT */
    ph->reserved = 0;
    sub[i] = source_subgrid;
  }
  /* 3-4. walks and scatterings until no packet is left */
  uint32_t n = num_photon;
  for (uint32_t g = 0; g < 4096u && n > 0; ++g) {
    st->generations += 1;
    uint32_t m = 0;
    for (uint32_t i = 0; i < n; ++i) {
      cmio_photon ph = cur[i];
      uint32_t s = sub[i];
      if (dust_walk(lat, nH, xH, &ph, &s, 1, st) == 1) {
        st->escaped += 1;
        continue;
      }
      const uint32_t gg = gen[i] + 1u;
      double dir[3];
      uint32_t w0 = 0, w3 = 0;
      dust_direction(seed, instance, iteration, id[i], gg, 2u, dir, &w0, &w3);
      if (!(dust_uniform(w0) < albedo)) {
        st->absorbed += 1;
        continue;
      }
      st->scatterings += 1;
      for (int a = 0; a < 3; ++a) ph.direction[a] = dir[a];
      ph.target_optical_depth = reemit_neg_log(dust_uniform(w3));
      ph.weight = ph.weight * 0.25 * 0.318309886183790671538;
      ph.type = 0;
      ph.reserved = 0;
      /* peel-off copy along +z */
      cmio_photon e = ph;
      e.direction[0] = 0.;
      e.direction[1] = 0.;
      e.direction[2] = 1.;
      e.target_optical_depth = 0.;
      e.type = 2; /* PEELOFF */
      uint32_t es = s;
      if (dust_walk(lat, nH, xH, &e, &es, 2, st) == 1) {
        const double fx = ((e.position[0] - box[0]) / box[3]) * (double)npix_x;
        const double fy = ((e.position[1] - box[1]) / box[4]) * (double)npix_y;
        if (fx >= 0. && fx < (double)npix_x && fy >= 0. && fy < (double)npix_y) {
          image[(size_t)(int)fx * npix_y + (int)fy] +=
              e.weight * cmio_dust_exp(-e.target_optical_depth);
        } else {
          st->peeloffs_off_image += 1;
        }
      }
      /* scattered packets move to the front, in order */
      cur[m] = ph;
      sub[m] = s;
      id[m] = id[i];
      gen[m] = gg;
      ++m;
    }
    n = m;
  }
  for (size_t k = 0; k < npix; ++k) image[k] /= (double)num_photon;
  free(cur);
  free(sub);
  free(id);
  free(gen);
}
