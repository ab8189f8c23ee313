// Dust scattering with forced first scattering and peel-off images: the
// algorithm of the reference's dust driver (testDensitySubGrid_omp_dust.cpp),
// on the same grid, subgrids and FP64 walk as the photoionization path.
//
// One call follows N source packets (the driver's photon loop, :2307-2512):
//  1. TAU packets leave the source isotropically, weight 1, cross section 1
//     (fill_buffer with FORCED_SCATTERING, :564-620), and add up the optical
//     depth tau0 to the box edge (compute_optical_depth, DensitySubGrid.hpp:
//     1482-1604).
//  2. Relaunch (execute_relaunch_photon_task, :1200-1260): back at the source
//     with the same direction as DIRECT packets of weight W = 1 - exp(-tau0)
//     and target depth -ln(1 - u W), which always lies inside the box.
//  3. DIRECT packets walk to their target depth without tallies (propagate,
//     DensitySubGrid.hpp:1333-1472); packets that leave the box are lost.
//  4. An absorbed packet is scattered with probability `albedo` (the driver's
//     reemission_probability; do_reemission, :730-760): new isotropic
//     direction, target -ln u, weight W / (4 pi).  Every scattered packet also
//     sends a PEELOFF copy along +z with depth 0 (execute_photon_reemit_task,
//     :1484-1560); the copy adds its depth to the box edge and, once out, puts
//     weight * exp(-depth) into the image pixel under its exit point
//     (do_photon_traversal, :685-693).  Steps 3-4 repeat for the scattered
//     packets until none is left.
//
// One thread walks one packet from subgrid to subgrid (no tallies, so no
// subgrid-wise staging is needed); n_H and x_H are read from the FP64 field
// arrays.  Random draws are counter-based (Philox4x32-10 keyed by seed and
// instance, counter = packet, generation, iteration, purpose) and use
// correctly rounded operations only, so the oracle's host copy draws the same
// bits.
#pragma once

#include "cmi_walk.cuh"

namespace cmi {

enum DustPacketType : int32_t { kDustDirect = 0, kDustTau = 1, kDustPeeloff = 2 };
enum DustPurpose : uint32_t { kDustEmit = 0, kDustRelaunch = 1, kDustScatter = 2 };
enum DustStatus : int32_t { kDustIn = 0, kDustAbsorbed = 1, kDustEscaped = 2, kDustLost = 3 };
constexpr uint32_t kPhiloxDustTag = 0x44555354u;
// subgrid visits of one packet walk (a straight line crosses at most
// sum(num_subgrid) + 2 subgrids)
constexpr int kDustMaxVisits = 4096;

// exp(x) for x <= 0 with correctly rounded operations only: x = k ln2 + r
// (Cody-Waite: ln2 = L1 + L2 with k L1 exact for |k| < 2^11), exp(r) from its
// Taylor series to r^18 / 18! (|r| <= ln2 / 2: truncation below 2^-60), times
// 2^k.  Results below e^-700 are 0.
__host__ __device__ inline double dust_exp(double x) {
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

__host__ __device__ inline double dust_uniform(uint32_t w) {
  return ((double)w + 0.5) * (1.0 / 4294967296.0);
}

// -ln(u), u in (0, 1]: u = m 2^e with m in [sqrt(1/2), sqrt(2)), ln m =
// 2 atanh((m - 1) / (m + 1)) by its series
__host__ __device__ inline double dust_neg_log(double u) {
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

__host__ __device__ inline void dust_words(uint64_t seed, uint32_t instance, uint32_t iteration,
                                           uint32_t id, uint32_t gen, uint32_t purpose,
                                           uint32_t attempt, uint32_t w[4]) {
  const uint32_t ctr[4] = {id, gen, iteration, kPhiloxDustTag + (purpose << 8) + attempt};
  philox4x32_10(ctr, (uint32_t)seed, (uint32_t)(seed >> 32) + instance, w);
}

// isotropic direction (Marsaglia: a point of the unit disc by rejection from
// the square, attempt k on its own counter); w0 = the first attempt's first
// word, w3 = the accepted attempt's fourth word.  16 rejections in a row
// (probability 0.21^16) give +z.
__host__ __device__ inline void dust_direction(uint64_t seed, uint32_t instance,
                                               uint32_t iteration, uint32_t id, uint32_t gen,
                                               uint32_t purpose, double dir[3], uint32_t *w0,
                                               uint32_t *w3) {
  for (uint32_t k = 0; k < 16u; ++k) {
    uint32_t w[4];
    dust_words(seed, instance, iteration, id, gen, purpose, k, w);
    if (k == 0u && w0) *w0 = w[0];
    const double x1 = 2. * dust_uniform(w[1]) - 1.;
    const double x2 = 2. * dust_uniform(w[2]) - 1.;
    const double s = x1 * x1 + x2 * x2;
    if (s < 1.) {
      const double f = 2. * sqrt(1. - s);
      dir[0] = x1 * f;
      dir[1] = x2 * f;
      dir[2] = 1. - 2. * s;
      if (w3) *w3 = w[3];
      return;
    }
  }
  dir[0] = 0.;
  dir[1] = 0.;
  dir[2] = 1.;
  if (w3) *w3 = 0x80000000u;
}

struct DustParams {
  const DevSubgrid *subs;
  const double *nH, *xH;
  DirectionTables tables;
  Packet64 *pk;       // packets of the current pass
  uint32_t *sub;      // subgrid each packet is in (or left the box from)
  uint32_t *id;       // source packet it descends from
  uint32_t *gen;      // scatterings so far
  int32_t *status;    // DustStatus after a walk
  const uint32_t *count;  // packets in pk (device)
  uint64_t seed;
  uint32_t instance, iteration;
  double src[3];
  uint32_t src_sub;
  unsigned long long *counters;  // [crossings, transits, walk-bound hits]
};

__device__ __forceinline__ unsigned long long warp_sum64(unsigned long long v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
  return v;
}

// 1. source packets: TAU type, weight 1, cross section 1, depth 0
__global__ void k_dust_emit(DustParams p, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    Packet64 q;
    for (int a = 0; a < 3; ++a) q.pos[a] = p.src[a];
    dust_direction(p.seed, p.instance, p.iteration, i, 0u, kDustEmit, q.dir, nullptr, nullptr);
    q.tau = 0.;
    q.sigma = 1.;
    q.weight = 1.;
    q.type = kDustTau;
    q.meta = 0u;  // TRAVELDIRECTION_INSIDE
    p.pk[i] = q;
    p.sub[i] = p.src_sub;
    p.id[i] = i;
    p.gen[i] = 0u;
  }
}

// walk of every packet to absorption or out of the box (kMode: kPropagate for
// DIRECT packets, kDepth for TAU and PEELOFF packets)
template <int kMode>
__global__ void __launch_bounds__(128) k_dust_walk(DustParams p) {
  const uint32_t n = *p.count;
  unsigned long long cross = 0, trans = 0, bound_hits = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    Packet64 q = p.pk[i];
    uint32_t s = p.sub[i];
    int32_t result = kDustLost;
    for (int visit = 0; visit < kDustMaxVisits; ++visit) {
      const DevSubgrid &S = p.subs[s];
      View64 v;
      v.nH = p.nH + S.field_offset;
      v.xH = p.xH + S.field_offset;
      v.J = nullptr;
      for (int a = 0; a < 3; ++a) {
        v.n[a] = S.ncell[a];
        v.anchor[a] = S.anchor[a];
        v.cs[a] = S.cell_size[a];
        v.inv_cs[a] = S.inv_cell_size[a];
      }
      v.nyz = S.ncell[1] * S.ncell[2];
      Walk64 w;
      int st = (kMode == kDepth) ? w.begin_depth(q, v, p.tables.sign_code)
                                 : w.begin(q, v, p.tables.sign_code);
      const int limit = S.ncell[0] + S.ncell[1] + S.ncell[2] + 3;
      while (st == kRun && w.steps <= limit) st = w.step<kMode>(v);
      cross += (unsigned long long)w.steps;
      ++trans;
      if (st == kRun) {  // no straight line takes this many steps
        ++bound_hits;
        break;
      }
      if (st == kAbsorbed) {
        q = w.packet(v, 0u);
        result = kDustAbsorbed;
        break;
      }
      const int od = p.tables.mask_dir[w.exit_mask(v)];
      if (od >= kNumDirections) {
        ++bound_hits;
        break;
      }
      Packet64 r = w.packet(v, p.tables.mirror[od]);
      if (kMode == kDepth) r.tau = w.tau_target + w.tau_done;
      q = r;
      const uint32_t ngb = S.ngb[od];
      if (ngb == kOutside) {
        result = kDustEscaped;
        break;
      }
      s = ngb;
    }
    p.pk[i] = q;
    p.sub[i] = s;
    p.status[i] = result;
  }
  // one atomic per warp and counter (every lane of the warp gets here)
  const unsigned long long wc = warp_sum64(cross), wt = warp_sum64(trans),
                           wb = warp_sum64(bound_hits);
  if ((threadIdx.x & 31) == 0) {
    if (wc) atomicAdd(&p.counters[0], wc);
    if (wt) atomicAdd(&p.counters[1], wt);
    if (wb) atomicAdd(&p.counters[2], wb);
  }
}

// 2. relaunch of the TAU packets as DIRECT packets with forced scattering
__global__ void k_dust_relaunch(DustParams p) {
  const uint32_t n = *p.count;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    Packet64 q = p.pk[i];
    const double weight = 1. - dust_exp(-q.tau);
    uint32_t w[4];
    dust_words(p.seed, p.instance, p.iteration, p.id[i], 0u, kDustRelaunch, 0u, w);
    for (int a = 0; a < 3; ++a) q.pos[a] = p.src[a];
    q.weight = weight;
    q.tau = dust_neg_log(1. - dust_uniform(w[0]) * weight);
    q.type = kDustDirect;
    q.meta = 0u;
    p.pk[i] = q;
    p.sub[i] = p.src_sub;
  }
}

struct DustScatterParams {
  const Packet64 *pk;
  const uint32_t *sub, *id, *gen;
  const int32_t *status;
  const uint32_t *count;
  Packet64 *out_pk, *peel_pk;
  uint32_t *out_sub, *out_id, *out_gen, *peel_sub;
  uint32_t *out_count;   // scattered packets written (also the peel-off count)
  uint64_t seed;
  uint32_t instance, iteration;
  double albedo;
  unsigned long long *counters;  // [3] absorbed for good, [4] escaped, [5] scattered
};

// 4. scattering of the absorbed packets, with their peel-off copies
__global__ void k_dust_scatter(DustScatterParams p) {
  const uint32_t n = *p.count;
  const int lane = threadIdx.x & 31;
  for (uint32_t b = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); b < n;
       b += gridDim.x * blockDim.x) {
    const uint32_t i = b + (uint32_t)lane;
    bool scatter = false, escaped = false, dropped = false;
    Packet64 q{};
    uint32_t g = 0;
    if (i < n) {
      const int32_t st = p.status[i];
      escaped = st == kDustEscaped;
      if (st == kDustAbsorbed) {
        q = p.pk[i];
        g = p.gen[i] + 1u;
        double dir[3];
        uint32_t w0 = 0, w3 = 0;
        dust_direction(p.seed, p.instance, p.iteration, p.id[i], g, kDustScatter, dir, &w0,
                       &w3);
        if (dust_uniform(w0) < p.albedo) {
          scatter = true;
          for (int a = 0; a < 3; ++a) q.dir[a] = dir[a];
          q.tau = dust_neg_log(dust_uniform(w3));
          q.weight = q.weight * 0.25 * 0.318309886183790671538;  // 1 / (4 pi)
          q.type = kDustDirect;
          q.meta = 0u;
        } else {
          dropped = true;
        }
      }
    }
    const unsigned me = __ballot_sync(0xFFFFFFFFu, escaped);
    const unsigned md = __ballot_sync(0xFFFFFFFFu, dropped);
    if (lane == 0) {
      if (me) atomicAdd(&p.counters[4], (unsigned long long)__popc(me));
      if (md) atomicAdd(&p.counters[3], (unsigned long long)__popc(md));
    }
    const unsigned m = __ballot_sync(0xFFFFFFFFu, scatter);
    const int leader = m ? __ffs(m) - 1 : 0;
    uint32_t base = 0;
    if (m && lane == leader) base = atomicAdd(p.out_count, (uint32_t)__popc(m));
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
    if (scatter) {
      const uint32_t o = base + (uint32_t)__popc(m & ((1u << lane) - 1u));
      p.out_pk[o] = q;
      p.out_sub[o] = p.sub[i];
      p.out_id[o] = p.id[i];
      p.out_gen[o] = g;
      Packet64 e = q;
      e.dir[0] = 0.;
      e.dir[1] = 0.;
      e.dir[2] = 1.;
      e.tau = 0.;
      e.type = kDustPeeloff;
      p.peel_pk[o] = e;
      p.peel_sub[o] = p.sub[i];
    }
    if (m && lane == leader) atomicAdd(&p.counters[5], (unsigned long long)__popc(m));
  }
}

// peel-off packets that left the box: weight * exp(-depth) into the pixel
// under the exit point (x over npx columns, y over npy rows of the box face)
__global__ void k_dust_image(const Packet64 *pk, const int32_t *status, const uint32_t *count,
                             double x0, double wx, double y0, double wy, int npx, int npy,
                             double *image, unsigned long long *outside) {
  const uint32_t n = *count;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (status[i] != kDustEscaped) continue;
    const Packet64 q = pk[i];
    const double fx = ((q.pos[0] - x0) / wx) * (double)npx;
    const double fy = ((q.pos[1] - y0) / wy) * (double)npy;
    if (!(fx >= 0. && fx < (double)npx && fy >= 0. && fy < (double)npy)) {
      atomicAdd(outside, 1ull);
      continue;
    }
    const int ix = (int)fx, iy = (int)fy;
    atomicAdd(&image[(size_t)ix * npy + iy], q.weight * dust_exp(-q.tau));
  }
}

// DensitySubGrid::propagate / compute_optical_depth of single photons through
// one subgrid (the per-buffer calls of the dust driver's do_photon_traversal,
// :646-652): out_dir = the TravelDirection the photon leaves by (INSIDE: it
// reached its target depth), -1 if the walk bound was hit.
template <int kMode>
__global__ void __launch_bounds__(128) k_walk_photons(const DevSubgrid *subs, uint32_t sub,
                                                       const double *nH, const double *xH,
                                                       DirectionTables tables, Packet64 *pk,
                                                       const int32_t *in_dir, uint32_t n,
                                                       int32_t *out_dir) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const DevSubgrid &S = subs[sub];
  View64 v;
  v.nH = nH + S.field_offset;
  v.xH = xH + S.field_offset;
  v.J = nullptr;
  for (int a = 0; a < 3; ++a) {
    v.n[a] = S.ncell[a];
    v.anchor[a] = S.anchor[a];
    v.cs[a] = S.cell_size[a];
    v.inv_cs[a] = S.inv_cell_size[a];
  }
  v.nyz = S.ncell[1] * S.ncell[2];
  Packet64 q = pk[i];
  const uint32_t meta0 = q.meta;
  q.meta = (uint32_t)in_dir[i];
  Walk64 w;
  int st = (kMode == kDepth) ? w.begin_depth(q, v, tables.sign_code)
                             : w.begin(q, v, tables.sign_code);
  const int limit = S.ncell[0] + S.ncell[1] + S.ncell[2] + 3;
  while (st == kRun && w.steps <= limit) st = w.step<kMode>(v);
  int32_t res = -1;
  if (st == kAbsorbed) {
    res = 0;  // TRAVELDIRECTION_INSIDE
  } else if (st == kExited) {
    const int od = tables.mask_dir[w.exit_mask(v)];
    res = od < kNumDirections ? od : -1;
  }
  Packet64 r = w.packet(v, meta0);
  if (kMode == kDepth) r.tau = w.tau_target + w.tau_done;
  pk[i] = r;
  out_dir[i] = res;
}

}  // namespace cmi
