// Kernels of the B200 transport engine.
//
// One iteration of the plain method (testDensitySubGrid_omp.cpp:2213-2434)
// runs as a wavefront over all instances of a context:
//
//   emission plan -> emit -> [plan -> scatter -> walk] x R -> balance
//
// * emit / walk append packets to an unsorted arena, warp-aggregated: one
//   atomic per warp for the arena slot and one per group of lanes heading to
//   the same subgrid for the rank inside that subgrid's bucket (the 27
//   TravelDirection output buffers of a subgrid, do_photon_traversal's
//   output_buffers, land in the buckets of its 26 neighbours);
// * plan turns the per-subgrid counts into bucket offsets and chunks of at
//   most `chunk` packets; scatter moves every packet to its bucket;
// * walk: persistent CTAs claim chunks; a CTA owns the chunk's subgrid, whose
//   fields are staged in shared memory by a TMA bulk copy; warps trace their
//   packets one crossing per loop trip, refilling idle lanes; path lengths
//   are tallied in shared-memory atomics and flushed to the FP64 J array in
//   HBM once per subgrid residency.
// R = max over instances of (sum of subgrids per axis - 2), the most subgrid
// transits a straight ray can make, so no packet is left over.
#pragma once

#include "cmi_device.cuh"
#include "cmi_walk.cuh"

namespace cmi {

constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kNone = 0xffffffffu;
constexpr int kDrop = 3;
constexpr uint32_t kFlagArenaOverflow = 1u;
constexpr uint32_t kFlagStageTimeout = 2u;
constexpr uint32_t kFlagWalkLimit = 4u;
constexpr uint32_t kFlagLeftover = 8u;
constexpr uint32_t kFlagBadInput = 16u;
constexpr int kPlanThreads = 1024;
constexpr int kPlanPerThread = 4;
constexpr int kPlanTile = kPlanThreads * kPlanPerThread;
constexpr unsigned long long kStageWaitNs = 1000000000ull;  // 1 s

// ---------------------------------------------------------------------------
// packet load/store as 16-byte vectors
// ---------------------------------------------------------------------------
template <class P>
__device__ __forceinline__ P load_packet(const P *src) {
  static_assert(sizeof(P) % 16 == 0, "packet size");
  P out;
  const uint4 *s = reinterpret_cast<const uint4 *>(src);
  uint4 *d = reinterpret_cast<uint4 *>(&out);
#pragma unroll
  for (int i = 0; i < (int)(sizeof(P) / 16); ++i) d[i] = __ldg(s + i);
  return out;
}

template <class P>
__device__ __forceinline__ void store_packet(P *dst, const P &v) {
  const uint4 *s = reinterpret_cast<const uint4 *>(&v);
  uint4 *d = reinterpret_cast<uint4 *>(dst);
#pragma unroll
  for (int i = 0; i < (int)(sizeof(P) / 16); ++i) d[i] = s[i];
}

// ---------------------------------------------------------------------------
// Warp-aggregated append of the lanes with `append` set to the arena.  Must
// be called by all 32 lanes.  key = destination subgrid (global index).
// ---------------------------------------------------------------------------
template <class P>
__device__ __forceinline__ void warp_append(bool append, uint32_t key, const P &rec, P *arena,
                                            uint32_t *keys, uint32_t *ranks, uint32_t *hist,
                                            RoundState *st, uint32_t capacity) {
  const unsigned am = __ballot_sync(kFull, append);
  if (am == 0u) return;
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  const int leader = __ffs(am) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(&st->arena_count, (uint32_t)__popc(am));
  base = __shfl_sync(kFull, base, leader);
  if (append) {
    const unsigned peers = __match_any_sync(am, key);
    const int pl = __ffs(peers) - 1;
    uint32_t kb = 0;
    if (lane == pl) kb = atomicAdd(&hist[key], (uint32_t)__popc(peers));
    kb = __shfl_sync(peers, kb, pl);
    const uint32_t slot = base + (uint32_t)__popc(am & lt);
    if (slot < capacity) {
      store_packet(arena + slot, rec);
      keys[slot] = key;
      ranks[slot] = kb + (uint32_t)__popc(peers & lt);
    } else {
      atomicOr(&st->flags, kFlagArenaOverflow);
    }
  }
}

// block-wide exclusive scan of one uint32 per thread (blockDim multiple of 32)
template <int kThreads>
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t *warp_sums,
                                                         uint32_t &total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = (lane < kThreads / 32) ? warp_sums[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(kFull, w, o);
      if (lane >= o) w += y;
    }
    if (lane < kThreads / 32) warp_sums[lane] = w;
  }
  __syncthreads();
  total = warp_sums[kThreads / 32 - 1];
  const uint32_t before = (warp > 0) ? warp_sums[warp - 1] : 0u;
  __syncthreads();
  return before + x - v;
}

// ---------------------------------------------------------------------------
// iteration bookkeeping
// ---------------------------------------------------------------------------
__global__ void k_begin_iteration(RoundState *st, DevStats *stats, int ninst) {
  for (int i = threadIdx.x; i < ninst; i += blockDim.x) {
    DevStats z = {};
    stats[i] = z;
  }
  if (threadIdx.x == 0) {
    st->rounds_active = 0;
    st->round_index = 0;
    st->arena_count = 0;
    st->num_chunks = 0;
    st->chunk_next = 0;
    st->total_in = 0;
  }
}

__global__ void k_end_iteration(RoundState *st, DevStats *stats, int ninst, int advance) {
  const uint32_t leftover = st->total_in ? kFlagLeftover : 0u;
  for (int i = threadIdx.x; i < ninst; i += blockDim.x) {
    stats[i].flags |= st->flags | leftover;
    stats[i].rounds = st->rounds_active;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    st->flags |= leftover;
    if (advance) st->iteration += 1;
  }
}

// Condition of the graph's round loop: another walk when the last plan left
// packets and fewer than max_rounds walks ran (a packet still in flight after
// that is reported as left over by k_end_iteration).
__global__ void k_round_gate(RoundState *st, cudaGraphConditionalHandle h, uint32_t max_rounds) {
  if (threadIdx.x == 0) {
    const bool more = st->num_chunks > 0u && st->round_index < max_rounds;
    if (more) st->round_index += 1u;
    cudaGraphSetConditional(h, more ? 1u : 0u);
  }
}

// Packets per source of every instance for this iteration: the reference split
// (testDensitySubGrid_omp.cpp:2199-2208) with the remainder given to the
// sources holding the smallest Philox draws (stand-in for distribute(),
// :1650-1677).  One block.
// With src_rank0 (direct emission) it also counts every source's packets into
// the bucket histogram of its subgrid and records where in that bucket the
// source's packets start, so the emitted packets can be written in sorted
// order (k_emit_philox_direct) without appends or a scatter.
__global__ void k_emission_plan(const DevInstance *inst, int ninst, const DevSource *src,
                                int nsrc_total, RoundState *st, uint64_t *src_count,
                                uint64_t *src_first, uint64_t *buf_first, DevStats *stats,
                                uint32_t *src_rank0, uint32_t *hist) {
  const uint64_t seed = st->seed;
  const uint32_t it = st->iteration;
  for (int i = threadIdx.x; i < ninst; i += blockDim.x) {
    DevInstance I = inst[i];
    if (I.frozen) I.num_photon = 0;
    double total = 0.;
    for (uint32_t k = 0; k < I.num_sources; ++k) total += src[I.first_source + k].luminosity;
    uint64_t assigned = 0;
    for (uint32_t k = 0; k < I.num_sources; ++k) {
      const uint64_t n =
          (uint64_t)(src[I.first_source + k].luminosity / total * (double)I.num_photon);
      src_count[I.first_source + k] = n;
      assigned += n;
    }
    uint64_t rem = (I.num_photon > assigned) ? I.num_photon - assigned : 0;
    // rem < num_sources: pick the rem smallest draws, lower index on ties
    uint32_t taken_lo = 0, taken_hi = 0;  // bitmask over <= 64 sources
    while (rem > 0 && I.num_sources > 0) {
      int best = -1;
      uint32_t best_w = 0;
      for (uint32_t k = 0; k < I.num_sources && k < 64; ++k) {
        const bool taken = (k < 32) ? ((taken_lo >> k) & 1u) : ((taken_hi >> (k - 32)) & 1u);
        if (taken) continue;
        const uint32_t ctr[4] = {k, 0u, it, kPhiloxSplitTag};
        uint32_t w[4];
        philox4x32_10(ctr, (uint32_t)seed, (uint32_t)(seed >> 32) + (uint32_t)i, w);
        if (best < 0 || w[0] < best_w) {
          best = (int)k;
          best_w = w[0];
        }
      }
      if (best < 0) break;
      src_count[I.first_source + best] += 1;
      if (best < 32) taken_lo |= 1u << best; else taken_hi |= 1u << (best - 32);
      --rem;
    }
    stats[i].emitted = I.num_photon;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t acc = 0, bacc = 0;
    for (int s = 0; s < nsrc_total; ++s) {
      src_first[s] = acc;
      buf_first[s] = bacc;
      acc += src_count[s];
      bacc += (src_count[s] + 199) / 200;
    }
    src_first[nsrc_total] = acc;
    buf_first[nsrc_total] = bacc;
    st->emit_total = (uint32_t)acc;
    st->arena_count = 0;
    if (src_rank0) {  // sources in order: ranks inside each subgrid's bucket
      for (int s = 0; s < nsrc_total; ++s) {
        const uint32_t sub = src[s].subgrid;
        src_rank0[s] = hist[sub];
        hist[sub] += (uint32_t)src_count[s];
      }
    }
  }
}

// index s with first[s] <= g < first[s + 1] (first has n + 1 entries)
__device__ __forceinline__ int find_bin(const uint64_t *first, int n, uint64_t g) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (first[mid] <= g) lo = mid; else hi = mid - 1;
  }
  return lo;
}

struct EmitParams {
  const DevInstance *inst;
  const DevSource *src;
  int nsrc_total;
  const uint64_t *src_count, *src_first, *buf_first;
  const uint32_t *src_rank0, *bucket_off;  // direct emission
  void *arena_sorted;                      // direct emission: the walk's input arena
  RoundState *st;
  void *arena;
  uint32_t *keys, *ranks, *hist;
  uint32_t capacity;
  // export (cmi_emit_photons): every packet as a reference Photon at its
  // index in the iteration (source after source, packet order within one)
  Packet64 *photons_out;
};

// A packet leaving source S (testDensitySubGrid_omp.cpp:580-592) in the
// record of the transport: FP32 (cell units relative to the source's
// subgrid), mixed (absolute FP64 position, FP32 optical depth) or FP64.
__device__ __forceinline__ void make_emitted(const DevSource &S, const DevInstance &,
                                             const double dir[3], double tau, Packet32 &p) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    p.pos[a] = S.pos_cell[a];
    p.dir[a] = (float)dir[a];
  }
  p.tau = (float)tau;
  p.meta = (uint32_t)kInside;
}
__device__ __forceinline__ void make_emitted(const DevSource &S, const DevInstance &,
                                             const double dir[3], double tau, PacketM &p) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    p.pos[a] = S.position[a];
    p.dir[a] = dir[a];
  }
  p.tau = tau32(tau);
  p.meta = (uint32_t)kInside;
  p.pad[0] = p.pad[1] = 0u;
}
__device__ __forceinline__ void make_emitted(const DevSource &S, const DevInstance &I,
                                             const double dir[3], double tau, Packet64 &p) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    p.pos[a] = S.position[a];
    p.dir[a] = dir[a];
  }
  p.tau = tau;
  p.sigma = I.sigma;
  p.weight = 1.;
  p.type = 0;
  p.meta = (uint32_t)kInside;
}

// Philox emission straight into the sorted arena.  Packet g of the iteration
// belongs to source s (src_first) and has id g - first packet of its instance
// in the instance's Philox stream; it goes to bucket_off[subgrid of s] +
// src_rank0[s] + (g - src_first[s]) (the plan ran on the histogram
// k_emission_plan filled), so no append atomics and no scatter are needed.
// kExport: write the photons to prm.photons_out (index g) instead.
template <int K, bool kExport = false>
__global__ void __launch_bounds__(256) k_emit_philox_direct(EmitParams prm) {
  using Pk = typename PacketOf<K>::type;
  const RoundState *st = prm.st;
  const uint64_t N = st->emit_total;
  const uint64_t seed = st->seed;
  const uint32_t it = st->iteration;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < N; g += stride) {
    const int s = find_bin(prm.src_first, prm.nsrc_total + 1, g);
    const DevSource S = prm.src[s];
    const DevInstance I = prm.inst[S.instance];
    const uint64_t id = g - prm.src_first[I.first_source];
    double dir[3], tau;
    philox_packet(seed, S.instance, it, id, dir, tau);
    if (kExport) {
      Packet64 ph{};
      make_emitted(S, I, dir, tau, ph);
      ph.meta = 0u;
      prm.photons_out[g] = ph;
      continue;
    }
    Pk pk{};
    make_emitted(S, I, dir, tau, pk);
    const uint64_t dst = (uint64_t)prm.bucket_off[S.subgrid] + prm.src_rank0[s] +
                         (g - prm.src_first[s]);
    if (dst >= prm.capacity) {
      atomicOr(&prm.st->flags, kFlagArenaOverflow);
      continue;
    }
    store_packet((Pk *)prm.arena_sorted + dst, pk);
  }
}

// Emission replaying the reference generator: buffer b of 200 packets (global
// order over sources) draws from ranlxd(seed + b + iteration * buffers), one
// draw for the subgrid-copy pick (Source.hpp:94-99), then per packet cos(theta),
// phi and the optical depth (testDensitySubGrid_omp.cpp:529-597), with
// correctly rounded sin, cos and log.  kExport: write the photons to
// prm.photons_out at their index in the iteration instead of appending.
template <int K, bool kExport = false>
__global__ void __launch_bounds__(128) k_emit_ranlux(EmitParams prm) {
  using Pk = typename PacketOf<K>::type;
  const RoundState *st = prm.st;
  const uint64_t nbuf = prm.buf_first[prm.nsrc_total];
  const uint64_t seed = st->seed;
  const uint32_t it = st->iteration;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < nbuf; base += stride) {
    const uint64_t b = base + threadIdx.x;
    const bool valid = b < nbuf;
    Ranlux rng;
    int s = 0;
    uint32_t n_b = 0;
    if (valid) {
      s = find_bin(prm.buf_first, prm.nsrc_total + 1, b);
      const uint64_t k0 = (b - prm.buf_first[s]) * 200u;
      const uint64_t cnt = prm.src_count[s];
      n_b = (uint32_t)min((uint64_t)200u, cnt - k0);
      rng.seed((int32_t)(int64_t)(seed + b + (uint64_t)it * nbuf));
      (void)rng.uniform();
    }
    const DevSource S = prm.src[valid ? s : 0];
    const DevInstance I = prm.inst[S.instance];
    for (uint32_t k = 0; k < 200u; ++k) {
      const bool live = valid && k < n_b;
      Pk pk{};
      if (live) {
        const double cost = 2. * rng.uniform() - 1.;
        const double phi = 2. * 3.14159265358979323846 * rng.uniform();
        const double s2 = 1. - cost * cost;
        const double sint = sqrt((s2 < 0.) ? 0. : s2);
        double sinp, cosp;
        cr_sincos(phi, &sinp, &cosp);
        const double dir[3] = {sint * cosp, sint * sinp, cost};
        const double tau = cr_neg_log(rng.uniform());
        if (kExport) {
          Packet64 ph{};
          make_emitted(S, I, dir, tau, ph);
          ph.meta = 0u;
          prm.photons_out[prm.src_first[s] + (b - prm.buf_first[s]) * 200u + k] = ph;
        } else {
          make_emitted(S, I, dir, tau, pk);
        }
      }
      if (kExport) {
        if (!__any_sync(kFull, live)) break;
        continue;
      }
      if (!__any_sync(kFull, live)) break;
      warp_append(live, S.subgrid, pk, (Pk *)prm.arena, prm.keys, prm.ranks, prm.hist, prm.st,
                  prm.capacity);
    }
  }
}

// Caller-supplied packets (cmi_transport_packets): FP64 photon records with
// their start subgrid, converted to the transport precision and appended.
struct UploadParams {
  const Packet64 *photons;
  const uint32_t *start;  // subgrid index inside the instance
  uint64_t n;
  const DevSubgrid *subs;
  uint32_t first_sub, nsub;
  RoundState *st;
  void *arena;
  uint32_t *keys, *ranks, *hist;
  uint32_t capacity;
};

template <int K>
__global__ void __launch_bounds__(256) k_upload(UploadParams prm) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < prm.n; base += stride) {
    const uint64_t g = base + threadIdx.x;
    bool valid = g < prm.n;
    uint32_t key = 0;
    Packet32 p32{};
    Packet64 p64{};
    PacketM pm{};
    if (valid) {
      const uint32_t ls = prm.start[g];
      if (ls >= prm.nsub) {
        atomicOr(&prm.st->flags, kFlagBadInput);
        valid = false;
      } else {
        key = prm.first_sub + ls;
        p64 = prm.photons[g];
        p64.meta = (uint32_t)kInside;
        if (K == kPkM) {
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            pm.pos[a] = p64.pos[a];
            pm.dir[a] = p64.dir[a];
          }
          pm.tau = tau32(p64.tau);
          pm.meta = (uint32_t)kInside;
        } else if (K == kPk32) {
          const DevSubgrid &S = prm.subs[key];
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            p32.pos[a] = (float)((p64.pos[a] - S.anchor[a]) * S.inv_cell_size[a]);
            p32.dir[a] = (float)p64.dir[a];
          }
          p32.tau = (float)p64.tau;
          p32.meta = (uint32_t)kInside;
        }
      }
    }
    if (K == kPk32) {
      warp_append(valid, key, p32, (Packet32 *)prm.arena, prm.keys, prm.ranks, prm.hist,
                  prm.st, prm.capacity);
    } else if (K == kPkM) {
      warp_append(valid, key, pm, (PacketM *)prm.arena, prm.keys, prm.ranks, prm.hist,
                  prm.st, prm.capacity);
    } else {
      warp_append(valid, key, p64, (Packet64 *)prm.arena, prm.keys, prm.ranks, prm.hist,
                  prm.st, prm.capacity);
    }
  }
}

// ---------------------------------------------------------------------------
// plan: per-subgrid counts -> bucket offsets + chunk list
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kPlanThreads) k_plan_count(const uint32_t *hist, uint32_t S,
                                                             uint32_t chunk,
                                                             uint32_t *tile_pk,
                                                             uint32_t *tile_ch) {
  __shared__ uint32_t ws[32];
  const uint32_t s0 = blockIdx.x * kPlanTile + threadIdx.x * kPlanPerThread;
  uint32_t pk = 0, ch = 0;
#pragma unroll
  for (int k = 0; k < kPlanPerThread; ++k) {
    const uint32_t s = s0 + k;
    const uint32_t c = (s < S) ? hist[s] : 0u;
    pk += c;
    ch += (c + chunk - 1) / chunk;
  }
  uint32_t tpk, tch;
  (void)block_exclusive_scan<kPlanThreads>(pk, ws, tpk);
  (void)block_exclusive_scan<kPlanThreads>(ch, ws, tch);
  if (threadIdx.x == 0) {
    tile_pk[blockIdx.x] = tpk;
    tile_ch[blockIdx.x] = tch;
  }
}

__global__ void __launch_bounds__(kPlanThreads) k_plan_offsets(uint32_t ntiles,
                                                               const uint32_t *tile_pk,
                                                               const uint32_t *tile_ch,
                                                               uint32_t *tile_pk_off,
                                                               uint32_t *tile_ch_off,
                                                               RoundState *st) {
  __shared__ uint32_t ws[32];
  uint32_t carry_pk = 0, carry_ch = 0;
  for (uint32_t b = 0; b < ntiles; b += kPlanThreads) {
    const uint32_t t = b + threadIdx.x;
    const uint32_t pk = (t < ntiles) ? tile_pk[t] : 0u;
    const uint32_t ch = (t < ntiles) ? tile_ch[t] : 0u;
    uint32_t tot_pk, tot_ch;
    const uint32_t opk = block_exclusive_scan<kPlanThreads>(pk, ws, tot_pk);
    const uint32_t och = block_exclusive_scan<kPlanThreads>(ch, ws, tot_ch);
    if (t < ntiles) {
      tile_pk_off[t] = carry_pk + opk;
      tile_ch_off[t] = carry_ch + och;
    }
    carry_pk += tot_pk;
    carry_ch += tot_ch;
  }
  if (threadIdx.x == 0) {
    st->total_in = carry_pk;
    st->num_chunks = carry_ch;
    st->chunk_next = 0;
    st->arena_count = 0;
    if (carry_pk > 0) st->rounds_active += 1;
  }
}

__global__ void __launch_bounds__(kPlanThreads) k_plan_write(uint32_t *hist, uint32_t S,
                                                             uint32_t chunk,
                                                             const uint32_t *tile_pk_off,
                                                             const uint32_t *tile_ch_off,
                                                             uint32_t *bucket_off,
                                                             Chunk *chunks) {
  __shared__ uint32_t ws[32];
  const uint32_t s0 = blockIdx.x * kPlanTile + threadIdx.x * kPlanPerThread;
  uint32_t c[kPlanPerThread];
  uint32_t pk = 0, ch = 0;
#pragma unroll
  for (int k = 0; k < kPlanPerThread; ++k) {
    const uint32_t s = s0 + k;
    c[k] = (s < S) ? hist[s] : 0u;
    pk += c[k];
    ch += (c[k] + chunk - 1) / chunk;
  }
  uint32_t tpk, tch;
  uint32_t opk = block_exclusive_scan<kPlanThreads>(pk, ws, tpk) + tile_pk_off[blockIdx.x];
  uint32_t och = block_exclusive_scan<kPlanThreads>(ch, ws, tch) + tile_ch_off[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kPlanPerThread; ++k) {
    const uint32_t s = s0 + k;
    if (s >= S) break;
    bucket_off[s] = opk;
    const uint32_t nch = (c[k] + chunk - 1) / chunk;
    for (uint32_t q = 0; q < nch; ++q) {
      Chunk cc;
      cc.subgrid = s;
      cc.begin = opk + q * chunk;
      cc.count = min(chunk, c[k] - q * chunk);
      cc.rem = nch - q;
      chunks[och++] = cc;
    }
    opk += c[k];
    hist[s] = 0u;
  }
}

// Whole plan in one block when every subgrid fits one tile (S <= 4096):
// counts -> bucket offsets -> chunk list, and the round-state update.
// The chunk q of subgrid lo (by binary search over the first chunk of each
// subgrid): begin, count and the chunks left in its subgrid.
__device__ __forceinline__ Chunk plan_chunk(const uint32_t *choff, const uint32_t *pkoff,
                                            uint32_t q, uint32_t chunk) {
  int lo = 0, hi = kPlanTile - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (choff[mid] <= q) lo = mid; else hi = mid - 1;
  }
  const uint32_t j = q - choff[lo];
  Chunk cc;
  cc.subgrid = (uint32_t)lo;
  cc.begin = pkoff[lo] + j * chunk;
  cc.count = min(chunk, (pkoff[lo + 1] - pkoff[lo]) - j * chunk);
  cc.rem = (choff[lo + 1] - choff[lo]) - j;
  return cc;
}

// Rounds with more chunks than this have their chunk list written by
// k_plan_chunks across the GPU instead of by the plan's single block (16 per
// thread cost about as much as the extra launch).
constexpr uint32_t kPlanChunksInBlock = 16384;

__global__ void __launch_bounds__(kPlanThreads) k_plan_fused(uint32_t *hist, uint32_t S,
                                                             uint32_t chunk,
                                                             uint32_t *bucket_off,
                                                             Chunk *chunks, RoundState *st,
                                                             uint32_t *choff_out,
                                                             uint32_t *pkoff_out) {
  __shared__ uint32_t ws[32];
  __shared__ uint32_t s_choff[kPlanTile + 1];  // first chunk of each subgrid
  __shared__ uint32_t s_pkoff[kPlanTile + 1];  // first packet of each subgrid
  const uint32_t s0 = threadIdx.x * kPlanPerThread;
  uint32_t c[kPlanPerThread];
  uint32_t pk = 0, ch = 0;
#pragma unroll
  for (int k = 0; k < kPlanPerThread; ++k) {
    const uint32_t s = s0 + k;
    c[k] = (s < S) ? hist[s] : 0u;
    pk += c[k];
    ch += (c[k] + chunk - 1) / chunk;
  }
  uint32_t tpk, tch;
  uint32_t opk = block_exclusive_scan<kPlanThreads>(pk, ws, tpk);
  uint32_t och = block_exclusive_scan<kPlanThreads>(ch, ws, tch);
#pragma unroll
  for (int k = 0; k < kPlanPerThread; ++k) {
    const uint32_t s = s0 + k;
    s_choff[s] = och;
    s_pkoff[s] = opk;
    if (s < S) {
      bucket_off[s] = opk;
      hist[s] = 0u;
    }
    opk += c[k];
    och += (c[k] + chunk - 1) / chunk;
  }
  if (threadIdx.x == 0) {
    s_choff[kPlanTile] = tch;
    s_pkoff[kPlanTile] = tpk;
  }
  __syncthreads();
  if (tch <= kPlanChunksInBlock) {
    // few chunks: every thread writes some
    for (uint32_t q = threadIdx.x; q < tch; q += kPlanThreads)
      chunks[q] = plan_chunk(s_choff, s_pkoff, q, chunk);
  } else {
    // many chunks: the offsets go to k_plan_chunks
    for (int i = threadIdx.x; i <= kPlanTile; i += kPlanThreads) {
      choff_out[i] = s_choff[i];
      pkoff_out[i] = s_pkoff[i];
    }
  }
  if (threadIdx.x == 0) {
    st->total_in = tpk;
    st->num_chunks = tch;
    st->chunk_next = 0;
    st->arena_count = 0;
    if (tpk > 0) st->rounds_active += 1;
  }
}

// Chunk list of a round with many chunks (after k_plan_fused), written by
// the whole GPU: each block copies the per-subgrid offsets to shared memory
// and writes chunks q in a grid-stride loop.
__global__ void __launch_bounds__(256) k_plan_chunks(const uint32_t *choff, const uint32_t *pkoff,
                                                     uint32_t chunk, Chunk *chunks,
                                                     const RoundState *st) {
  __shared__ uint32_t s_choff[kPlanTile + 1];
  __shared__ uint32_t s_pkoff[kPlanTile + 1];
  const uint32_t tch = st->num_chunks;
  if (tch <= kPlanChunksInBlock) return;  // written by k_plan_fused (whole block returns)
  for (int i = threadIdx.x; i <= kPlanTile; i += blockDim.x) {
    s_choff[i] = choff[i];
    s_pkoff[i] = pkoff[i];
  }
  __syncthreads();
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < tch; q += gridDim.x * blockDim.x)
    chunks[q] = plan_chunk(s_choff, s_pkoff, q, chunk);
}

// Scatter of the round's packets into their buckets.  Inside the captured
// round loop it also decides whether another round follows (gate: the plan
// before it has set num_chunks), which saves the loop a separate launch.
template <class P>
__global__ void __launch_bounds__(256) k_scatter(const P *out, const uint32_t *keys,
                                                 const uint32_t *ranks,
                                                 const uint32_t *bucket_off, P *in,
                                                 RoundState *st, uint32_t capacity,
                                                 bool gate, cudaGraphConditionalHandle h,
                                                 uint32_t max_rounds) {
  if (gate && blockIdx.x == 0 && threadIdx.x == 0) {
    const bool more = st->num_chunks > 0u && st->round_index < max_rounds;
    if (more) st->round_index += 1u;
    cudaGraphSetConditional(h, more ? 1u : 0u);
  }
  const uint32_t n = min(st->total_in, capacity);
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint32_t dst = bucket_off[keys[i]] + ranks[i];
    if (dst < capacity) store_packet(in + dst, load_packet(out + i));
  }
}

// ---------------------------------------------------------------------------
// walk: one wavefront round
// ---------------------------------------------------------------------------
struct WalkParams {
  uint32_t chunk;          // largest chunk (packets), FP32 packet-buffer size
  uint32_t max_run;        // most chunks claimed at once
  uint32_t refill;         // FP32 walk: lanes not walking before a warp routes + refills
  const DevSubgrid *subs;
  const DevInstance *inst;
  const Chunk *chunks;
  RoundState *st;
  DevStats *stats;
  const void *arena_in;
  void *arena_out;
  uint32_t *keys, *ranks, *hist;
  uint32_t capacity;
  int32_t max_padded;     // largest padded cell count of any subgrid
  int32_t max_faces;      // mixed walk: largest nx + ny + nz + 3 of any subgrid
  const float *kappa;     // FP32 mode
  const double *nH, *xH;  // FP64 mode
  double *J;
  DirectionTables tables;
};

struct WalkShared {
  DirectionTables tab;
  uint32_t ngb[kNumDirections];
  int32_t n[3];
  int32_t nyz;
  int32_t ncells;
  int32_t padded;
  float cs_f[3];
  double anchor[3], cs[3], inv_cs[3];
  int64_t field_offset;
  double sigma;
  double reemission;
  uint32_t instance;
  int32_t chunk_id;
  uint32_t chunk_sub, chunk_begin, chunk_count;
  uint32_t claim;
  alignas(8) unsigned long long mbar;
};

struct Walk32Shared {
  DirectionTables tab;
  uint32_t ngb[kNumDirections];
  int32_t n[3];
  int32_t nyz;
  int32_t ncells;
  int32_t padded;
  float cs_f[3];
  float inv_cs_f[3];
  float tally_scale;   // 2^22 / lref
  double tally_unit;   // lref / 2^22 (m)
  double anchor[3], cs[3], inv_cs[3];  // FP64 geometry (mixed-precision walk)
  int64_t field_offset;
  double sigma;
  double reemission;
  uint32_t instance;
  // current run of chunks and segment of equal subgrid
  uint32_t run_c0, run_c1;
  uint32_t seg_sub, seg_begin, seg_chunks, seg_n, seg_next;
  // packet ring: claims, per-slot copies, fills
  uint32_t claim;
  uint32_t loaded[2];
  uint32_t uses[2];
  uint32_t seg_use0[2];
  alignas(8) unsigned long long mbar_field;
  alignas(8) unsigned long long mbar_pk[2];
};

template <class Sh>
__device__ __forceinline__ void load_subgrid(Sh &sh, const WalkParams &prm, uint32_t sub) {
  const DevSubgrid &S = prm.subs[sub];
  for (int d = 0; d < kNumDirections; ++d) sh.ngb[d] = S.ngb[d];
  for (int a = 0; a < 3; ++a) {
    sh.n[a] = S.ncell[a];
    sh.cs_f[a] = S.cell_size_f[a];
    sh.anchor[a] = S.anchor[a];
    sh.cs[a] = S.cell_size[a];
    sh.inv_cs[a] = S.inv_cell_size[a];
  }
  sh.nyz = S.ncell[1] * S.ncell[2];
  sh.ncells = S.ncells;
  sh.padded = S.padded_cells;
  sh.field_offset = S.field_offset;
  sh.instance = S.instance;
  sh.sigma = prm.inst[S.instance].sigma;
  sh.reemission = prm.inst[S.instance].reemission;
}

__device__ __forceinline__ void load_subgrid32(Walk32Shared &sh, const DevSubgrid &S,
                                               const WalkParams &prm) {
  for (int d = 0; d < kNumDirections; ++d) sh.ngb[d] = S.ngb[d];
  float lref = 0.f;
  for (int a = 0; a < 3; ++a) {
    sh.n[a] = S.ncell[a];
    sh.cs_f[a] = S.cell_size_f[a];
    sh.inv_cs_f[a] = (float)S.inv_cell_size[a];
    sh.anchor[a] = S.anchor[a];
    sh.cs[a] = S.cell_size[a];
    sh.inv_cs[a] = S.inv_cell_size[a];
    lref = fmaxf(lref, S.cell_size_f[a]);
  }
  sh.tally_scale = 4194304.f / lref;
  sh.tally_unit = (double)lref / 4194304.0;
  sh.nyz = S.ncell[1] * S.ncell[2];
  sh.ncells = S.ncells;
  sh.padded = S.padded_cells;
  sh.field_offset = S.field_offset;
  sh.instance = S.instance;
  sh.sigma = prm.inst[S.instance].sigma;
  sh.reemission = prm.inst[S.instance].reemission;
}

// The walk's view of the subgrid staged in shared memory.
__device__ __forceinline__ void make_view(const Walk32Shared &sh, const float *kappa,
                                          View32 &v) {
  v.kappa = kappa;
  for (int a = 0; a < 3; ++a) {
    v.n[a] = sh.n[a];
    v.cs[a] = sh.cs_f[a];
    v.inv_cs[a] = sh.inv_cs_f[a];
  }
  v.nyz = sh.nyz;
}
__device__ __forceinline__ void make_view(const Walk32Shared &sh, const float *kappa,
                                          const double *faces, ViewM &v) {
  v.kappa = kappa;
  v.anchor = sh.anchor;
  v.cs = sh.cs;
  v.inv_cs = sh.inv_cs;
  v.faces = faces;
  for (int a = 0; a < 3; ++a) v.n[a] = sh.n[a];
  v.face_off[0] = 0;
  v.face_off[1] = sh.n[0] + 1;
  v.face_off[2] = sh.n[0] + sh.n[1] + 2;
  v.nyz = sh.nyz;
}
__device__ __forceinline__ void make_view(const Walk32Shared &sh, const float *kappa,
                                          const double *, View32 &v) {
  make_view(sh, kappa, v);
}

// per-thread counters -> instance statistics (one atomic per warp and counter)
__device__ __forceinline__ void flush_counters(DevStats *stats, uint32_t instance,
                                               uint32_t &c_cross, uint32_t &c_trans,
                                               uint32_t &c_abs, uint32_t &c_esc,
                                               uint32_t &c_reem) {
  const uint32_t wc = __reduce_add_sync(kFull, c_cross);
  const uint32_t wt = __reduce_add_sync(kFull, c_trans);
  const uint32_t wa = __reduce_add_sync(kFull, c_abs);
  const uint32_t we = __reduce_add_sync(kFull, c_esc);
  const uint32_t wr = __reduce_add_sync(kFull, c_reem);
  if ((threadIdx.x & 31) == 0) {
    DevStats &S = stats[instance];
    if (wc) atomicAdd(&S.crossings, (unsigned long long)wc);
    if (wt) atomicAdd(&S.transits, (unsigned long long)wt);
    if (wa) atomicAdd(&S.absorbed, (unsigned long long)wa);
    if (we) atomicAdd(&S.escaped, (unsigned long long)we);
    if (wr) atomicAdd(&S.reemitted, (unsigned long long)wr);
  }
  c_cross = c_trans = c_abs = c_esc = c_reem = 0;
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long *mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(mbar)), "r"(count)
               : "memory");
  // make the initialised barrier visible to the async (TMA) proxy
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long *mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(mbar)),
               "r"(bytes)
               : "memory");
}

// TMA bulk copy global -> this CTA's shared memory (no multicast); completion
// is signalled on mbar.  dst, src and bytes are multiples of 16.
__device__ __forceinline__ void tma_load_1d(void *dst, const void *src, uint32_t bytes,
                                            unsigned long long *mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(mbar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *mbar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(mbar)), "r"(phase)
      : "memory");
  return ok != 0u;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait (1 s) for a staging copy.  On timeout the flag is raised and a
// second bounded wait (1 s) lets the copy land before the CTA reuses or
// releases the buffer.
__device__ __forceinline__ void mbar_wait_bounded(unsigned long long *mbar, uint32_t phase,
                                                  uint32_t *flags) {
  if (mbar_try_wait(mbar, phase)) return;
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait(mbar, phase)) {
    if (global_ns() - t0 > kStageWaitNs) {
      atomicOr(flags, kFlagStageTimeout);
      const unsigned long long t1 = global_ns();
      while (!mbar_try_wait(mbar, phase) && global_ns() - t1 < kStageWaitNs) {
      }
      return;
    }
  }
}

// Bounded wait until the counter *p has passed `target` (a shared-memory
// count bumped by another warp).
__device__ __forceinline__ void wait_count_above(const uint32_t *p, uint32_t target,
                                                 uint32_t *flags) {
  if ((int32_t)(*(const volatile uint32_t *)p - target) > 0) return;
  const unsigned long long t0 = global_ns();
  while ((int32_t)(*(const volatile uint32_t *)p - target) <= 0) {
    if (global_ns() - t0 > kStageWaitNs) {
      atomicOr(flags, kFlagStageTimeout);
      return;
    }
  }
  __threadfence_block();
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// FP64 wavefront round: the reference walk, fields staged by TMA, packets
// read from the sorted arena, FP64 tallies in shared memory.
constexpr int kSteps64PerCheck = 16;
template <int kThreads>
__global__ void __launch_bounds__(kThreads) k_walk64(WalkParams prm) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WalkShared &sh = *reinterpret_cast<WalkShared *>(smem_raw);
  const size_t head = (sizeof(WalkShared) + 15) & ~(size_t)15;
  const int P = prm.max_padded;
  double *s_n = reinterpret_cast<double *>(smem_raw + head);
  double *s_x = s_n + P;
  double *s_J = s_x + P;

  RoundState *st = prm.st;
  const uint32_t nchunks = st->num_chunks;
  if (nchunks == 0u) return;
  const int tid = threadIdx.x;
  if (tid < (int)sizeof(DirectionTables) / 4) {
    reinterpret_cast<uint32_t *>(&sh.tab)[tid] =
        reinterpret_cast<const uint32_t *>(&prm.tables)[tid];
  }
  if (tid == 0) mbar_init(&sh.mbar, 1);
  for (int c = tid; c < P; c += kThreads) s_J[c] = 0.;
  __syncthreads();

  const int lane = tid & 31;
  const unsigned lt = (1u << lane) - 1u;
  uint32_t phase = 0;
  uint32_t staged = kNone;
  uint32_t c_cross = 0, c_trans = 0, c_abs = 0, c_esc = 0, c_reem = 0;
  const uint64_t rseed = st->seed;
  const uint32_t riter = st->iteration;

  auto flush = [&]() {
    const int64_t off = sh.field_offset;
    for (int c = tid; c < sh.ncells; c += kThreads) {
      const double v = s_J[c];
      if (v != 0.) atomicAdd(&prm.J[off + c], v);
      s_J[c] = 0.;
    }
    flush_counters(prm.stats, sh.instance, c_cross, c_trans, c_abs, c_esc, c_reem);
  };

  for (;;) {
    if (tid == 0) {
      const uint32_t c = atomicAdd(&st->chunk_next, 1u);
      if (c < nchunks) {
        const Chunk ch = prm.chunks[c];
        sh.chunk_id = (int32_t)c;
        sh.chunk_sub = ch.subgrid;
        sh.chunk_begin = ch.begin;
        sh.chunk_count = ch.count;
      } else {
        sh.chunk_id = -1;
      }
      sh.claim = 0;
    }
    __syncthreads();
    if (sh.chunk_id < 0) break;
    const uint32_t sub = sh.chunk_sub;
    if (sub != staged) {
      if (staged != kNone) flush();
      __syncthreads();
      if (tid == 0) {
        load_subgrid(sh, prm, sub);
        fence_proxy_async();
        const uint32_t bytes = (uint32_t)sh.padded * 8u;
        mbar_expect_tx(&sh.mbar, 2u * bytes);
        tma_load_1d(s_n, prm.nH + sh.field_offset, bytes, &sh.mbar);
        tma_load_1d(s_x, prm.xH + sh.field_offset, bytes, &sh.mbar);
      }
      mbar_wait_bounded(&sh.mbar, phase, &st->flags);
      phase ^= 1u;
      staged = sub;
      __syncthreads();
    }

    const uint32_t count = sh.chunk_count, begin = sh.chunk_begin;
    const int limit = sh.n[0] + sh.n[1] + sh.n[2] + 3;
    View64 v64;
    v64.nH = s_n;
    v64.xH = s_x;
    v64.J = s_J;
    for (int a = 0; a < 3; ++a) {
      v64.n[a] = sh.n[a];
      v64.anchor[a] = sh.anchor[a];
      v64.cs[a] = sh.cs[a];
      v64.inv_cs[a] = sh.inv_cs[a];
    }
    v64.nyz = sh.nyz;
    Walk64 w64;
    uint32_t wq_b = 0, wq_e = 0;
    bool exhausted = false, have = false, fresh = false;
    int entry = kRun;
    uint32_t rcount = 0;  // reemissions of the lane's packet in this visit
    for (;;) {
      const unsigned idle = __ballot_sync(kFull, !have);
      if (idle != 0u && !exhausted) {
        if (wq_b >= wq_e) {
          uint32_t base = 0;
          if (lane == 0) base = atomicAdd(&sh.claim, 32u);
          base = __shfl_sync(kFull, base, 0);
          if (base >= count) {
            exhausted = true;
          } else {
            wq_b = base;
            wq_e = min(base + 32u, count);
          }
        }
        if (wq_b < wq_e) {
          const uint32_t take = min((uint32_t)__popc(idle), wq_e - wq_b);
          const uint32_t r = (uint32_t)__popc(idle & lt);
          if (!have && r < take) {
            const Packet64 pk = load_packet(((const Packet64 *)prm.arena_in) + begin + wq_b + r);
            entry = w64.begin(pk, v64, sh.tab.sign_code);
            rcount = 0u;
            have = true;
            fresh = true;
          }
          wq_b += take;
        }
      }
      if (!__any_sync(kFull, have)) {
        if (exhausted) break;
        continue;
      }
      int status = kRun;
      if (have) {
        if (fresh) {
          status = entry;
          fresh = false;
        }
        if (status == kRun) {
          // up to kSteps64PerCheck crossings between two looks at the warp
          // (swept on B200, 128^3 log-normal: 1 -> 5.8e9, 8 -> 1.53e10,
          // 16 -> 1.64e10 crossings/s; the results are unchanged)
          status = w64.step(v64);
          ++c_cross;
#pragma unroll 1
          for (int u = 1; u < kSteps64PerCheck && status == kRun; ++u) {
            status = w64.step(v64);
            ++c_cross;
          }
          if (status == kRun && w64.steps > limit) status = kDrop;
        }
      }
      const bool fin = have && status != kRun;
      if (__any_sync(kFull, fin)) {
        uint32_t key = kOutside, meta = 0;
        bool append = false, reemitted = false;
        if (fin) {
          ++c_trans;
          if (status == kExited) {
            const int od = sh.tab.mask_dir[w64.exit_mask(v64)];
            if (od >= kNumDirections) {
              atomicOr(&st->flags, kFlagWalkLimit);
            } else {
              key = sh.ngb[od];
              meta = sh.tab.mirror[od];
              if (key == kOutside) ++c_esc; else append = true;
            }
          } else if (status == kAbsorbed) {
            // reemission from the absorption point (the photon as the
            // reference's next traversal task would receive it)
            Packet64 rp = w64.packet(v64, (uint32_t)kInside);
            double rd[4];
            if (sh.reemission > 0. &&
                reemit_draw_call(rseed, sh.instance, riter, reemit_hash(rp.pos[0]),
                                 reemit_hash(rp.pos[1]), reemit_hash(rp.pos[2]), rcount,
                                 sh.reemission, rd)) {
              ++c_reem;
              ++rcount;
              for (int a = 0; a < 3; ++a) rp.dir[a] = rd[a];
              rp.tau = rd[3];
              entry = w64.begin(rp, v64, sh.tab.sign_code);
              fresh = true;
              reemitted = true;
            } else {
              ++c_abs;
            }
          } else {
            atomicOr(&st->flags, kFlagWalkLimit);
          }
        }
        Packet64 rec{};
        if (append) rec = w64.packet(v64, meta);
        warp_append(append, key, rec, (Packet64 *)prm.arena_out, prm.keys, prm.ranks, prm.hist,
                    st, prm.capacity);
        if (fin && !reemitted) have = false;
      }
    }
    __syncthreads();
  }
  if (staged != kNone) flush();
}

// FP32 wavefront round.
//
// Work distribution: the plan's chunks (<= CH packets, sorted by subgrid) are
// claimed in runs of consecutive chunks (guided: shorter runs as the round
// drains).  A run splits into segments of equal subgrid; per segment the CTA
// stages the subgrid's kappa = sigma*n*x (TMA) unless it is already resident.
//
// Packet flow inside a segment: a two-slot shared-memory ring, each slot
// filled with one chunk by a TMA bulk copy from the sorted arena.  Warps claim
// exactly as many packets as they have idle lanes and copy them into
// registers; the warp whose copy completes a slot issues the TMA of the chunk
// after next into it.  Warps therefore flow across the chunks of a subgrid
// without block-wide barriers; one barrier per segment remains (tally flush
// and restaging happen there).
//
// Packets leaving the subgrid are staged per warp and appended 32 at a time
// (one 1 KB coalesced store, one arena atomic, one bucket atomic per
// destination).  Path lengths go to shared-memory tallies (Tally32), merged
// into FP64 J in HBM when the CTA leaves the subgrid.
// per-warp output staging: flushed when it holds >= kStageFlush packets, so
// it never holds more than kStageFlush - 1 + 32
constexpr int kStage = 48;
constexpr uint32_t kStageFlush = 16;
// crossings per lane between warp-level batch tests (swept on B200: 1 -> 7.5e10,
// 2 -> 8.3e10, 4 -> 8.7e10, 8 -> 9.0e10, 12 -> 8.4e10 crossings/s on the 128^3
// log-normal workload)
constexpr int kStepsPerCheck = 8;

// One wavefront round of the FP32 opacity walks: W = Walk32 (cell-unit FP32
// geometry, 32-byte packets) or WalkM (the reference's FP64 geometry, 64-byte
// packets).  kReemit: the build with reemission (any instance with p > 0);
// without it the absorbed-packet path carries no reemission code.
template <class W, int kThreads, int kTally, bool kReemit>
__device__ __forceinline__ void walk_round(const WalkParams &prm) {
  using Pk = typename WalkTraits<W>::Packet;
  using View = typename WalkTraits<W>::View;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Walk32Shared &sh = *reinterpret_cast<Walk32Shared *>(smem_raw);
  constexpr int kWarps = kThreads / 32;
  const int P = prm.max_padded;
  const uint32_t CH = prm.chunk;
  const uint32_t ch_shift = (uint32_t)(__ffs(CH) - 1);  // CH is a power of two
  unsigned char *cur_ptr = smem_raw + ((sizeof(Walk32Shared) + 15) & ~(size_t)15);
  double *s_faces = reinterpret_cast<double *>(cur_ptr);  // mixed walk: face table
  cur_ptr += ((size_t)prm.max_faces * 8 + 15) & ~(size_t)15;
  float *s_kappa = reinterpret_cast<float *>(cur_ptr);
  cur_ptr += (size_t)P * 4;
  Tally32<kTally> tally;
  tally.f_hi = tally.f_lo = nullptr;
  tally.u_lo = tally.u_hi = nullptr;
  tally.u64 = nullptr;
  if (kTally == 3) {
    cur_ptr = (unsigned char *)(((uintptr_t)cur_ptr + 15) & ~(uintptr_t)15);
    tally.u64 = reinterpret_cast<unsigned long long *>(cur_ptr);
    cur_ptr += (size_t)P * 8;
  } else if (kTally == 2) {
    tally.u_lo = reinterpret_cast<uint32_t *>(cur_ptr);
    cur_ptr += (size_t)P * 4;
  } else {
    tally.f_hi = reinterpret_cast<float *>(cur_ptr);
    tally.f_lo = tally.f_hi + P;
    cur_ptr += (size_t)P * (kTally == 1 ? 8 : 4);
  }
  tally.carry_J = nullptr;
  tally.carry_value = 0.;
  Pk *s_pk = reinterpret_cast<Pk *>(cur_ptr);  // [2][CH]
  cur_ptr += sizeof(Pk) * 2 * (size_t)CH;
  Pk *s_stage = reinterpret_cast<Pk *>(cur_ptr);  // [kWarps][kStage]
  cur_ptr += sizeof(Pk) * kWarps * kStage;
  uint32_t *s_skey = reinterpret_cast<uint32_t *>(cur_ptr);  // [kWarps][kStage]

  RoundState *st = prm.st;
  const uint32_t nchunks = st->num_chunks;
  if (nchunks == 0u) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const unsigned lt = (1u << lane) - 1u;
  if (tid < (int)sizeof(DirectionTables) / 4) {
    reinterpret_cast<uint32_t *>(&sh.tab)[tid] =
        reinterpret_cast<const uint32_t *>(&prm.tables)[tid];
  }
  if (tid == 0) {
    mbar_init(&sh.mbar_field, 1);
    mbar_init(&sh.mbar_pk[0], 1);
    mbar_init(&sh.mbar_pk[1], 1);
    sh.uses[0] = sh.uses[1] = 0u;
  }
  for (int c = tid; c < P; c += kThreads) tally.zero(c);
  __syncthreads();

  // TMA of chunk k of the current segment into ring slot k & 1
  auto issue = [&](uint32_t k) {
    const uint32_t slot = k & 1u;
    const uint32_t cnt = (k + 1u < sh.seg_chunks) ? CH : sh.seg_n - (k << ch_shift);
    const uint32_t bytes = cnt * (uint32_t)sizeof(Pk);
    *(volatile uint32_t *)&sh.uses[slot] = sh.uses[slot] + 1u;
    fence_proxy_async();
    mbar_expect_tx(&sh.mbar_pk[slot], bytes);
    tma_load_1d(s_pk + (size_t)slot * CH,
                ((const Pk *)prm.arena_in) + sh.seg_begin + (k << ch_shift), bytes,
                &sh.mbar_pk[slot]);
  };
  // packets of chunk k copied out of the ring by this warp (lane 0): the copy
  // that completes a chunk refills its slot with chunk k + 2
  auto consumed = [&](uint32_t k, uint32_t n) {
    const uint32_t slot = k & 1u;
    const uint32_t cnt = (k + 1u < sh.seg_chunks) ? CH : sh.seg_n - (k << ch_shift);
    __threadfence_block();
    const uint32_t old = atomicAdd(&sh.loaded[slot], n);
    if (old + n == cnt) {
      __threadfence_block();
      *(volatile uint32_t *)&sh.loaded[slot] = 0u;
      __threadfence_block();  // the reset is seen before the refill's issue count
      if (k + 2u < sh.seg_chunks) issue(k + 2u);
    }
  };
  // wait until chunk k of the segment is in its slot (all lanes).  Claims run
  // up to kThreads packets ahead of the copies, so a warp can claim chunk k
  // while its slot still serves chunk k - 2 (or earlier).  A parity wait cannot
  // tell fill `use` from fill `use - 2`, so the warp first waits until fill
  // `use` has been issued: that happens only after chunk k - 2 was copied out
  // completely, which leaves fill `use` as the barrier's current phase.
  auto wait_chunk = [&](uint32_t k) {
    const uint32_t slot = k & 1u;
    const uint32_t use = sh.seg_use0[slot] + (k >> 1);  // this chunk is the use-th fill
    wait_count_above(&sh.uses[slot], use, &st->flags);
    mbar_wait_bounded(&sh.mbar_pk[slot], use & 1u, &st->flags);
  };

  uint32_t phase_field = 0;
  uint32_t staged = kNone;
  uint32_t c_cross = 0, c_trans = 0, c_abs = 0, c_esc = 0, c_reem = 0;
  const uint64_t rseed = st->seed;
  const uint32_t riter = st->iteration;
  uint32_t nstage = 0;  // warp-uniform
  Pk *my_stage = s_stage + warp * kStage;
  uint32_t *my_skey = s_skey + warp * kStage;

  auto flush = [&]() {
    const int64_t off = sh.field_offset;
    const double scale = (kTally >= 2) ? sh.tally_unit : 1.0;
    for (int c = tid; c < sh.ncells; c += kThreads) {
      const double v = tally.take(c, scale);
      if (v != 0.) atomicAdd(&prm.J[off + c], v * sh.sigma);
    }
    flush_counters(prm.stats, sh.instance, c_cross, c_trans, c_abs, c_esc, c_reem);
  };

  // append the first n staged packets of this warp, then move the rest down
  auto flush_stage = [&](uint32_t n) {
    __syncwarp();
    const bool valid = (uint32_t)lane < n;
    Pk rec{};
    uint32_t key = 0;
    if (valid) {
      rec = my_stage[lane];
      key = my_skey[lane];
    }
    warp_append(valid, key, rec, (Pk *)prm.arena_out, prm.keys, prm.ranks, prm.hist, st,
                prm.capacity);
    __syncwarp();
    if ((uint32_t)lane + n < nstage) {
      my_stage[lane] = my_stage[lane + n];
      my_skey[lane] = my_skey[lane + n];
    }
    __syncwarp();
    nstage -= n;
  };

  for (;;) {
    if (tid == 0) {
      // guided run length: about half of an even share of what is left
      const uint32_t done = *(volatile uint32_t *)&st->chunk_next;
      const uint32_t left = (nchunks > done) ? nchunks - done : 0u;
      const uint32_t run = max(1u, min(prm.max_run, left / (2u * gridDim.x)));
      const uint32_t c0 = atomicAdd(&st->chunk_next, run);
      sh.run_c0 = c0;
      sh.run_c1 = min(c0 + run, nchunks);
    }
    __syncthreads();
    if (sh.run_c0 >= nchunks) break;
    uint32_t a = sh.run_c0;
    const uint32_t run_end = sh.run_c1;
    while (a < run_end) {
      if (tid == 0) {
        const Chunk ca = prm.chunks[a];
        const uint32_t b = min(run_end, a + ca.rem);
        const Chunk cl = prm.chunks[b - 1u];
        sh.seg_sub = ca.subgrid;
        sh.seg_begin = ca.begin;
        sh.seg_chunks = b - a;
        sh.seg_n = ((b - 1u - a) << ch_shift) + cl.count;
        sh.seg_next = b;
      }
      __syncthreads();
      const uint32_t sub = sh.seg_sub;
      const uint32_t nseg = sh.seg_n;
      a = sh.seg_next;
      if (sub != staged) {
        if (staged != kNone) flush();
        __syncthreads();
        if (tid == 0) {
          const DevSubgrid &S = prm.subs[sub];
          load_subgrid32(sh, S, prm);
          fence_proxy_async();
          const uint32_t bytes = (uint32_t)S.padded_cells * 4u;
          mbar_expect_tx(&sh.mbar_field, bytes);
          tma_load_1d(s_kappa, prm.kappa + S.field_offset, bytes, &sh.mbar_field);
        }
        mbar_wait_bounded(&sh.mbar_field, phase_field, &st->flags);
        phase_field ^= 1u;
        staged = sub;
        // the mbarrier wait acquires thread 0's writes of the subgrid's geometry
        if (prm.max_faces > 0) fill_faces(s_faces, sh.n, sh.cs, tid, kThreads);
      }
      if (tid == 0) {
        sh.claim = 0u;
        sh.loaded[0] = sh.loaded[1] = 0u;
        sh.seg_use0[0] = sh.uses[0];
        sh.seg_use0[1] = sh.uses[1];
        issue(0u);
        if (sh.seg_chunks > 1u) issue(1u);
      }
      __syncthreads();

      const int limit = sh.n[0] + sh.n[1] + sh.n[2] + 3;
      View v;
      make_view(sh, s_kappa, s_faces, v);
      tally.scale = sh.tally_scale;
      tally.carry_J = prm.J + sh.field_offset;
      tally.carry_value = 4294967296.0 * sh.tally_unit * sh.sigma;
      W w;
      // lane states: active (walking), pending (finished, not yet routed), free
      bool exhausted = false, active = false, pending = false;
      int pstatus = kRun;
      uint32_t rcount = 0;  // reemissions of the lane's packet in this visit
      for (;;) {
        const unsigned running = __ballot_sync(kFull, active);
        // Finished packets are routed and free lanes refilled in one batch,
        // once at least `refill` lanes are not walking (or none is): both
        // blocks are divergent, so running them for one or two lanes at a time
        // would cost more than the crossings they serve.
        if ((uint32_t)(32 - __popc(running)) >= prm.refill || running == 0u) {
          if (__any_sync(kFull, pending)) {
            uint32_t key = kOutside, meta = 0;
            bool append = false;
            bool route = pending;
            if (pending) {
              ++c_trans;
              c_cross += (uint32_t)w.steps;  // one step per crossed cell
              double rd[4];
              uint32_t h[3] = {0u, 0u, 0u};
              if (kReemit && pstatus == kAbsorbed) w.reemit_counter(v, staged, h);
              if (kReemit && pstatus == kAbsorbed && sh.reemission > 0. &&
                  reemit_draw_call(rseed, sh.instance, riter, h[0], h[1], h[2], rcount,
                                   sh.reemission, rd)) {
                // re-emitted in place: the lane walks on from the absorption point
                ++c_reem;
                ++rcount;
                pstatus = w.begin(w.reemitted(v, rd), v, sh.tab.sign_code);
                route = false;
                if (pstatus == kRun) {
                  active = true;
                  pending = false;
                }
              }
            }
            if (route) {
              if (pstatus == kExited) {
                const int od = sh.tab.mask_dir[w.exit_mask(v)];
                if (od >= kNumDirections) {
                  atomicOr(&st->flags, kFlagWalkLimit);
                } else {
                  key = sh.ngb[od];
                  meta = sh.tab.mirror[od];
                  if (key == kOutside) ++c_esc; else append = true;
                }
              } else if (pstatus == kAbsorbed) {
                ++c_abs;
              } else {
                atomicOr(&st->flags, kFlagWalkLimit);
              }
              pending = false;
            }
            const unsigned am = __ballot_sync(kFull, append);
            if (append) {
              const uint32_t slot = nstage + (uint32_t)__popc(am & lt);
              my_stage[slot] = w.packet(v, meta);
              my_skey[slot] = key;
            }
            nstage += (uint32_t)__popc(am);
            if (nstage >= kStageFlush) flush_stage(min(nstage, 32u));
          }
          if (!exhausted) {
            // every lane neither walking nor holding a packet (a re-emitted
            // packet walks on, or waits to be routed in the next batch)
            const unsigned idle = __ballot_sync(kFull, !active && !pending);
            const uint32_t need = (uint32_t)__popc(idle);
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(&sh.claim, need);
            base = __shfl_sync(kFull, base, 0);
            if (need == 0u) {
              // every lane busy after reemission: claim nothing this batch
            } else if (base >= nseg) {
              exhausted = true;
            } else {
              const uint32_t take = min(need, nseg - base);
              const uint32_t k0 = base >> ch_shift, k1 = (base + take - 1u) >> ch_shift;
              wait_chunk(k0);
              if (k1 != k0) wait_chunk(k1);
              const uint32_t r = (uint32_t)__popc(idle & lt);
              if (((idle >> lane) & 1u) && r < take) {
                const uint32_t vi = base + r;
                const uint32_t k = vi >> ch_shift;
                const Pk pk = s_pk[(size_t)(k & 1u) * CH + (vi - (k << ch_shift))];
                const int entry = w.begin(pk, v, sh.tab.sign_code);
                rcount = 0u;
                if (entry == kRun) {
                  active = true;
                } else {  // absorbed or outside at entry: routed next batch
                  pending = true;
                  pstatus = entry;
                }
              }
              __syncwarp();
              if (lane == 0) {
                const uint32_t n0 = min(take, ((k0 + 1u) << ch_shift) - base);
                consumed(k0, n0);
                if (take > n0) consumed(k1, take - n0);
              }
            }
          }
          if (exhausted && !__any_sync(kFull, active || pending)) break;
        }
        if (active) {
          int tcell;
          float len;
          int status = w.step(v, tcell, len);
          tally.add(tcell, len);
          // up to kStepsPerCheck crossings per lane between two looks at the
          // warp (ballot, batch test, reconvergence), which cost more than the
          // idle lanes the longer stretch leaves
#pragma unroll(WalkTraits<W>::kUnroll)
          for (int u = 1; u < kStepsPerCheck; ++u) {
            if (status != kRun) break;
            status = w.step(v, tcell, len);
            tally.add(tcell, len);
          }
          if (status == kRun && w.steps > limit) status = kDrop;
          if (status != kRun) {
            active = false;
            pending = true;
            pstatus = status;
          }
        }
      }
      __syncthreads();  // segment done: every packet of it is traced
    }
  }
  if (nstage > 0u) flush_stage(nstage);
  __syncthreads();
  if (staged != kNone) flush();
  // every issued ring fill has been waited on by its consumers; make sure no
  // bulk copy into this CTA's shared memory outlives it
  if (tid == 0) {
    for (int s = 0; s < 2; ++s)
      if (sh.uses[s] != 0u) mbar_wait_bounded(&sh.mbar_pk[s], (sh.uses[s] - 1u) & 1u, &st->flags);
  }
}

// FP32 walk (cell-unit geometry, 32-byte packets)
template <int kThreads, int kTally, int kMinBlocks, bool kReemit>
__global__ void __launch_bounds__(kThreads, kMinBlocks) k_walk32(WalkParams prm) {
  walk_round<Walk32, kThreads, kTally, kReemit>(prm);
}

// Mixed-precision walk (the reference's FP64 geometry, FP32 optical depths
// and tallies, 64-byte packets)
template <int kThreads, int kTally, int kMinBlocks, bool kReemit>
__global__ void __launch_bounds__(kThreads, kMinBlocks) k_walkm(WalkParams prm) {
  walk_round<WalkM, kThreads, kTally, kReemit>(prm);
}

// ---------------------------------------------------------------------------
// ionization balance (DensitySubGrid.hpp:1628-1658), one block per subgrid
// ---------------------------------------------------------------------------
struct BalanceParams {
  const DevSubgrid *subs;
  const DevInstance *inst;
  const double *nH;
  double *xH, *J;
  float *kappa;  // refreshed for the FP32 walk (may be null)
  DevStats *stats;
  uint32_t first_sub, num_subs;
  double jfac_override;  // >= 0: use instead of the instance's jfac
};

template <int kForm>
__global__ void __launch_bounds__(256) k_balance(BalanceParams prm) {
  __shared__ double red[8];
  const uint32_t s = prm.first_sub + blockIdx.x;
  const DevSubgrid &S = prm.subs[s];
  const DevInstance &I = prm.inst[S.instance];
  if (I.frozen) return;  // converged: x_H kept, J is zero (no packets)
  const double jfac = (prm.jfac_override >= 0.) ? prm.jfac_override : I.jfac;
  const double alpha = I.alpha;
  const double sigma = I.sigma;
  double dx = 0.;
  for (int c = threadIdx.x; c < S.ncells; c += blockDim.x) {
    const int64_t i = S.field_offset + c;
    const double jH = jfac * prm.J[i];
    const double x_old = prm.xH[i];
    double x;
    if (jH > 0.) {
      const double ntot = prm.nH[i];
      const double aa = 0.5 * jH / (ntot * alpha);
      if (kForm == 0) {
        const double bb = 2. / aa;
        const double cc = sqrt(bb + 1.);
        x = 1. + aa * (1. - cc);
      } else {
        x = 1. / (1. + aa + sqrt(aa * (aa + 2.)));
      }
    } else {
      x = 1.;
    }
    prm.xH[i] = x;
    prm.J[i] = 0.;
    if (prm.kappa) prm.kappa[i] = (float)(sigma * prm.nH[i] * x);
    dx += fabs(x - x_old);
  }
  for (int o = 16; o > 0; o >>= 1) dx += __shfl_down_sync(kFull, dx, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = dx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    if (prm.stats) atomicAdd(&prm.stats[S.instance].dx_sum, t);
  }
}

// ---------------------------------------------------------------------------
// fields: layout conversion between caller arrays and the padded device order
// ---------------------------------------------------------------------------
// src index of cell c of (instance-local) subgrid ls
__device__ __forceinline__ int64_t layout_index(const DevSubgrid &S, uint32_t ls, int c,
                                                int layout, const int32_t ns[3],
                                                const int32_t ncell_tot[3]) {
  if (layout == 0) return (int64_t)ls * S.ncells + c;
  const int ix = c / (S.ncell[1] * S.ncell[2]);
  const int iy = (c / S.ncell[2]) % S.ncell[1];
  const int iz = c % S.ncell[2];
  const int sx = ls / (ns[1] * ns[2]);
  const int sy = (ls / ns[2]) % ns[1];
  const int sz = ls % ns[2];
  const int64_t gx = (int64_t)sx * S.ncell[0] + ix, gy = (int64_t)sy * S.ncell[1] + iy,
                gz = (int64_t)sz * S.ncell[2] + iz;
  return (gx * ncell_tot[1] + gy) * ncell_tot[2] + gz;
}

struct LayoutParams {
  const DevSubgrid *subs;
  uint32_t first_sub;
  int32_t ns[3], ncell[3];
  int layout;
};

__global__ void k_fields_in(LayoutParams lp, const double *src, double *dst) {
  const uint32_t ls = blockIdx.x;
  const DevSubgrid &S = lp.subs[lp.first_sub + ls];
  for (int c = threadIdx.x; c < S.ncells; c += blockDim.x) {
    dst[S.field_offset + c] = src[layout_index(S, ls, c, lp.layout, lp.ns, lp.ncell)];
  }
}

__global__ void k_fields_out(LayoutParams lp, const double *src, double *dst) {
  const uint32_t ls = blockIdx.x;
  const DevSubgrid &S = lp.subs[lp.first_sub + ls];
  for (int c = threadIdx.x; c < S.ncells; c += blockDim.x) {
    dst[layout_index(S, ls, c, lp.layout, lp.ns, lp.ncell)] = src[S.field_offset + c];
  }
}

__global__ void k_kappa(const DevSubgrid *subs, const DevInstance *inst, uint32_t first_sub,
                        const double *nH, const double *xH, float *kappa) {
  const DevSubgrid &S = subs[first_sub + blockIdx.x];
  const double sigma = inst[S.instance].sigma;
  for (int c = threadIdx.x; c < S.padded_cells; c += blockDim.x) {
    const int64_t i = S.field_offset + c;
    kappa[i] = (c < S.ncells) ? (float)(sigma * nH[i] * xH[i]) : 0.f;
  }
}

__global__ void k_fill(double *a, double v, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    a[i] = v;
}

// ---------------------------------------------------------------------------
// one buffer through one subgrid (do_photon_traversal), optional trace
// ---------------------------------------------------------------------------
struct TraverseParams {
  const DevSubgrid *subs;
  const DevInstance *inst;
  uint32_t sub;
  int32_t input_direction;
  const Packet64 *in;
  uint32_t n;
  Packet64 *out;
  int32_t *out_dir;
  const float *kappa;
  const double *nH, *xH;
  double *J;
  int32_t max_padded;
  int32_t *trace_cells;  // packet 0 only
  double *trace_len;
  int32_t max_steps;
  int32_t *trace_steps;
  RoundState *st;
  DirectionTables tables;
};

// K: the transport's packet record.  The mixed-precision walk takes each
// photon's own cross section: its cell opacity is (float)(sigma n x) of the
// photon's sigma (the production kappa when sigma is the instance's), and it
// tallies (lmin sigma) weight into J as the reference does.
template <int K>
__global__ void __launch_bounds__(256) k_traverse(TraverseParams prm) {
  constexpr bool kF32 = K == kPk32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ DirectionTables tab;
  const DevSubgrid &S = prm.subs[prm.sub];
  const int P = prm.max_padded;
  float *s_kappa = reinterpret_cast<float *>(smem_raw);
  float *s_hi = s_kappa + P;
  float *s_lo = s_hi + P;
  double *s_n = reinterpret_cast<double *>(smem_raw);
  double *s_x = s_n + P;
  double *s_J = s_x + P;
  double *s_faces = s_J + P;  // mixed walk: face table (nx + ny + nz + 3 entries)
  if (threadIdx.x < sizeof(DirectionTables) / 4) {
    reinterpret_cast<uint32_t *>(&tab)[threadIdx.x] =
        reinterpret_cast<const uint32_t *>(&prm.tables)[threadIdx.x];
  }
  for (int c = threadIdx.x; c < S.ncells; c += blockDim.x) {
    if (kF32) {
      s_kappa[c] = prm.kappa[S.field_offset + c];
      s_hi[c] = 0.f;
      s_lo[c] = 0.f;
    } else {
      s_n[c] = prm.nH[S.field_offset + c];
      s_x[c] = prm.xH[S.field_offset + c];
      s_J[c] = 0.;
    }
  }
  if (K == kPkM) fill_faces(s_faces, S.ncell, S.cell_size, threadIdx.x, blockDim.x);
  __syncthreads();
  View32 v32;
  View64 v64;
  for (int a = 0; a < 3; ++a) {
    v32.n[a] = v64.n[a] = S.ncell[a];
    v32.cs[a] = S.cell_size_f[a];
    v32.inv_cs[a] = (float)S.inv_cell_size[a];
    v64.anchor[a] = S.anchor[a];
    v64.cs[a] = S.cell_size[a];
    v64.inv_cs[a] = S.inv_cell_size[a];
  }
  v32.nyz = v64.nyz = S.ncell[1] * S.ncell[2];
  v32.kappa = s_kappa;
  Tally32<1> tally32;
  tally32.f_hi = s_hi;
  tally32.f_lo = s_lo;
  tally32.u_lo = tally32.u_hi = nullptr;
  tally32.u64 = nullptr;
  tally32.scale = 1.f;
  v64.nH = s_n;
  v64.xH = s_x;
  v64.J = s_J;
  const int limit = S.ncell[0] + S.ncell[1] + S.ncell[2] + 3;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < prm.n) {
    Packet64 ph = prm.in[i];
    ph.meta = (uint32_t)prm.input_direction;
    const bool tracing = (i == 0 && prm.trace_steps != nullptr);
    int status, nsteps = 0;
    int result = kInside;
    if (kF32) {
      Packet32 pk;
      for (int a = 0; a < 3; ++a) {
        pk.pos[a] = (float)((ph.pos[a] - S.anchor[a]) * S.inv_cell_size[a]);
        pk.dir[a] = (float)ph.dir[a];
      }
      pk.tau = (float)ph.tau;
      pk.meta = ph.meta;
      Walk32 w;
      status = w.begin(pk, v32, tab.sign_code);
      while (status == kRun) {
        int cell;
        float len;
        status = w.step(v32, cell, len);
        tally32.add(cell, len);
        if (tracing && nsteps < prm.max_steps) {
          prm.trace_cells[nsteps] = cell;
          prm.trace_len[nsteps] = (double)len;
        }
        ++nsteps;
        if (status == kRun && w.steps > limit) status = kDrop;
      }
      for (int a = 0; a < 3; ++a) ph.pos[a] = S.anchor[a] + (double)w.p[a] * S.cell_size[a];
      ph.tau = (double)__fsub_rn(w.tau_target, w.tau_done);
      if (status == kExited) result = tab.mask_dir[w.exit_mask(v32, false)];
    } else if (K == kPkM) {
      ViewM vm;
      vm.kappa = nullptr;
      vm.anchor = S.anchor;
      vm.cs = S.cell_size;
      vm.inv_cs = S.inv_cell_size;
      vm.faces = s_faces;
      for (int a = 0; a < 3; ++a) vm.n[a] = S.ncell[a];
      vm.face_off[0] = 0;
      vm.face_off[1] = S.ncell[0] + 1;
      vm.face_off[2] = S.ncell[0] + S.ncell[1] + 2;
      vm.nyz = v64.nyz;
      PacketM pk;
      for (int a = 0; a < 3; ++a) {
        pk.pos[a] = ph.pos[a];
        pk.dir[a] = ph.dir[a];
      }
      pk.tau = tau32(ph.tau);
      pk.meta = ph.meta;
      const double sg = ph.sigma, wt = ph.weight;
      WalkM w;
      status = w.begin(pk, vm, tab.sign_code);
      while (status == kRun) {
        const int c = w.cell;
        const float k = (float)(sg * s_n[c] * s_x[c]);
        int cell;
        float lf;
        double len;
        status = w.step_k(vm, k, cell, lf, &len);
        atomicAdd(&s_J[cell], len * sg * wt);
        if (tracing && nsteps < prm.max_steps) {
          prm.trace_cells[nsteps] = cell;
          prm.trace_len[nsteps] = len;
        }
        ++nsteps;
        if (status == kRun && w.steps > limit) status = kDrop;
      }
      const PacketM o = w.packet(vm, 0u);
      for (int a = 0; a < 3; ++a) ph.pos[a] = o.pos[a];
      ph.tau = (double)o.tau;
      if (status == kExited) result = tab.mask_dir[w.exit_mask(vm)];
    } else {
      Walk64 w;
      status = w.begin(ph, v64, tab.sign_code);
      while (status == kRun) {
        const int cell = w.cell;
        double len;
        status = w.step(v64, &len);
        if (tracing && nsteps < prm.max_steps) {
          prm.trace_cells[nsteps] = cell;
          prm.trace_len[nsteps] = len;
        }
        ++nsteps;
        if (status == kRun && w.steps > limit) status = kDrop;
      }
      ph = w.packet(v64, 0u);
      if (status == kExited) result = tab.mask_dir[w.exit_mask(v64)];
    }
    if (status == kDrop || result >= kNumDirections) {
      atomicOr(&prm.st->flags, kFlagWalkLimit);
      result = kInside;
    }
    ph.meta = 0u;
    prm.out[i] = ph;
    prm.out_dir[i] = result;
    if (tracing) *prm.trace_steps = nsteps;
  }
  __syncthreads();
  const double sw = prm.inst[S.instance].sigma;
  for (int c = threadIdx.x; c < S.ncells; c += blockDim.x) {
    if (kF32) {
      const double v = ((double)s_hi[c] + (double)s_lo[c]) * sw;
      if (v != 0.) atomicAdd(&prm.J[S.field_offset + c], v);
    } else {
      if (s_J[c] != 0.) atomicAdd(&prm.J[S.field_offset + c], s_J[c]);
    }
  }
}

// Stable grouping of the traversed photons by output direction (the 27
// output buffers of do_photon_traversal, in input order).  One block.
__global__ void __launch_bounds__(256) k_partition(const Packet64 *photons,
                                                   const int32_t *dirs, uint32_t n,
                                                   const uint8_t *enabled, Packet64 *out,
                                                   uint32_t *counts, uint32_t *done) {
  __shared__ uint32_t cnt[256][kNumDirections + 1];
  __shared__ uint32_t base[kNumDirections + 1];
  const uint32_t per = (n + 255) / 256;
  const uint32_t b = threadIdx.x * per, e = min(n, b + per);
  for (int d = 0; d < kNumDirections; ++d) cnt[threadIdx.x][d] = 0;
  for (uint32_t i = b; i < e; ++i) cnt[threadIdx.x][dirs[i]] += 1;
  __syncthreads();
  if (threadIdx.x < kNumDirections) {
    const int d = threadIdx.x;
    uint32_t acc = 0;
    for (int t = 0; t < 256; ++t) {
      const uint32_t c = cnt[t][d];
      cnt[t][d] = acc;
      acc += c;
    }
    base[d] = acc;  // total of direction d for now
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t acc = 0, dropped = 0;
    for (int d = 0; d < kNumDirections; ++d) {
      const uint32_t tot = base[d];
      const bool on = enabled == nullptr || enabled[d] != 0;
      counts[d] = on ? tot : 0u;
      base[d] = on ? acc : kNone;
      if (on) acc += tot; else dropped += tot;
    }
    *done = dropped;
  }
  __syncthreads();
  for (uint32_t i = b; i < e; ++i) {
    const int d = dirs[i];
    if (base[d] != kNone) {
      out[base[d] + cnt[threadIdx.x][d]] = photons[i];
    }
    cnt[threadIdx.x][d] += 1;
  }
}

}  // namespace cmi
