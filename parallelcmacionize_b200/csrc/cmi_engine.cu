// Host side of the B200 transport engine: context, device memory, launch
// sequence of one iteration, CUDA-graph capture and the extern "C" ABI of
// include/cmacionize_b200.h.
#include "cmacionize_b200.h"

#include "cmi_kernels.cuh"
#include "cmi_dust.cuh"

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

using namespace cmi;

namespace {

thread_local std::string g_last_error;

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

#define CMI_CUDA(call)                                                                     \
  do {                                                                                     \
    const cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) {                                                               \
      (void)cudaGetLastError(); /* a non-sticky error must not fail the next check */      \
      return fail(e_ == cudaErrorMemoryAllocation ? CMI_ERR_OUT_OF_MEMORY : CMI_ERR_CUDA, \
                  "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__,       \
                  __LINE__);                                                               \
    }                                                                                      \
  } while (0)

#define CMI_TRY(expr)           \
  do {                          \
    const int rc_ = (expr);     \
    if (rc_ != CMI_OK) return rc_; \
  } while (0)

constexpr int kWalkThreads = 256;
constexpr int kSpareRounds = 3;  // wavefront rounds beyond the straight-line bound
// With reemission a packet starts new straight paths, so its subgrid transits
// have no fixed bound: the round loop runs until no packet is left, capped
// here only against a runaway loop.
constexpr int kReemissionRoundCap = 4096;
// lanes not walking before a warp routes + refills: FP32 walk 16 (sweep on B200,
// lognormal128: 12 -> 6.77e10, 16 -> 6.92e10, 24 -> 6.86e10); the mixed walk's
// longer FP64 steps favour 12 (8 -> 6.05e10, 12 -> 6.07e10, 16 -> 5.98e10,
// 24 -> 5.69e10)
constexpr uint32_t kDefaultRefill = 16;
constexpr uint32_t kDefaultRefillMixed = 12;

struct HostInstance {
  cmi_grid_desc desc;
  int32_t sub_ncell[3];
  int32_t cells_per_sub;
  int32_t padded_per_sub;
  uint32_t first_sub, nsub;
  int64_t first_cell;  // padded offset of the first subgrid
  int64_t ncells;
  std::vector<double> src_pos, src_lum;
  uint64_t num_photon = 0;
  double reemission = 0.;  // reemission_probability (params.txt)
};

template <class T>
int dev_alloc(T **p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  CMI_CUDA(cudaMalloc((void **)p, sizeof(T) * count));
  return CMI_OK;
}

template <class T>
void dev_free(T *&p) {
  if (p) cudaFree((void *)p);
  p = nullptr;
}

}  // namespace

struct DustBuffers;
void free_dust_buffers(DustBuffers *b);

struct cmi_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  cmi_options opt{};
  int num_sms = 0;
  std::vector<HostInstance> inst;
  std::vector<DevSubgrid> h_sub;
  uint32_t S = 0;
  int64_t total_padded = 0;
  int32_t max_padded = 0;
  int32_t max_faces = 0;  // largest nx + ny + nz + 3 of a subgrid (the mixed walk's face table)
  int rounds = 1;     // straight-line bound + spares
  int round_cap = 1;  // rounds an iteration may run (rounds, or more with reemission)
  bool reemission = false;  // some instance re-emits absorbed packets
  DirectionTables tables{};

  DevSubgrid *d_sub = nullptr;
  DevInstance *d_inst = nullptr;
  DevSource *d_src = nullptr;
  int nsrc_total = 0;
  double *d_nH = nullptr, *d_xH = nullptr, *d_J = nullptr;
  float *d_kappa = nullptr;
  uint64_t *d_src_count = nullptr, *d_src_first = nullptr, *d_buf_first = nullptr;
  uint32_t *d_src_rank0 = nullptr;  // first place of each source's packets in its bucket
  RoundState *d_state = nullptr;
  DevStats *d_stats = nullptr;
  uint32_t *d_hist = nullptr, *d_bucket_off = nullptr;
  uint32_t *d_tile_pk = nullptr, *d_tile_ch = nullptr, *d_tile_pk_off = nullptr,
           *d_tile_ch_off = nullptr;
  uint32_t *d_plan_choff = nullptr, *d_plan_pkoff = nullptr;  // kPlanTile + 1 each
  uint32_t ntiles = 0;
  Chunk *d_chunks = nullptr;
  uint64_t chunk_capacity = 0;
  void *d_arena_in = nullptr, *d_arena_out = nullptr;
  uint32_t *d_keys = nullptr, *d_ranks = nullptr;
  uint64_t capacity = 0;  // packets
  double *d_stage = nullptr;
  size_t stage_bytes = 0;

  // walk launch configuration
  int walk_grid = 0;
  size_t walk_smem = 0;
  uint32_t chunk = 4096;

  // graph of one iteration
  // captured iterations: [0] transport only (cmi_shoot_packets), [1] with the balance
  cudaGraphExec_t graph_exec[2] = {nullptr, nullptr};
  bool graph_dirty = true;
  bool capturing = false;        // enqueue_iteration is being captured
  cudaStream_t body_stream = nullptr;  // captures the round loop's body
  uint64_t graph_kernels[2] = {0, 0};  // kernels per iteration outside the round loop
  uint64_t graph_body_kernels = 0;  // kernels per round of the loop
  uint64_t last_launches = 0;
  uint64_t enqueued = 0;  // kernel launches of the current enqueue
  DevStats *h_stats = nullptr;  // pinned
  size_t h_stats_count = 0;

  // optional per-kernel event timing
  bool timing = false;
  struct Timed {
    int cls;
    cudaEvent_t start, stop;
  };
  std::vector<Timed> timed;
  std::vector<cudaEvent_t> event_pool;

  // cmi_prefetch_number_density: n_H copied on a side stream into its own
  // staging (the padded layout's offsets); cmi_set_fields_prefetched takes it
  // up on the same stream, after the copy
  cudaStream_t copy_stream = nullptr;
  double *d_nh_stage = nullptr;
  std::vector<int32_t> nh_layout;  // -1: nothing prefetched for the instance
  // cmi_set_fields_prefetched issues its copies and the kappa refresh on
  // copy_stream (after main_mark, the main stream's work so far) and records
  // fields_ready.  An iteration waits for it after the emission, which reads
  // no field, so the copies overlap the emission; every other entry point
  // waits before its first use (fields_pending)
  cudaEvent_t fields_ready = nullptr;
  cudaEvent_t main_mark = nullptr;
  bool fields_pending = false;

  // cmi_dust_run's packet buffers, grown to the largest call and kept
  DustBuffers *dust = nullptr;
  uint64_t dust_capacity = 0;  // packets
  size_t dust_pixels = 0;

  bool fp32() const { return opt.transport_precision == CMI_TRANSPORT_FP32; }
  bool mixed() const { return opt.transport_precision == CMI_TRANSPORT_MIXED; }
  // the FP32 and mixed walks read the FP32 opacity field kappa = sigma n x
  bool uses_kappa() const { return fp32() || mixed(); }
  int kind() const { return fp32() ? kPk32 : (mixed() ? kPkM : kPk64); }
  size_t packet_bytes() const {
    return fp32() ? sizeof(Packet32) : (mixed() ? sizeof(PacketM) : sizeof(Packet64));
  }
  const char *precision_name() const { return fp32() ? "FP32" : (mixed() ? "mixed" : "FP64"); }
};

namespace {

// await_fields: order the main stream after fields still being copied in by
// cmi_set_fields_prefetched (the iteration entry points pass false: their
// iteration waits inside, after the emission)
int check_ctx(cmi_context *c, bool await_fields = true) {
  if (!c) return fail(CMI_ERR_INVALID_ARGUMENT, "null context");
  CMI_CUDA(cudaSetDevice(c->device));
  if (await_fields && c->fields_pending) {
    CMI_CUDA(cudaStreamWaitEvent(c->stream, c->fields_ready, 0));
    c->fields_pending = false;
  }
  return CMI_OK;
}

int check_instance(cmi_context *c, int32_t i) {
  if (i < 0 || i >= (int32_t)c->inst.size())
    return fail(CMI_ERR_INVALID_ARGUMENT, "instance %d out of range [0, %zu)", i, c->inst.size());
  return CMI_OK;
}

void free_graph(cmi_context *c) {
  for (cudaGraphExec_t &g : c->graph_exec) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
  }
  c->graph_dirty = true;
}

cudaEvent_t pool_event(cmi_context *c) {
  if (!c->event_pool.empty()) {
    cudaEvent_t e = c->event_pool.back();
    c->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Event pair around the launches issued by `launch` (timing mode only).
template <class F>
int timed_launch(cmi_context *c, int cls, F &&launch) {
  if (!c->timing) return launch();
  cmi_context::Timed t{cls, pool_event(c), pool_event(c)};
  cudaEventRecord(t.start, c->stream);
  const int rc = launch();
  cudaEventRecord(t.stop, c->stream);
  c->timed.push_back(t);
  return rc;
}

// Arena for `packets` packets in flight.
int ensure_capacity(cmi_context *c, uint64_t packets) {
  if (packets <= c->capacity && c->d_arena_in) return CMI_OK;
  if (packets > 0xF0000000ull)
    return fail(CMI_ERR_CAPACITY, "%llu packets exceed the 32-bit arena index",
                (unsigned long long)packets);
  const uint64_t cap = std::max<uint64_t>(packets, 1024);
  free_graph(c);
  dev_free(c->d_arena_in);
  dev_free(c->d_arena_out);
  dev_free(c->d_keys);
  dev_free(c->d_ranks);
  dev_free(c->d_chunks);
  const size_t pb = c->packet_bytes();
  CMI_CUDA(cudaMalloc(&c->d_arena_in, pb * cap));
  CMI_CUDA(cudaMalloc(&c->d_arena_out, pb * cap));
  CMI_TRY(dev_alloc(&c->d_keys, cap));
  CMI_TRY(dev_alloc(&c->d_ranks, cap));
  c->chunk_capacity = (uint64_t)c->S + cap / c->chunk + 16;
  CMI_TRY(dev_alloc(&c->d_chunks, c->chunk_capacity));
  c->capacity = cap;
  const uint32_t cap32 = (uint32_t)cap;
  CMI_CUDA(cudaMemcpyAsync(&c->d_state->capacity, &cap32, sizeof(cap32), cudaMemcpyHostToDevice,
                           c->stream));
  CMI_CUDA(cudaStreamSynchronize(c->stream));
  return CMI_OK;
}

int ensure_stage(cmi_context *c, size_t bytes) {
  if (bytes <= c->stage_bytes) return CMI_OK;
  dev_free(c->d_stage);
  CMI_CUDA(cudaMalloc(&c->d_stage, bytes));
  c->stage_bytes = bytes;
  return CMI_OK;
}

uint64_t total_budget(const cmi_context *c) {
  uint64_t n = 0;
  for (const auto &I : c->inst) n += I.num_photon;
  return n;
}

// Upload instance + source tables (after sources or budgets change).
int upload_tables(cmi_context *c) {
  bool reemission = false;
  for (const HostInstance &I : c->inst) reemission = reemission || I.reemission > 0.;
  c->round_cap = reemission ? std::max(c->rounds, kReemissionRoundCap) : c->rounds;
  c->reemission = reemission;
  std::vector<DevInstance> di(c->inst.size());
  std::vector<DevSource> ds;
  for (size_t i = 0; i < c->inst.size(); ++i) {
    HostInstance &I = c->inst[i];
    DevInstance &D = di[i];
    double L = 0.;
    for (double l : I.src_lum) L += l;
    const double inv[3] = {I.sub_ncell[0] / (I.desc.box[3] / I.desc.num_subgrid[0]),
                           I.sub_ncell[1] / (I.desc.box[4] / I.desc.num_subgrid[1]),
                           I.sub_ncell[2] / (I.desc.box[5] / I.desc.num_subgrid[2])};
    // DensitySubGrid.hpp:1633: luminosity / num_photon * inv_cell_size^3
    D.jfac = (I.num_photon > 0) ? L / (double)I.num_photon * inv[0] * inv[1] * inv[2] : 0.;
    D.alpha = I.desc.recombination_rate;
    D.sigma = I.desc.cross_section;
    D.total_luminosity = L;
    D.num_photon = I.num_photon;
    D.first_subgrid = I.first_sub;
    D.num_subgrids = I.nsub;
    D.first_source = (uint32_t)ds.size();
    D.num_sources = (uint32_t)I.src_lum.size();
    D.num_cells = I.ncells;
    D.reemission = (float)I.reemission;
    const int32_t *ns = I.desc.num_subgrid;
    for (size_t k = 0; k < I.src_lum.size(); ++k) {
      DevSource s{};
      uint32_t si[3];
      for (int a = 0; a < 3; ++a) {
        s.position[a] = I.src_pos[3 * k + a];
        // testDensitySubGrid_omp.cpp:1983-1990, clamped to the box
        long v = (long)((s.position[a] - I.desc.box[a]) / I.desc.box[3 + a] * ns[a]);
        v = std::min<long>(std::max<long>(v, 0), ns[a] - 1);
        si[a] = (uint32_t)v;
      }
      const uint32_t local = (si[0] * ns[1] + si[1]) * ns[2] + si[2];
      s.subgrid = I.first_sub + local;
      const DevSubgrid &S = c->h_sub[s.subgrid];
      for (int a = 0; a < 3; ++a) {
        s.pos_cell[a] = (float)((s.position[a] - S.anchor[a]) * S.inv_cell_size[a]);
      }
      s.luminosity = I.src_lum[k];
      s.instance = (uint32_t)i;
      s.local_index = (uint32_t)k;
      ds.push_back(s);
    }
  }
  dev_free(c->d_src);
  dev_free(c->d_src_count);
  dev_free(c->d_src_first);
  dev_free(c->d_src_rank0);
  dev_free(c->d_buf_first);
  c->nsrc_total = (int)ds.size();
  CMI_TRY(dev_alloc(&c->d_src, ds.size()));
  CMI_TRY(dev_alloc(&c->d_src_count, ds.size() + 1));
  CMI_TRY(dev_alloc(&c->d_src_first, ds.size() + 1));
  CMI_TRY(dev_alloc(&c->d_buf_first, ds.size() + 1));
  CMI_TRY(dev_alloc(&c->d_src_rank0, ds.size() + 1));
  if (!ds.empty())
    CMI_CUDA(cudaMemcpyAsync(c->d_src, ds.data(), sizeof(DevSource) * ds.size(),
                             cudaMemcpyHostToDevice, c->stream));
  CMI_CUDA(cudaMemcpyAsync(c->d_inst, di.data(), sizeof(DevInstance) * di.size(),
                           cudaMemcpyHostToDevice, c->stream));
  CMI_CUDA(cudaStreamSynchronize(c->stream));
  free_graph(c);
  return CMI_OK;
}

int refresh_kappa(cmi_context *c, int32_t i, cudaStream_t s = nullptr) {
  if (!c->uses_kappa()) return CMI_OK;
  const HostInstance &I = c->inst[i];
  k_kappa<<<I.nsub, 256, 0, s ? s : c->stream>>>(c->d_sub, c->d_inst, I.first_sub, c->d_nH,
                                                 c->d_xH, c->d_kappa);
  CMI_CUDA(cudaGetLastError());
  return CMI_OK;
}

// ---------------------------------------------------------------------------
// launch helpers (each counts its kernel)
// ---------------------------------------------------------------------------
// Plan of a round from the bucket histogram; with scatter, the packets the
// previous step appended are moved into their buckets.
// gate: inside the captured round loop, the scatter also sets the loop's
// condition (handle h)
int launch_plan(cmi_context *c, bool scatter, bool gate = false,
                cudaGraphConditionalHandle h = 0) {
  if (c->ntiles == 1) {
    k_plan_fused<<<1, kPlanThreads, 0, c->stream>>>(c->d_hist, c->S, c->chunk, c->d_bucket_off,
                                                    c->d_chunks, c->d_state, c->d_plan_choff,
                                                    c->d_plan_pkoff);
    c->enqueued += 1;
    // a round has at most capacity / chunk + S chunks; below the in-block
    // limit k_plan_fused writes every list itself and the launch is left out
    if (c->capacity / c->chunk + c->S + 1 > kPlanChunksInBlock) {
      k_plan_chunks<<<c->num_sms * 2, 256, 0, c->stream>>>(c->d_plan_choff, c->d_plan_pkoff,
                                                           c->chunk, c->d_chunks, c->d_state);
      c->enqueued += 1;
    }
  } else {
    k_plan_count<<<c->ntiles, kPlanThreads, 0, c->stream>>>(c->d_hist, c->S, c->chunk,
                                                            c->d_tile_pk, c->d_tile_ch);
    k_plan_offsets<<<1, kPlanThreads, 0, c->stream>>>(c->ntiles, c->d_tile_pk, c->d_tile_ch,
                                                       c->d_tile_pk_off, c->d_tile_ch_off,
                                                       c->d_state);
    k_plan_write<<<c->ntiles, kPlanThreads, 0, c->stream>>>(c->d_hist, c->S, c->chunk,
                                                            c->d_tile_pk_off, c->d_tile_ch_off,
                                                            c->d_bucket_off, c->d_chunks);
    c->enqueued += 3;
  }
  if (scatter) {
    const int grid = c->num_sms * 8;
    if (c->fp32()) {
      k_scatter<Packet32><<<grid, 256, 0, c->stream>>>(
          (const Packet32 *)c->d_arena_out, c->d_keys, c->d_ranks, c->d_bucket_off,
          (Packet32 *)c->d_arena_in, c->d_state, (uint32_t)c->capacity, gate, h,
          (uint32_t)c->round_cap);
    } else if (c->mixed()) {
      k_scatter<PacketM><<<grid, 256, 0, c->stream>>>(
          (const PacketM *)c->d_arena_out, c->d_keys, c->d_ranks, c->d_bucket_off,
          (PacketM *)c->d_arena_in, c->d_state, (uint32_t)c->capacity, gate, h,
          (uint32_t)c->round_cap);
    } else {
      k_scatter<Packet64><<<grid, 256, 0, c->stream>>>(
          (const Packet64 *)c->d_arena_out, c->d_keys, c->d_ranks, c->d_bucket_off,
          (Packet64 *)c->d_arena_in, c->d_state, (uint32_t)c->capacity, gate, h,
          (uint32_t)c->round_cap);
    }
    c->enqueued += 1;
  }
  CMI_CUDA(cudaGetLastError());
  return CMI_OK;
}

WalkParams walk_params(cmi_context *c) {
  WalkParams p{};
  p.chunk = c->chunk;
  p.max_run = c->opt.max_run_chunks > 0 ? (uint32_t)c->opt.max_run_chunks : 64u;
  p.refill = c->opt.refill_lanes > 0 ? (uint32_t)c->opt.refill_lanes
                                      : (c->mixed() ? kDefaultRefillMixed : kDefaultRefill);
  p.subs = c->d_sub;
  p.inst = c->d_inst;
  p.chunks = c->d_chunks;
  p.st = c->d_state;
  p.stats = c->d_stats;
  p.arena_in = c->d_arena_in;
  p.arena_out = c->d_arena_out;
  p.keys = c->d_keys;
  p.ranks = c->d_ranks;
  p.hist = c->d_hist;
  p.capacity = (uint32_t)c->capacity;
  p.max_padded = c->max_padded;
  p.max_faces = c->mixed() ? c->max_faces : 0;
  p.kappa = c->d_kappa;
  p.nH = c->d_nH;
  p.xH = c->d_xH;
  p.J = c->d_J;
  p.tables = c->tables;
  return p;
}

// the fixed-point default is built for 4 resident CTAs per SM (<= 64
// registers); ctas_per_sm = 3 selects a build for 3 (<= 85 registers)
template <int kTally>
constexpr int walk32_min_blocks() { return kTally == 2 ? 4 : 1; }

bool walk32_three_per_sm(const cmi_context *c) {
  return c->opt.tally_mode == CMI_TALLY_FIXED64 && c->opt.ctas_per_sm == 3;
}

// the mixed-precision walk: 64-byte packets, FP64 geometry in registers; built
// for 3 resident CTAs per SM (<= 85 registers)
template <int kTally>
constexpr int walkm_min_blocks() { return kTally == 2 ? 3 : 1; }

template <int kTally, bool kReemit>
void launch_walk32_r(cmi_context *c, const WalkParams &p) {
  if (c->mixed())
    k_walkm<kWalkThreads, kTally, walkm_min_blocks<kTally>(), kReemit>
        <<<c->walk_grid, kWalkThreads, c->walk_smem, c->stream>>>(p);
  else if (kTally == 2 && walk32_three_per_sm(c))
    k_walk32<kWalkThreads, 2, 3, kReemit>
        <<<c->walk_grid, kWalkThreads, c->walk_smem, c->stream>>>(p);
  else
    k_walk32<kWalkThreads, kTally, walk32_min_blocks<kTally>(), kReemit>
        <<<c->walk_grid, kWalkThreads, c->walk_smem, c->stream>>>(p);
}

template <int kTally>
void launch_walk32_t(cmi_context *c, const WalkParams &p) {
  if (c->reemission) launch_walk32_r<kTally, true>(c, p);
  else launch_walk32_r<kTally, false>(c, p);
}

int launch_walk(cmi_context *c) {
  const WalkParams p = walk_params(c);
  if (c->uses_kappa()) {
    switch (c->opt.tally_mode) {
      case 0: launch_walk32_t<0>(c, p); break;
      case 1: launch_walk32_t<1>(c, p); break;
      case 2: launch_walk32_t<2>(c, p); break;
      default: launch_walk32_t<3>(c, p); break;
    }
  } else {
    k_walk64<kWalkThreads><<<c->walk_grid, kWalkThreads, c->walk_smem, c->stream>>>(p);
  }
  c->enqueued += 1;
  CMI_CUDA(cudaGetLastError());
  return CMI_OK;
}

template <class F>
int config_kernel(cmi_context *c, F fn) {
  int optin = 0;
  CMI_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
  if (c->walk_smem > (size_t)optin)
    return fail(CMI_ERR_NOT_SUPPORTED,
                "the %s walk needs %zu B of shared memory per CTA (largest subgrid %d cells%s), "
                "the device allows %d B",
                c->precision_name(), c->walk_smem, (int)c->max_padded,
                c->uses_kappa() ? ", two packet-ring chunks: lower packets_per_chunk" : "", optin);
  CMI_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)c->walk_smem));
  int per_sm = 0;
  CMI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kWalkThreads,
                                                         c->walk_smem));
  if (per_sm <= 0)
    return fail(CMI_ERR_NOT_SUPPORTED, "walk kernel does not fit on an SM (smem %zu B)",
                c->walk_smem);
  if (c->opt.ctas_per_sm > 0) per_sm = std::min(per_sm, (int)c->opt.ctas_per_sm);
  c->walk_grid = c->num_sms * per_sm;
  return CMI_OK;
}

int config_walk(cmi_context *c) {
  if (c->uses_kappa()) {
    const size_t head = (sizeof(Walk32Shared) + 15) & ~(size_t)15;
    const int tm = c->opt.tally_mode;
    const size_t tally_bytes = (tm == 0 || tm == 2 ? 4 : 8) * (size_t)c->max_padded + 16;
    const size_t pb = c->packet_bytes();
    const size_t faces = c->mixed() ? (((size_t)c->max_faces * 8 + 15) & ~(size_t)15) : 0;
    c->walk_smem = head + faces + 4 * (size_t)c->max_padded + tally_bytes +
                   pb * 2 * (size_t)c->chunk + (pb + 4) * (kWalkThreads / 32) * kStage;
    if (c->mixed()) {
      switch (tm) {
        case 0:
          CMI_TRY(config_kernel(c, k_walkm<kWalkThreads, 0, walkm_min_blocks<0>(), true>));
          return config_kernel(c, k_walkm<kWalkThreads, 0, walkm_min_blocks<0>(), false>);
        case 1:
          CMI_TRY(config_kernel(c, k_walkm<kWalkThreads, 1, walkm_min_blocks<1>(), true>));
          return config_kernel(c, k_walkm<kWalkThreads, 1, walkm_min_blocks<1>(), false>);
        case 2:
          CMI_TRY(config_kernel(c, k_walkm<kWalkThreads, 2, walkm_min_blocks<2>(), true>));
          return config_kernel(c, k_walkm<kWalkThreads, 2, walkm_min_blocks<2>(), false>);
        default:
          CMI_TRY(config_kernel(c, k_walkm<kWalkThreads, 3, walkm_min_blocks<3>(), true>));
          return config_kernel(c, k_walkm<kWalkThreads, 3, walkm_min_blocks<3>(), false>);
      }
    }
    // both builds (with and without reemission) get the attribute; the grid
    // comes from the build without (the same 64-register occupancy bound)
    switch (tm) {
      case 0:
        CMI_TRY(config_kernel(c, k_walk32<kWalkThreads, 0, walk32_min_blocks<0>(), true>));
        return config_kernel(c, k_walk32<kWalkThreads, 0, walk32_min_blocks<0>(), false>);
      case 1:
        CMI_TRY(config_kernel(c, k_walk32<kWalkThreads, 1, walk32_min_blocks<1>(), true>));
        return config_kernel(c, k_walk32<kWalkThreads, 1, walk32_min_blocks<1>(), false>);
      case 2:
        if (walk32_three_per_sm(c)) {
          CMI_TRY(config_kernel(c, k_walk32<kWalkThreads, 2, 3, true>));
          return config_kernel(c, k_walk32<kWalkThreads, 2, 3, false>);
        }
        CMI_TRY(config_kernel(c, k_walk32<kWalkThreads, 2, 4, true>));
        return config_kernel(c, k_walk32<kWalkThreads, 2, 4, false>);
      default:
        CMI_TRY(config_kernel(c, k_walk32<kWalkThreads, 3, walk32_min_blocks<3>(), true>));
        return config_kernel(c, k_walk32<kWalkThreads, 3, walk32_min_blocks<3>(), false>);
    }
  }
  const size_t head = (sizeof(WalkShared) + 15) & ~(size_t)15;
  c->walk_smem = head + 24 * (size_t)c->max_padded;
  return config_kernel(c, k_walk64<kWalkThreads>);
}

EmitParams emit_params(cmi_context *c) {
  EmitParams e{};
  e.inst = c->d_inst;
  e.src = c->d_src;
  e.nsrc_total = c->nsrc_total;
  e.src_count = c->d_src_count;
  e.src_first = c->d_src_first;
  e.buf_first = c->d_buf_first;
  e.st = c->d_state;
  e.arena = c->d_arena_out;
  e.keys = c->d_keys;
  e.ranks = c->d_ranks;
  e.hist = c->d_hist;
  e.capacity = (uint32_t)c->capacity;
  e.src_rank0 = c->d_src_rank0;
  e.bucket_off = c->d_bucket_off;
  e.arena_sorted = c->d_arena_in;
  return e;
}

// Wavefront rounds once round 0 is planned: walk, then plan (+ scatter) the
// packets it passed on; the last plan counts what is left over (must be zero).
// Outside a graph the host reads the plan's chunk count and stops when no
// packet is left (the graph's round loop does the same on the device).
int enqueue_rounds(cmi_context *c) {
  for (int r = 0; r < c->round_cap; ++r) {
    uint32_t remaining = 0;
    CMI_CUDA(cudaMemcpyAsync(&remaining, &c->d_state->num_chunks, sizeof(uint32_t),
                             cudaMemcpyDeviceToHost, c->stream));
    CMI_CUDA(cudaStreamSynchronize(c->stream));
    if (remaining == 0u) break;
    CMI_TRY(timed_launch(c, 0, [&] { return launch_walk(c); }));
    CMI_TRY(timed_launch(c, 1, [&] { return launch_plan(c, true); }));
  }
  return CMI_OK;
}

// The rounds inside a captured iteration: a WHILE conditional node runs
// (walk -> plan -> scatter, whose first thread sets the condition) while
// packets remain, so an iteration stops after the rounds it needs instead of
// the worst-case count.  k_round_gate decides whether the first round runs.
int enqueue_rounds_graph(cmi_context *c) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t *deps = nullptr;
  size_t nd = 0;
  CMI_CUDA(cudaStreamGetCaptureInfo(c->stream, &cs, nullptr, &g, &deps, &nd));
  if (cs != cudaStreamCaptureStatusActive) return fail(CMI_ERR_CUDA, "stream is not capturing");
  cudaGraphConditionalHandle h;
  CMI_CUDA(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
  k_round_gate<<<1, 32, 0, c->stream>>>(c->d_state, h, (uint32_t)c->round_cap);
  c->enqueued += 1;
  CMI_CUDA(cudaGetLastError());
  CMI_CUDA(cudaStreamGetCaptureInfo(c->stream, &cs, nullptr, &g, &deps, &nd));
  cudaGraphNodeParams np = {};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  CMI_CUDA(cudaGraphAddNode(&node, g, deps, nd, &np));
  cudaGraph_t body = np.conditional.phGraph_out[0];
  CMI_CUDA(cudaStreamUpdateCaptureDependencies(c->stream, &node, 1,
                                               cudaStreamSetCaptureDependencies));
  // the loop body, captured on the second stream into the node's graph
  CMI_CUDA(cudaStreamBeginCaptureToGraph(c->body_stream, body, nullptr, nullptr, 0,
                                         cudaStreamCaptureModeThreadLocal));
  cudaStream_t outer = c->stream;
  const uint64_t before = c->enqueued;
  c->stream = c->body_stream;
  int rc = launch_walk(c);
  if (rc == CMI_OK) rc = launch_plan(c, true, true, h);
  c->stream = outer;
  cudaGraph_t captured = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(c->body_stream, &captured);
  if (rc != CMI_OK) return rc;
  if (ee != cudaSuccess)
    return fail(CMI_ERR_CUDA, "round loop capture: %s", cudaGetErrorString(ee));
  c->graph_body_kernels = c->enqueued - before;
  c->enqueued = before;  // body kernels are counted per executed round
  return CMI_OK;
}

int enqueue_iteration(cmi_context *c, bool balance) {
  const int ninst = (int)c->inst.size();
  k_begin_iteration<<<1, 128, 0, c->stream>>>(c->d_state, c->d_stats, ninst);
  // Philox packets are written straight into their sorted place: the
  // emission plan fills the round-0 histogram, the plan places the buckets
  const bool direct = c->opt.rng == CMI_RNG_PHILOX;
  k_emission_plan<<<1, 128, 0, c->stream>>>(c->d_inst, ninst, c->d_src, c->nsrc_total,
                                            c->d_state, c->d_src_count, c->d_src_first,
                                            c->d_buf_first, c->d_stats,
                                            direct ? c->d_src_rank0 : nullptr, c->d_hist);
  c->enqueued += 2;
  const EmitParams e = emit_params(c);
  const int egrid = c->num_sms * 8;
  if (direct) CMI_TRY(timed_launch(c, 1, [&] { return launch_plan(c, false); }));
  CMI_TRY(timed_launch(c, 2, [&] {
    if (c->opt.rng == CMI_RNG_RANLUX) {
      if (c->fp32()) k_emit_ranlux<kPk32><<<egrid, 128, 0, c->stream>>>(e);
      else if (c->mixed()) k_emit_ranlux<kPkM><<<egrid, 128, 0, c->stream>>>(e);
      else k_emit_ranlux<kPk64><<<egrid, 128, 0, c->stream>>>(e);
    } else {
      if (c->fp32()) k_emit_philox_direct<kPk32><<<egrid, 256, 0, c->stream>>>(e);
      else if (c->mixed()) k_emit_philox_direct<kPkM><<<egrid, 256, 0, c->stream>>>(e);
      else k_emit_philox_direct<kPk64><<<egrid, 256, 0, c->stream>>>(e);
    }
    return CMI_OK;
  }));
  c->enqueued += 1;
  CMI_CUDA(cudaGetLastError());
  if (!direct) CMI_TRY(timed_launch(c, 1, [&] { return launch_plan(c, true); }));
  // fields sent by cmi_set_fields_prefetched arrive on the copy stream: the
  // walk waits for them here, so their copy overlaps the emission above (a
  // graph holds this as an event-wait node on the latest record)
  CMI_CUDA(cudaStreamWaitEvent(c->stream, c->fields_ready,
                               c->capturing ? cudaEventWaitExternal : cudaEventWaitDefault));
  CMI_TRY(c->capturing ? enqueue_rounds_graph(c) : enqueue_rounds(c));
  if (balance) {
    BalanceParams b{};
    b.subs = c->d_sub;
    b.inst = c->d_inst;
    b.nH = c->d_nH;
    b.xH = c->d_xH;
    b.J = c->d_J;
    b.kappa = c->uses_kappa() ? c->d_kappa : nullptr;
    b.stats = c->d_stats;
    b.first_sub = 0;
    b.num_subs = c->S;
    b.jfac_override = -1.;
    CMI_TRY(timed_launch(c, 3, [&] {
      if (c->opt.balance_form == CMI_BALANCE_REFERENCE)
        k_balance<0><<<c->S, 256, 0, c->stream>>>(b);
      else
        k_balance<1><<<c->S, 256, 0, c->stream>>>(b);
      return CMI_OK;
    }));
    c->enqueued += 1;
  }
  k_end_iteration<<<1, 128, 0, c->stream>>>(c->d_state, c->d_stats, ninst, 1);
  c->enqueued += 1;
  CMI_CUDA(cudaGetLastError());
  return CMI_OK;
}

int validate_ready(cmi_context *c) {
  for (size_t i = 0; i < c->inst.size(); ++i) {
    if (c->inst[i].num_photon > 0 && c->inst[i].src_lum.empty())
      return fail(CMI_ERR_INVALID_ARGUMENT, "instance %zu has a packet budget but no sources", i);
  }
  return ensure_capacity(c, total_budget(c));
}

void to_stats(const DevStats &d, const HostInstance &I, cmi_stats &s) {
  s.packets_emitted = d.emitted;
  s.packets_absorbed = d.absorbed;
  s.packets_escaped = d.escaped;
  s.cell_crossings = d.crossings;
  s.subgrid_transits = d.transits;
  s.mean_abs_dx = (I.ncells > 0) ? d.dx_sum / (double)I.ncells : 0.;
  s.error_flags = d.flags;
  s.rounds = d.rounds;
  s.packets_reemitted = d.reemitted;
}

int ensure_host_stats(cmi_context *c, size_t n) {
  if (n <= c->h_stats_count) return CMI_OK;
  if (c->h_stats) cudaFreeHost(c->h_stats);
  c->h_stats = nullptr;
  CMI_CUDA(cudaMallocHost((void **)&c->h_stats, sizeof(DevStats) * n));
  c->h_stats_count = n;
  return CMI_OK;
}

int run(cmi_context *c, int32_t iterations, uint64_t seed, uint32_t first_iteration,
        bool balance, cmi_stats *stats) {
  CMI_TRY(validate_ready(c));
  const int ninst = (int)c->inst.size();
  CMI_TRY(ensure_host_stats(c, (size_t)iterations * ninst));
  const uint64_t hs[2] = {seed, 0};
  CMI_CUDA(cudaMemcpyAsync(&c->d_state->seed, hs, sizeof(uint64_t), cudaMemcpyHostToDevice,
                           c->stream));
  CMI_CUDA(cudaMemcpyAsync(&c->d_state->iteration, &first_iteration, sizeof(uint32_t),
                           cudaMemcpyHostToDevice, c->stream));
  c->last_launches = 0;
  const bool use_graph = c->opt.use_graph != 0 && !c->timing;
  const int gi = balance ? 1 : 0;
  if (use_graph && c->graph_dirty) free_graph(c);
  if (use_graph && !c->graph_exec[gi]) {
    cudaGraph_t g = nullptr;
    CMI_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    c->enqueued = 0;
    c->capturing = true;
    const int rc = enqueue_iteration(c, balance);
    c->capturing = false;
    const cudaError_t ec = cudaStreamEndCapture(c->stream, &g);
    if (rc != CMI_OK) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (ec != cudaSuccess) return fail(CMI_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ec));
    const cudaError_t ei = cudaGraphInstantiate(&c->graph_exec[gi], g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess)
      return fail(CMI_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ei));
    c->graph_kernels[gi] = c->enqueued;
    c->graph_dirty = false;
  }
  for (int32_t it = 0; it < iterations; ++it) {
    if (use_graph) {
      CMI_CUDA(cudaGraphLaunch(c->graph_exec[gi], c->stream));
      c->last_launches += c->graph_kernels[gi];
    } else {
      c->enqueued = 0;
      CMI_TRY(enqueue_iteration(c, balance));
      c->last_launches += c->enqueued;
    }
    CMI_CUDA(cudaMemcpyAsync(c->h_stats + (size_t)it * ninst, c->d_stats,
                             sizeof(DevStats) * ninst, cudaMemcpyDeviceToHost, c->stream));
    c->fields_pending = false;  // the iteration waited for the fields
  }
  CMI_CUDA(cudaStreamSynchronize(c->stream));
  uint32_t flags_any = 0;
  for (int32_t it = 0; it < iterations; ++it) {
    if (use_graph && ninst > 0) {  // the round loop ran once per round with packets
      const uint32_t r = std::min<uint32_t>(c->h_stats[(size_t)it * ninst].rounds,
                                            (uint32_t)c->round_cap);
      c->last_launches += c->graph_body_kernels * r;
    }
    for (int i = 0; i < ninst; ++i) {
      const DevStats &d = c->h_stats[(size_t)it * ninst + i];
      flags_any |= d.flags;
      if (stats) to_stats(d, c->inst[i], stats[(size_t)it * ninst + i]);
    }
  }
  if (flags_any & (kFlagArenaOverflow | kFlagLeftover))
    return fail(CMI_ERR_CAPACITY, "device queue overflow or packets left over (flags 0x%x)",
                flags_any);
  if (flags_any & kFlagStageTimeout)
    return fail(CMI_ERR_DEVICE_TIMEOUT, "shared-memory staging wait timed out (flags 0x%x)",
                flags_any);
  if (flags_any & (kFlagWalkLimit | kFlagBadInput))
    return fail(CMI_ERR_INVARIANT, "device invariant violated (flags 0x%x)", flags_any);
  return CMI_OK;
}

int clear_flags(cmi_context *c) {
  const uint32_t z = 0;
  CMI_CUDA(cudaMemcpyAsync(&c->d_state->flags, &z, sizeof(z), cudaMemcpyHostToDevice, c->stream));
  return CMI_OK;
}

}  // namespace

// ===========================================================================
// extern "C" ABI
// ===========================================================================
extern "C" {

int cmi_abi_version(void) { return CMI_ABI_VERSION; }

const char *cmi_last_error_string(void) { return g_last_error.c_str(); }

void cmi_default_options(cmi_options *o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->transport_precision = CMI_TRANSPORT_MIXED;
  o->balance_form = CMI_BALANCE_STABLE;
  o->rng = CMI_RNG_PHILOX;
  o->device = 0;
  o->threads_per_cta = 0;
  o->ctas_per_sm = 0;
  o->packets_per_chunk = 0;
  o->tally_mode = CMI_TALLY_FIXED64;
  o->use_graph = 1;
}

int cmi_create(const cmi_grid_desc *grids, int32_t num_instances, const cmi_options *options,
               cmi_context **out) {
  if (!out) return fail(CMI_ERR_INVALID_ARGUMENT, "null output pointer");
  *out = nullptr;
  if (!grids || num_instances <= 0) return fail(CMI_ERR_INVALID_ARGUMENT, "no grid given");
  cmi_options opt;
  if (options) opt = *options; else cmi_default_options(&opt);
  if (opt.transport_precision != CMI_TRANSPORT_FP32 && opt.transport_precision != CMI_TRANSPORT_FP64 &&
      opt.transport_precision != CMI_TRANSPORT_MIXED)
    return fail(CMI_ERR_INVALID_ARGUMENT, "unknown transport precision %d", opt.transport_precision);
  if (opt.balance_form != CMI_BALANCE_REFERENCE && opt.balance_form != CMI_BALANCE_STABLE)
    return fail(CMI_ERR_INVALID_ARGUMENT, "unknown balance form %d", opt.balance_form);
  if (opt.rng != CMI_RNG_PHILOX && opt.rng != CMI_RNG_RANLUX)
    return fail(CMI_ERR_INVALID_ARGUMENT, "unknown rng %d", opt.rng);
  if (opt.threads_per_cta != 0 && opt.threads_per_cta != kWalkThreads)
    return fail(CMI_ERR_NOT_SUPPORTED, "threads_per_cta must be 0 or %d", kWalkThreads);
  if (opt.packets_per_chunk < 0 || opt.packets_per_chunk > 4096 ||
      (opt.packets_per_chunk > 0 &&
       (opt.packets_per_chunk < 32 || (opt.packets_per_chunk & (opt.packets_per_chunk - 1)))))
    return fail(CMI_ERR_INVALID_ARGUMENT,
                "packets_per_chunk must be 0 or a power of two in [32, 4096]");
  if (opt.max_run_chunks < 0) return fail(CMI_ERR_INVALID_ARGUMENT, "negative max_run_chunks");
  if (opt.refill_lanes < 0 || opt.refill_lanes > 32)
    return fail(CMI_ERR_INVALID_ARGUMENT, "refill_lanes must be in [0, 32]");
  if (opt.tally_mode < CMI_TALLY_FP32 || opt.tally_mode > CMI_TALLY_FIXED64_ATOMIC64)
    return fail(CMI_ERR_INVALID_ARGUMENT, "unknown tally mode %d", opt.tally_mode);

  cmi_context *c = new (std::nothrow) cmi_context();
  if (!c) return fail(CMI_ERR_OUT_OF_MEMORY, "host allocation failed");
  c->opt = opt;
  c->device = opt.device;
  c->tables = make_direction_tables();
  c->chunk = opt.packets_per_chunk > 0 ? (uint32_t)opt.packets_per_chunk : 128u;
  auto bail = [&](int rc) {
    cmi_destroy(c);
    return rc;
  };
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    delete c;
    return fail(CMI_ERR_CUDA, "no CUDA device available");
  }
  if (c->device < 0 || c->device >= ndev) {
    const int dev = c->device;
    delete c;
    return fail(CMI_ERR_INVALID_ARGUMENT, "device %d out of range", dev);
  }
  if (cudaSetDevice(c->device) != cudaSuccess) {
    delete c;
    return fail(CMI_ERR_CUDA, "cudaSetDevice failed");
  }
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->body_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->fields_ready, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->main_mark, cudaEventDisableTiming) != cudaSuccess) {
    if (c->fields_ready) cudaEventDestroy(c->fields_ready);
    if (c->body_stream) cudaStreamDestroy(c->body_stream);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return fail(CMI_ERR_CUDA, "stream creation failed");
  }
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device);

  // ---- instances and the global subgrid table ----
  int64_t cell_off = 0;
  for (int32_t i = 0; i < num_instances; ++i) {
    const cmi_grid_desc &g = grids[i];
    HostInstance I;
    I.desc = g;
    for (int a = 0; a < 3; ++a) {
      if (g.ncell[a] <= 0 || g.num_subgrid[a] <= 0 || g.ncell[a] % g.num_subgrid[a] != 0)
        return bail(fail(CMI_ERR_INVALID_ARGUMENT,
                         "instance %d: ncell must be a positive multiple of num_subgrid", i));
      if (!(g.box[3 + a] > 0.))
        return bail(fail(CMI_ERR_INVALID_ARGUMENT, "instance %d: box sides must be > 0", i));
      I.sub_ncell[a] = g.ncell[a] / g.num_subgrid[a];
    }
    if (!(g.recombination_rate > 0.) || !(g.cross_section > 0.))
      return bail(fail(CMI_ERR_INVALID_ARGUMENT,
                       "instance %d: recombination rate and cross section must be > 0", i));
    I.cells_per_sub = I.sub_ncell[0] * I.sub_ncell[1] * I.sub_ncell[2];
    I.padded_per_sub = (I.cells_per_sub + 3) & ~3;
    if (I.padded_per_sub > 8192 || (opt.transport_precision == CMI_TRANSPORT_FP64 && I.padded_per_sub > 4096))
      return bail(fail(CMI_ERR_NOT_SUPPORTED,
                       "instance %d: %d cells per subgrid exceed the shared-memory limit "
                       "(4096 in FP64, 8192 in FP32 and mixed)",
                       i, I.cells_per_sub));
    I.first_sub = (uint32_t)c->h_sub.size();
    I.nsub = (uint32_t)g.num_subgrid[0] * g.num_subgrid[1] * g.num_subgrid[2];
    I.first_cell = cell_off;
    I.ncells = (int64_t)g.ncell[0] * g.ncell[1] * g.ncell[2];
    const double side[3] = {g.box[3] / g.num_subgrid[0], g.box[4] / g.num_subgrid[1],
                            g.box[5] / g.num_subgrid[2]};
    const int32_t *ns = g.num_subgrid;
    for (uint32_t s = 0; s < I.nsub; ++s) {
      const int ix = s / (ns[1] * ns[2]);
      const int iy = (s - ix * ns[1] * ns[2]) / ns[2];
      const int iz = s - ix * ns[1] * ns[2] - iy * ns[2];
      DevSubgrid S{};
      const int idx3[3] = {ix, iy, iz};
      for (int a = 0; a < 3; ++a) {
        // DensitySubGrid(box, ncell), testDensitySubGrid_omp.cpp:1822-1828
        S.anchor[a] = g.box[a] + idx3[a] * side[a];
        S.cell_size[a] = side[a] / I.sub_ncell[a];
        S.inv_cell_size[a] = I.sub_ncell[a] / side[a];
        S.cell_size_f[a] = (float)S.cell_size[a];
        S.ncell[a] = I.sub_ncell[a];
      }
      S.ncells = I.cells_per_sub;
      S.padded_cells = I.padded_per_sub;
      S.field_offset = cell_off;
      cell_off += I.padded_per_sub;
      S.instance = (uint32_t)i;
      for (int d = 0; d < kNumDirections; ++d) S.ngb[d] = kOutside;
      for (int nx = -1; nx < 2; ++nx)
        for (int ny = -1; ny < 2; ++ny)
          for (int nz = -1; nz < 2; ++nz) {
            const int cx = ix + nx, cy = iy + ny, cz = iz + nz;
            if (cx >= 0 && cx < ns[0] && cy >= 0 && cy < ns[1] && cz >= 0 && cz < ns[2])
              S.ngb[dir_from_signs(nx, ny, nz)] = I.first_sub + (uint32_t)((cx * ns[1] + cy) * ns[2] + cz);
          }
      c->h_sub.push_back(S);
    }
    c->max_padded = std::max(c->max_padded, I.padded_per_sub);
    c->max_faces = std::max(c->max_faces, I.sub_ncell[0] + I.sub_ncell[1] + I.sub_ncell[2] + 3);
    // a straight path visits at most ns[0] + ns[1] + ns[2] - 2 subgrids; a
    // packet whose position rounds exactly onto a face of a neighbouring
    // subgrid makes one extra transit that crosses no cell, hence the spares
    c->rounds = std::max(c->rounds, ns[0] + ns[1] + ns[2] - 2 + kSpareRounds);
    c->inst.push_back(I);
  }
  c->S = (uint32_t)c->h_sub.size();
  c->total_padded = cell_off;
  // default chunk: 256 packets for small subgrids (<= 1024 cells: a visit is a
  // few crossings, so claims and ring refills are a larger share of a packet's
  // cost; B200, stromgren64's 8^3 subgrids: 3.20e10 -> 3.63e10 crossings/s),
  // else 128 (16^3 subgrids: 128 beats 256 by 14% on lognormal128)
  if (opt.packets_per_chunk == 0 && c->max_padded <= 1024) c->chunk = 256u;
  c->ntiles = (c->S + kPlanTile - 1) / kPlanTile;

  int rc = CMI_OK;
  if ((rc = dev_alloc(&c->d_sub, c->S)) || (rc = dev_alloc(&c->d_inst, c->inst.size())) ||
      (rc = dev_alloc(&c->d_nH, c->total_padded)) || (rc = dev_alloc(&c->d_xH, c->total_padded)) ||
      (rc = dev_alloc(&c->d_J, c->total_padded)) ||
      (rc = dev_alloc(&c->d_kappa, c->uses_kappa() ? c->total_padded : 1)) ||
      (rc = dev_alloc(&c->d_state, 1)) || (rc = dev_alloc(&c->d_stats, c->inst.size())) ||
      (rc = dev_alloc(&c->d_hist, c->S)) || (rc = dev_alloc(&c->d_bucket_off, c->S)) ||
      (rc = dev_alloc(&c->d_tile_pk, c->ntiles)) || (rc = dev_alloc(&c->d_tile_ch, c->ntiles)) ||
      (rc = dev_alloc(&c->d_tile_pk_off, c->ntiles)) ||
      (rc = dev_alloc(&c->d_tile_ch_off, c->ntiles)) ||
      (rc = dev_alloc(&c->d_plan_choff, kPlanTile + 1)) ||
      (rc = dev_alloc(&c->d_plan_pkoff, kPlanTile + 1)))
    return bail(rc);
  if (cudaMemcpyAsync(c->d_sub, c->h_sub.data(), sizeof(DevSubgrid) * c->S,
                      cudaMemcpyHostToDevice, c->stream) != cudaSuccess ||
      cudaMemsetAsync(c->d_state, 0, sizeof(RoundState), c->stream) != cudaSuccess ||
      cudaMemsetAsync(c->d_hist, 0, sizeof(uint32_t) * c->S, c->stream) != cudaSuccess ||
      cudaMemsetAsync(c->d_J, 0, sizeof(double) * c->total_padded, c->stream) != cudaSuccess)
    return bail(fail(CMI_ERR_CUDA, "initial upload failed"));
  // reference initial state, DensitySubGrid.hpp:544-551
  k_fill<<<c->num_sms * 4, 256, 0, c->stream>>>(c->d_nH, 1.e8, c->total_padded);
  k_fill<<<c->num_sms * 4, 256, 0, c->stream>>>(c->d_xH, 1.e-6, c->total_padded);
  if (cudaGetLastError() != cudaSuccess) return bail(fail(CMI_ERR_CUDA, "initial fill failed"));
  if ((rc = upload_tables(c))) return bail(rc);
  for (int32_t i = 0; i < num_instances; ++i)
    if ((rc = refresh_kappa(c, i))) return bail(rc);
  if ((rc = config_walk(c))) return bail(rc);
  int64_t max_cells = 0;
  for (const auto &I : c->inst) max_cells = std::max(max_cells, I.ncells);
  if ((rc = ensure_stage(c, sizeof(double) * (size_t)max_cells))) return bail(rc);
  if ((rc = ensure_capacity(c, 1024))) return bail(rc);
  // pinned per-iteration statistics: allocated here, not inside a timed run
  if ((rc = ensure_host_stats(c, 256 * c->inst.size()))) return bail(rc);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess)
    return bail(fail(CMI_ERR_CUDA, "context set-up failed: %s",
                     cudaGetErrorString(cudaGetLastError())));
  *out = c;
  return CMI_OK;
}

int cmi_destroy(cmi_context *c) {
  if (!c) return CMI_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);  // a prefetch in flight
  free_graph(c);
  dev_free(c->d_sub);
  dev_free(c->d_inst);
  dev_free(c->d_src);
  dev_free(c->d_nH);
  dev_free(c->d_xH);
  dev_free(c->d_J);
  dev_free(c->d_kappa);
  dev_free(c->d_src_count);
  dev_free(c->d_src_first);
  dev_free(c->d_buf_first);
  dev_free(c->d_state);
  dev_free(c->d_stats);
  dev_free(c->d_hist);
  dev_free(c->d_bucket_off);
  dev_free(c->d_tile_pk);
  dev_free(c->d_tile_ch);
  dev_free(c->d_tile_pk_off);
  dev_free(c->d_tile_ch_off);
  dev_free(c->d_plan_choff);
  dev_free(c->d_plan_pkoff);
  dev_free(c->d_chunks);
  dev_free(c->d_arena_in);
  dev_free(c->d_arena_out);
  dev_free(c->d_keys);
  dev_free(c->d_ranks);
  dev_free(c->d_stage);
  free_dust_buffers(c->dust);
  c->dust = nullptr;
  if (c->h_stats) cudaFreeHost(c->h_stats);
  for (auto &t : c->timed) {
    cudaEventDestroy(t.start);
    cudaEventDestroy(t.stop);
  }
  for (cudaEvent_t e : c->event_pool) cudaEventDestroy(e);
  if (c->fields_ready) cudaEventDestroy(c->fields_ready);
  if (c->main_mark) cudaEventDestroy(c->main_mark);
  dev_free(c->d_nh_stage);
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  if (c->stream) cudaStreamDestroy(c->stream);
  if (c->body_stream) cudaStreamDestroy(c->body_stream);
  delete c;
  return CMI_OK;
}

static int copy_field_in(cmi_context *c, int32_t instance, int32_t layout, int32_t memory,
                         const double *src, double *dst, cudaStream_t s = nullptr) {
  const HostInstance &I = c->inst[instance];
  if (!s) s = c->stream;
  const double *dsrc = src;
  if (memory == CMI_MEMORY_HOST) {
    CMI_CUDA(cudaMemcpyAsync(c->d_stage, src, sizeof(double) * I.ncells, cudaMemcpyHostToDevice,
                             s));
    dsrc = c->d_stage;
  }
  LayoutParams lp{};
  lp.subs = c->d_sub;
  lp.first_sub = I.first_sub;
  for (int a = 0; a < 3; ++a) {
    lp.ns[a] = I.desc.num_subgrid[a];
    lp.ncell[a] = I.desc.ncell[a];
  }
  lp.layout = layout;
  k_fields_in<<<I.nsub, 256, 0, s>>>(lp, dsrc, dst);
  CMI_CUDA(cudaGetLastError());
  return CMI_OK;
}

static int copy_field_out(cmi_context *c, int32_t instance, int32_t layout, int32_t memory,
                          const double *src, double *dst) {
  const HostInstance &I = c->inst[instance];
  double *ddst = (memory == CMI_MEMORY_HOST) ? c->d_stage : dst;
  LayoutParams lp{};
  lp.subs = c->d_sub;
  lp.first_sub = I.first_sub;
  for (int a = 0; a < 3; ++a) {
    lp.ns[a] = I.desc.num_subgrid[a];
    lp.ncell[a] = I.desc.ncell[a];
  }
  lp.layout = layout;
  k_fields_out<<<I.nsub, 256, 0, c->stream>>>(lp, src, ddst);
  CMI_CUDA(cudaGetLastError());
  if (memory == CMI_MEMORY_HOST) {
    CMI_CUDA(cudaMemcpyAsync(dst, c->d_stage, sizeof(double) * I.ncells, cudaMemcpyDeviceToHost,
                             c->stream));
    CMI_CUDA(cudaStreamSynchronize(c->stream));
  }
  return CMI_OK;
}

static int check_layout(int32_t layout, int32_t memory) {
  if (layout != CMI_LAYOUT_BLOCKED && layout != CMI_LAYOUT_CUBE)
    return fail(CMI_ERR_INVALID_ARGUMENT, "unknown layout %d", layout);
  if (memory != CMI_MEMORY_HOST && memory != CMI_MEMORY_DEVICE)
    return fail(CMI_ERR_INVALID_ARGUMENT, "unknown memory kind %d", memory);
  return CMI_OK;
}

int cmi_set_fields(cmi_context *c, int32_t instance, int32_t layout, int32_t memory,
                   const double *nH, const double *xH) {
  CMI_TRY(check_ctx(c));
  CMI_TRY(check_instance(c, instance));
  CMI_TRY(check_layout(layout, memory));
  if (nH) CMI_TRY(copy_field_in(c, instance, layout, memory, nH, c->d_nH));
  if (xH) CMI_TRY(copy_field_in(c, instance, layout, memory, xH, c->d_xH));
  CMI_TRY(refresh_kappa(c, instance));
  CMI_CUDA(cudaStreamSynchronize(c->stream));
  return CMI_OK;
}

int cmi_prefetch_number_density(cmi_context *c, int32_t instance, int32_t layout,
                                const double *nH) {
  CMI_TRY(check_ctx(c));
  CMI_TRY(check_instance(c, instance));
  CMI_TRY(check_layout(layout, CMI_MEMORY_HOST));
  if (!nH) return fail(CMI_ERR_INVALID_ARGUMENT, "null density array");
  if (!c->copy_stream) {
    CMI_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    CMI_TRY(dev_alloc(&c->d_nh_stage, (size_t)c->total_padded));
    c->nh_layout.assign(c->inst.size(), -1);
  }
  if (c->nh_layout[instance] >= 0)
    return fail(CMI_ERR_INVALID_ARGUMENT,
                "instance %d: a prefetched density has not been consumed yet", instance);
  const HostInstance &I = c->inst[instance];
  CMI_CUDA(cudaMemcpyAsync(c->d_nh_stage + I.first_cell, nH, sizeof(double) * I.ncells,
                           cudaMemcpyHostToDevice, c->copy_stream));
  c->nh_layout[instance] = layout;
  return CMI_OK;
}

int cmi_set_fields_prefetched(cmi_context *c, int32_t instance, int32_t memory,
                              const double *xH) {
  CMI_TRY(check_ctx(c));
  CMI_TRY(check_instance(c, instance));
  if (c->nh_layout.empty() || c->nh_layout[instance] < 0)
    return fail(CMI_ERR_INVALID_ARGUMENT, "instance %d: no prefetched density", instance);
  const int32_t layout = c->nh_layout[instance];
  CMI_TRY(check_layout(layout, memory));
  const HostInstance &I = c->inst[instance];
  // on the copy stream, after the main stream's work so far (which may still
  // read the fields and the staging buffer) and after the n_H copy (FIFO)
  CMI_CUDA(cudaEventRecord(c->main_mark, c->stream));
  CMI_CUDA(cudaStreamWaitEvent(c->copy_stream, c->main_mark, 0));
  CMI_TRY(copy_field_in(c, instance, layout, CMI_MEMORY_DEVICE, c->d_nh_stage + I.first_cell,
                        c->d_nH, c->copy_stream));
  c->nh_layout[instance] = -1;
  if (xH) CMI_TRY(copy_field_in(c, instance, layout, memory, xH, c->d_xH, c->copy_stream));
  CMI_TRY(refresh_kappa(c, instance, c->copy_stream));
  CMI_CUDA(cudaEventRecord(c->fields_ready, c->copy_stream));
  c->fields_pending = true;
  return CMI_OK;
}

int cmi_get_fields(cmi_context *c, int32_t instance, int32_t layout, int32_t memory, double *xH,
                   double *J) {
  CMI_TRY(check_ctx(c));
  CMI_TRY(check_instance(c, instance));
  CMI_TRY(check_layout(layout, memory));
  if (xH) CMI_TRY(copy_field_out(c, instance, layout, memory, c->d_xH, xH));
  if (J) CMI_TRY(copy_field_out(c, instance, layout, memory, c->d_J, J));
  CMI_CUDA(cudaStreamSynchronize(c->stream));
  return CMI_OK;
}

int cmi_set_intensity(cmi_context *c, int32_t instance, int32_t layout, int32_t memory,
                      const double *J) {
  CMI_TRY(check_ctx(c));
  CMI_TRY(check_instance(c, instance));
  CMI_TRY(check_layout(layout, memory));
  if (!J) return fail(CMI_ERR_INVALID_ARGUMENT, "null intensity array");
  CMI_TRY(copy_field_in(c, instance, layout, memory, J, c->d_J));
  CMI_CUDA(cudaStreamSynchronize(c->stream));
  return CMI_OK;
}

int cmi_set_sources(cmi_context *c, int32_t instance, const double *positions,
                    const double *luminosities, int32_t n) {
  CMI_TRY(check_ctx(c));
  CMI_TRY(check_instance(c, instance));
  if (n < 0 || n > 64) return fail(CMI_ERR_INVALID_ARGUMENT, "0..64 sources per instance, got %d", n);
  if (n > 0 && (!positions || !luminosities))
    return fail(CMI_ERR_INVALID_ARGUMENT, "null source arrays");
  HostInstance &I = c->inst[instance];
  for (int32_t k = 0; k < n; ++k) {
    if (!(luminosities[k] > 0.) || !std::isfinite(luminosities[k]))
      return fail(CMI_ERR_INVALID_ARGUMENT, "source %d: luminosity must be finite and > 0", k);
    for (int a = 0; a < 3; ++a) {
      const double p = positions[3 * k + a];
      if (!(p >= I.desc.box[a] && p <= I.desc.box[a] + I.desc.box[3 + a]))
        return fail(CMI_ERR_INVALID_ARGUMENT, "source %d lies outside the box", k);
    }
  }
  I.src_pos.assign(positions, positions + 3 * n);
  I.src_lum.assign(luminosities, luminosities + n);
  return upload_tables(c);
}

int cmi_set_packet_budget(cmi_context *c, int32_t instance, uint64_t num_photon) {
  CMI_TRY(check_ctx(c));
  CMI_TRY(check_instance(c, instance));
  c->inst[instance].num_photon = num_photon;
  CMI_TRY(upload_tables(c));
  return ensure_capacity(c, total_budget(c));
}

int cmi_set_reemission_probability(cmi_context *c, int32_t instance, double probability) {
  CMI_TRY(check_ctx(c));
  CMI_TRY(check_instance(c, instance));
  if (!(probability >= 0. && probability < 1.))
    return fail(CMI_ERR_INVALID_ARGUMENT, "reemission probability must be in [0, 1)");
  c->inst[instance].reemission = probability;
  return upload_tables(c);
}

int cmi_run_iterations(cmi_context *c, int32_t iterations, uint64_t seed, cmi_stats *stats) {
  CMI_TRY(check_ctx(c, false));
  if (iterations <= 0) return fail(CMI_ERR_INVALID_ARGUMENT, "iterations must be > 0");
  CMI_TRY(clear_flags(c));
  // the first iteration index of this call continues from the previous call
  uint32_t it0 = 0;
  CMI_CUDA(cudaMemcpyAsync(&it0, &c->d_state->iteration, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                           c->stream));
  CMI_CUDA(cudaStreamSynchronize(c->stream));
  return run(c, iterations, seed, it0, true, stats);
}

static int set_frozen(cmi_context *c, int32_t i, uint32_t v) {
  CMI_CUDA(cudaMemcpyAsync(&c->d_inst[i].frozen, &v, sizeof(uint32_t), cudaMemcpyHostToDevice,
                           c->stream));
  return CMI_OK;
}

int cmi_run_until_converged(cmi_context *c, int32_t max_iterations, int32_t min_iterations,
                            double tolerance, uint64_t seed, cmi_stats *stats,
                            int32_t *iterations_done, int32_t *converged_at) {
  CMI_TRY(check_ctx(c, false));
  if (max_iterations <= 0) return fail(CMI_ERR_INVALID_ARGUMENT, "max_iterations must be > 0");
  if (min_iterations < 1 || min_iterations > max_iterations)
    return fail(CMI_ERR_INVALID_ARGUMENT, "min_iterations must be in [1, max_iterations]");
  if (!(tolerance >= 0.) || !std::isfinite(tolerance))
    return fail(CMI_ERR_INVALID_ARGUMENT, "tolerance must be finite and >= 0");
  const int ninst = (int)c->inst.size();
  std::vector<int32_t> at(ninst, 0);
  int remaining = ninst;
  CMI_TRY(clear_flags(c));
  uint32_t it0 = 0;
  CMI_CUDA(cudaMemcpyAsync(&it0, &c->d_state->iteration, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                           c->stream));
  CMI_CUDA(cudaStreamSynchronize(c->stream));
  std::vector<cmi_stats> st(ninst);
  int32_t done = 0;
  int rc = CMI_OK;
  while (done < max_iterations && remaining > 0) {
    // one iteration (graph replay); the host reads the per-instance change
    rc = run(c, 1, seed, it0 + (uint32_t)done, true, st.data());
    if (rc != CMI_OK) break;
    ++done;
    if (stats) std::copy(st.begin(), st.end(), stats + (size_t)(done - 1) * ninst);
    for (int i = 0; i < ninst && rc == CMI_OK; ++i) {
      if (at[i] != 0 || done < min_iterations || !(st[i].mean_abs_dx < tolerance)) continue;
      at[i] = done;
      --remaining;
      if (remaining > 0) rc = set_frozen(c, i, 1u);
    }
  }
  // leave every instance active for later calls
  for (int i = 0; i < ninst; ++i)
    if (at[i] != 0) {
      const int r = set_frozen(c, i, 0u);
      if (rc == CMI_OK) rc = r;
    }
  if (rc == CMI_OK) {
    const cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) rc = fail(CMI_ERR_CUDA, "unfreeze: %s", cudaGetErrorString(e));
  }
  if (iterations_done) *iterations_done = done;
  if (converged_at) std::copy(at.begin(), at.end(), converged_at);
  return rc;
}

int cmi_emit_photons(cmi_context *c, uint64_t seed, uint32_t iteration, cmi_photon *out,
                     uint64_t capacity, uint64_t *count) {
  CMI_TRY(check_ctx(c));
  if (!count) return fail(CMI_ERR_INVALID_ARGUMENT, "null count");
  *count = 0;
  for (size_t i = 0; i < c->inst.size(); ++i) {
    if (c->inst[i].num_photon > 0 && c->inst[i].src_lum.empty())
      return fail(CMI_ERR_INVALID_ARGUMENT, "instance %zu has a packet budget but no sources", i);
  }
  const uint64_t budget = total_budget(c);
  if (budget > 0xF0000000ull)
    return fail(CMI_ERR_CAPACITY, "%llu packets exceed the 32-bit packet index",
                (unsigned long long)budget);
  const uint64_t hs[2] = {seed, 0};
  CMI_CUDA(cudaMemcpyAsync(&c->d_state->seed, hs, sizeof(uint64_t), cudaMemcpyHostToDevice,
                           c->stream));
  CMI_CUDA(cudaMemcpyAsync(&c->d_state->iteration, &iteration, sizeof(uint32_t),
                           cudaMemcpyHostToDevice, c->stream));
  const int ninst = (int)c->inst.size();
  k_begin_iteration<<<1, 128, 0, c->stream>>>(c->d_state, c->d_stats, ninst);
  k_emission_plan<<<1, 128, 0, c->stream>>>(c->d_inst, ninst, c->d_src, c->nsrc_total,
                                            c->d_state, c->d_src_count, c->d_src_first,
                                            c->d_buf_first, c->d_stats, nullptr, c->d_hist);
  CMI_CUDA(cudaGetLastError());
  uint32_t emitted = 0;
  CMI_CUDA(cudaMemcpyAsync(&emitted, &c->d_state->emit_total, sizeof(uint32_t),
                           cudaMemcpyDeviceToHost, c->stream));
  CMI_CUDA(cudaStreamSynchronize(c->stream));
  *count = emitted;
  if (emitted == 0) return CMI_OK;
  if (!out || capacity < emitted)
    return fail(CMI_ERR_CAPACITY, "%u photons emitted, room for %llu", emitted,
                (unsigned long long)(out ? capacity : 0));
  CMI_TRY(ensure_stage(c, sizeof(Packet64) * (size_t)emitted));
  EmitParams e = emit_params(c);
  e.photons_out = reinterpret_cast<Packet64 *>(c->d_stage);
  const int egrid = c->num_sms * 8;
  if (c->opt.rng == CMI_RNG_RANLUX) k_emit_ranlux<kPk64, true><<<egrid, 128, 0, c->stream>>>(e);
  else k_emit_philox_direct<kPk64, true><<<egrid, 256, 0, c->stream>>>(e);
  CMI_CUDA(cudaGetLastError());
  CMI_CUDA(cudaMemcpyAsync(out, c->d_stage, sizeof(Packet64) * (size_t)emitted,
                           cudaMemcpyDeviceToHost, c->stream));
  CMI_CUDA(cudaStreamSynchronize(c->stream));
  return CMI_OK;
}

int cmi_shoot_packets(cmi_context *c, uint64_t seed, uint32_t iteration, cmi_stats *stats) {
  CMI_TRY(check_ctx(c, false));
  CMI_TRY(clear_flags(c));
  return run(c, 1, seed, iteration, false, stats);
}

int cmi_transport_packets(cmi_context *c, int32_t instance, const cmi_photon *packets,
                          const uint32_t *start_subgrid, uint64_t n, cmi_stats *stats) {
  CMI_TRY(check_ctx(c));
  CMI_TRY(check_instance(c, instance));
  if (n > 0 && (!packets || !start_subgrid))
    return fail(CMI_ERR_INVALID_ARGUMENT, "null packet arrays");
  CMI_TRY(clear_flags(c));
  CMI_TRY(ensure_capacity(c, std::max<uint64_t>(n, total_budget(c))));
  const size_t bytes = sizeof(Packet64) * n + sizeof(uint32_t) * n + 64;
  CMI_TRY(ensure_stage(c, bytes));
  Packet64 *d_ph = reinterpret_cast<Packet64 *>(c->d_stage);
  uint32_t *d_start = reinterpret_cast<uint32_t *>(
      reinterpret_cast<char *>(c->d_stage) + ((sizeof(Packet64) * n + 15) & ~(size_t)15));
  if (n > 0) {
    CMI_CUDA(cudaMemcpyAsync(d_ph, packets, sizeof(Packet64) * n, cudaMemcpyHostToDevice,
                             c->stream));
    CMI_CUDA(cudaMemcpyAsync(d_start, start_subgrid, sizeof(uint32_t) * n,
                             cudaMemcpyHostToDevice, c->stream));
  }
  const int ninst = (int)c->inst.size();
  k_begin_iteration<<<1, 128, 0, c->stream>>>(c->d_state, c->d_stats, ninst);
  const HostInstance &I = c->inst[instance];
  UploadParams u{};
  u.photons = d_ph;
  u.start = d_start;
  u.n = n;
  u.subs = c->d_sub;
  u.first_sub = I.first_sub;
  u.nsub = I.nsub;
  u.st = c->d_state;
  u.arena = c->d_arena_out;
  u.keys = c->d_keys;
  u.ranks = c->d_ranks;
  u.hist = c->d_hist;
  u.capacity = (uint32_t)c->capacity;
  const int grid = c->num_sms * 8;
  if (c->fp32()) k_upload<kPk32><<<grid, 256, 0, c->stream>>>(u);
  else if (c->mixed()) k_upload<kPkM><<<grid, 256, 0, c->stream>>>(u);
  else k_upload<kPk64><<<grid, 256, 0, c->stream>>>(u);
  CMI_CUDA(cudaGetLastError());
  c->enqueued = 0;
  CMI_TRY(launch_plan(c, true));
  CMI_TRY(enqueue_rounds(c));
  k_end_iteration<<<1, 128, 0, c->stream>>>(c->d_state, c->d_stats, ninst, 0);
  CMI_CUDA(cudaGetLastError());
  c->last_launches = c->enqueued + 3;
  CMI_TRY(ensure_host_stats(c, ninst));
  CMI_CUDA(cudaMemcpyAsync(c->h_stats, c->d_stats, sizeof(DevStats) * ninst,
                           cudaMemcpyDeviceToHost, c->stream));
  CMI_CUDA(cudaStreamSynchronize(c->stream));
  DevStats d = c->h_stats[instance];
  d.emitted = n;
  if (stats) to_stats(d, I, *stats);
  if (d.flags & (kFlagArenaOverflow | kFlagLeftover))
    return fail(CMI_ERR_CAPACITY, "device queue overflow or packets left over (flags 0x%x)",
                d.flags);
  if (d.flags & kFlagBadInput) return fail(CMI_ERR_INVALID_ARGUMENT, "start subgrid out of range");
  if (d.flags & kFlagStageTimeout) return fail(CMI_ERR_DEVICE_TIMEOUT, "staging wait timed out");
  if (d.flags & kFlagWalkLimit) return fail(CMI_ERR_INVARIANT, "walk step bound exceeded");
  return CMI_OK;
}

static int traverse(cmi_context *c, int32_t instance, uint32_t subgrid, int32_t input_direction,
                    const cmi_photon *in, uint32_t n, cmi_photon *out_grouped,
                    int32_t *out_dir_host, const uint8_t *enabled, uint32_t *out_count,
                    uint32_t *num_done, int32_t max_steps, int32_t *cells, double *lengths,
                    int32_t *num_steps) {
  CMI_TRY(check_ctx(c));
  CMI_TRY(check_instance(c, instance));
  const HostInstance &I = c->inst[instance];
  if (subgrid >= I.nsub)
    return fail(CMI_ERR_INVALID_ARGUMENT, "subgrid %u out of range [0, %u)", subgrid, I.nsub);
  if (input_direction < 0 || input_direction >= kNumDirections)
    return fail(CMI_ERR_INVALID_ARGUMENT, "input direction %d out of range", input_direction);
  if (n > 0 && !in) return fail(CMI_ERR_INVALID_ARGUMENT, "null input buffer");
  CMI_TRY(clear_flags(c));
  const size_t a16 = (sizeof(Packet64) * (size_t)n + 15) & ~(size_t)15;
  const size_t bytes = 2 * a16 + 16 * (size_t)n + 27 * 4 + 256 + 16 * (size_t)std::max(max_steps, 0);
  CMI_TRY(ensure_stage(c, bytes));
  char *base = reinterpret_cast<char *>(c->d_stage);
  Packet64 *d_in = reinterpret_cast<Packet64 *>(base);
  Packet64 *d_out = reinterpret_cast<Packet64 *>(base + a16);
  int32_t *d_dir = reinterpret_cast<int32_t *>(base + 2 * a16);
  char *tail = base + 2 * a16 + (((size_t)n * 4 + 15) & ~(size_t)15);
  uint32_t *d_counts = reinterpret_cast<uint32_t *>(tail);
  uint32_t *d_done = d_counts + 28;
  uint8_t *d_enabled = reinterpret_cast<uint8_t *>(d_counts + 32);
  int32_t *d_steps = reinterpret_cast<int32_t *>(d_counts + 48);
  int32_t *d_cells = reinterpret_cast<int32_t *>(d_counts + 64);
  double *d_len = reinterpret_cast<double *>(
      (reinterpret_cast<uintptr_t>(d_cells + std::max(max_steps, 1)) + 15) & ~(uintptr_t)15);
  if (n > 0)
    CMI_CUDA(cudaMemcpyAsync(d_in, in, sizeof(Packet64) * n, cudaMemcpyHostToDevice, c->stream));
  if (enabled)
    CMI_CUDA(cudaMemcpyAsync(d_enabled, enabled, 27, cudaMemcpyHostToDevice, c->stream));
  TraverseParams t{};
  t.subs = c->d_sub;
  t.inst = c->d_inst;
  t.sub = I.first_sub + subgrid;
  t.input_direction = input_direction;
  t.in = d_in;
  t.n = n;
  t.out = d_out;
  t.out_dir = d_dir;
  t.kappa = c->d_kappa;
  t.nH = c->d_nH;
  t.xH = c->d_xH;
  t.J = c->d_J;
  t.max_padded = c->max_padded;
  t.trace_cells = d_cells;
  t.trace_len = d_len;
  t.max_steps = max_steps;
  t.trace_steps = num_steps ? d_steps : nullptr;
  t.st = c->d_state;
  t.tables = c->tables;
  const size_t smem = (c->fp32() ? 12 : 24) * (size_t)c->max_padded +
                     (c->mixed() ? 8 * (size_t)c->max_faces : 0);
  if (n > 0) {
    const int grid = (int)((n + 255) / 256);
    if (c->fp32()) {
      CMI_CUDA(cudaFuncSetAttribute(k_traverse<kPk32>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      k_traverse<kPk32><<<grid, 256, smem, c->stream>>>(t);
    } else if (c->mixed()) {
      CMI_CUDA(cudaFuncSetAttribute(k_traverse<kPkM>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      k_traverse<kPkM><<<grid, 256, smem, c->stream>>>(t);
    } else {
      CMI_CUDA(cudaFuncSetAttribute(k_traverse<kPk64>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      k_traverse<kPk64><<<grid, 256, smem, c->stream>>>(t);
    }
    CMI_CUDA(cudaGetLastError());
  }
  if (out_grouped) {
    k_partition<<<1, 256, 0, c->stream>>>(d_out, d_dir, n, enabled ? d_enabled : nullptr,
                                          reinterpret_cast<Packet64 *>(d_in), d_counts, d_done);
    CMI_CUDA(cudaGetLastError());
  }
  uint32_t flags = 0;
  CMI_CUDA(cudaMemcpyAsync(&flags, &c->d_state->flags, sizeof(flags), cudaMemcpyDeviceToHost,
                           c->stream));
  uint32_t counts[28] = {0};
  if (out_grouped) {
    CMI_CUDA(cudaMemcpyAsync(counts, d_counts, sizeof(uint32_t) * 28, cudaMemcpyDeviceToHost,
                             c->stream));
  }
  if (out_dir_host && n > 0)
    CMI_CUDA(cudaMemcpyAsync(out_dir_host, d_dir, sizeof(int32_t) * n, cudaMemcpyDeviceToHost,
                             c->stream));
  int32_t steps = 0;
  if (num_steps)
    CMI_CUDA(cudaMemcpyAsync(&steps, d_steps, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  CMI_CUDA(cudaStreamSynchronize(c->stream));
  if (out_grouped) {
    uint32_t kept = 0;
    for (int d = 0; d < kNumDirections; ++d) {
      out_count[d] = counts[d];
      kept += counts[d];
    }
    uint32_t done = 0;
    CMI_CUDA(cudaMemcpy(&done, d_done, sizeof(done), cudaMemcpyDeviceToHost));
    if (num_done) *num_done = done;
    if (kept > 0)
      CMI_CUDA(cudaMemcpy(out_grouped, d_in, sizeof(Packet64) * kept, cudaMemcpyDeviceToHost));
  } else if (n > 0 && out_dir_host) {
    // single packet trace: photon comes back in place of the input
    CMI_CUDA(cudaMemcpy(const_cast<cmi_photon *>(in), d_out, sizeof(Packet64) * n,
                        cudaMemcpyDeviceToHost));
  }
  if (num_steps) {
    *num_steps = steps;
    const int32_t k = std::min(steps, max_steps);
    if (k > 0) {
      CMI_CUDA(cudaMemcpy(cells, d_cells, sizeof(int32_t) * k, cudaMemcpyDeviceToHost));
      CMI_CUDA(cudaMemcpy(lengths, d_len, sizeof(double) * k, cudaMemcpyDeviceToHost));
    }
  }
  if (flags & kFlagWalkLimit) return fail(CMI_ERR_INVARIANT, "walk step bound exceeded");
  return CMI_OK;
}

int cmi_traverse_buffer(cmi_context *c, int32_t instance, uint32_t subgrid,
                        int32_t input_direction, const cmi_photon *in, uint32_t n,
                        const uint8_t *enabled, cmi_photon *out, uint32_t out_count[27],
                        uint32_t *num_done) {
  if (!out || !out_count) return fail(CMI_ERR_INVALID_ARGUMENT, "null output buffers");
  return traverse(c, instance, subgrid, input_direction, in, n, out, nullptr, enabled,
                  out_count, num_done, 0, nullptr, nullptr, nullptr);
}

int cmi_trace_packet(cmi_context *c, int32_t instance, uint32_t subgrid, int32_t input_direction,
                     cmi_photon *photon, int32_t max_steps, int32_t *cells, double *lengths,
                     int32_t *num_steps, int32_t *output_direction) {
  if (!photon || !num_steps || !output_direction)
    return fail(CMI_ERR_INVALID_ARGUMENT, "null photon or outputs");
  if (max_steps < 0 || (max_steps > 0 && (!cells || !lengths)))
    return fail(CMI_ERR_INVALID_ARGUMENT, "bad trace arrays");
  return traverse(c, instance, subgrid, input_direction, photon, 1, nullptr, output_direction,
                  nullptr, nullptr, nullptr, max_steps, cells, lengths, num_steps);
}

int cmi_compute_neutral_fraction_subgrids(cmi_context *c, int32_t instance,
                                          uint32_t first_subgrid, uint32_t count,
                                          double luminosity, uint64_t num_photon,
                                          double *mean_abs_dx) {
  CMI_TRY(check_ctx(c));
  CMI_TRY(check_instance(c, instance));
  if (num_photon == 0) return fail(CMI_ERR_INVALID_ARGUMENT, "num_photon must be > 0");
  const HostInstance &I = c->inst[instance];
  if (count == 0 || first_subgrid >= I.nsub || count > I.nsub - first_subgrid)
    return fail(CMI_ERR_INVALID_ARGUMENT, "subgrid range [%u, %u + %u) outside [0, %u)",
                first_subgrid, first_subgrid, count, I.nsub);
  const double inv[3] = {I.sub_ncell[0] / (I.desc.box[3] / I.desc.num_subgrid[0]),
                         I.sub_ncell[1] / (I.desc.box[4] / I.desc.num_subgrid[1]),
                         I.sub_ncell[2] / (I.desc.box[5] / I.desc.num_subgrid[2])};
  // DensitySubGrid.hpp:1633 (num_photon is an unsigned int there)
  const double jfac = luminosity / (double)num_photon * inv[0] * inv[1] * inv[2];
  const int ninst = (int)c->inst.size();
  k_begin_iteration<<<1, 128, 0, c->stream>>>(c->d_state, c->d_stats, ninst);
  BalanceParams b{};
  b.subs = c->d_sub;
  b.inst = c->d_inst;
  b.nH = c->d_nH;
  b.xH = c->d_xH;
  b.J = c->d_J;
  b.kappa = c->uses_kappa() ? c->d_kappa : nullptr;
  b.stats = c->d_stats;
  b.first_sub = I.first_sub + first_subgrid;
  b.num_subs = count;
  b.jfac_override = jfac;
  if (c->opt.balance_form == CMI_BALANCE_REFERENCE)
    k_balance<0><<<count, 256, 0, c->stream>>>(b);
  else
    k_balance<1><<<count, 256, 0, c->stream>>>(b);
  CMI_CUDA(cudaGetLastError());
  DevStats d{};
  CMI_CUDA(cudaMemcpyAsync(&d, c->d_stats + instance, sizeof(DevStats), cudaMemcpyDeviceToHost,
                           c->stream));
  CMI_CUDA(cudaStreamSynchronize(c->stream));
  if (mean_abs_dx) *mean_abs_dx = d.dx_sum / ((double)count * (double)I.cells_per_sub);
  return CMI_OK;
}

int cmi_compute_neutral_fraction(cmi_context *c, int32_t instance, double luminosity,
                                 uint64_t num_photon, double *mean_abs_dx) {
  CMI_TRY(check_ctx(c));
  CMI_TRY(check_instance(c, instance));
  return cmi_compute_neutral_fraction_subgrids(c, instance, 0, c->inst[instance].nsub,
                                               luminosity, num_photon, mean_abs_dx);
}

int cmi_device_field(cmi_context *c, int32_t instance, int32_t which, double **ptr,
                     uint64_t *count) {
  CMI_TRY(check_ctx(c));
  CMI_TRY(check_instance(c, instance));
  if (!ptr || !count) return fail(CMI_ERR_INVALID_ARGUMENT, "null output");
  const HostInstance &I = c->inst[instance];
  double *base = (which == 0) ? c->d_J : (which == 1) ? c->d_xH : (which == 2) ? c->d_nH : nullptr;
  if (!base) return fail(CMI_ERR_INVALID_ARGUMENT, "which must be 0 (J), 1 (x_H) or 2 (n_H)");
  // the caller may read the array on any stream: the fields are settled first
  CMI_CUDA(cudaStreamSynchronize(c->stream));
  *ptr = base + I.first_cell;
  *count = (uint64_t)I.nsub * (uint64_t)I.padded_per_sub;
  return CMI_OK;
}

int cmi_get_stream(cmi_context *c, void **s) {
  if (!s) return fail(CMI_ERR_INVALID_ARGUMENT, "null argument");
  CMI_TRY(check_ctx(c));  // work queued on the stream comes after the fields
  *s = (void *)c->stream;
  return CMI_OK;
}

int cmi_synchronize(cmi_context *c) {
  CMI_TRY(check_ctx(c));
  CMI_CUDA(cudaStreamSynchronize(c->stream));
  return CMI_OK;
}

int cmi_set_kernel_timing(cmi_context *c, int32_t enable) {
  CMI_TRY(check_ctx(c));
  c->timing = enable != 0;
  return CMI_OK;
}

int cmi_kernel_timing(cmi_context *c, double ms[CMI_KERNEL_CLASSES],
                      uint64_t launches[CMI_KERNEL_CLASSES]) {
  CMI_TRY(check_ctx(c));
  if (!ms || !launches) return fail(CMI_ERR_INVALID_ARGUMENT, "null output");
  CMI_CUDA(cudaStreamSynchronize(c->stream));
  for (int k = 0; k < CMI_KERNEL_CLASSES; ++k) {
    ms[k] = 0.;
    launches[k] = 0;
  }
  for (auto &t : c->timed) {
    float v = 0.f;
    CMI_CUDA(cudaEventElapsedTime(&v, t.start, t.stop));
    ms[t.cls] += v;
    launches[t.cls] += (t.cls == 1) ? ((c->ntiles == 1) ? 2 : 4) : 1;
    c->event_pool.push_back(t.start);
    c->event_pool.push_back(t.stop);
  }
  c->timed.clear();
  return CMI_OK;
}

int cmi_last_launch_count(cmi_context *c, uint64_t *launches) {
  if (!c || !launches) return fail(CMI_ERR_INVALID_ARGUMENT, "null argument");
  *launches = c->last_launches;
  return CMI_OK;
}

}  // extern "C"

// ===========================================================================
// Dust scattering with peel-off image (cmi_dust_run; cmi_dust.cuh)
// ===========================================================================
// device buffers of cmi_dust_run, kept by the context between calls
struct DustBuffers {
  Packet64 *pk[2] = {nullptr, nullptr}, *peel = nullptr;
  uint32_t *sub[2] = {nullptr, nullptr}, *id[2] = {nullptr, nullptr}, *gen[2] = {nullptr, nullptr};
  uint32_t *peel_sub = nullptr, *counts = nullptr;
  int32_t *status = nullptr;
  unsigned long long *counters = nullptr;
  double *image = nullptr;
  ~DustBuffers() {
    for (int k = 0; k < 2; ++k) {
      cudaFree(pk[k]);
      cudaFree(sub[k]);
      cudaFree(id[k]);
      cudaFree(gen[k]);
    }
    cudaFree(peel);
    cudaFree(peel_sub);
    cudaFree(counts);
    cudaFree(status);
    cudaFree(counters);
    cudaFree(image);
  }
};

void free_dust_buffers(DustBuffers *b) { delete b; }

namespace {

unsigned dust_blocks(uint64_t n, int threads) {
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + threads - 1) / threads, 148 * 32));
}

}  // namespace

extern "C" int cmi_walk_photons(cmi_context *c, int32_t instance, uint32_t subgrid,
                                int32_t mode, cmi_photon *photons,
                                const int32_t *input_directions, uint32_t n,
                                int32_t *output_directions) {
  CMI_TRY(check_ctx(c));
  CMI_TRY(check_instance(c, instance));
  const HostInstance &I = c->inst[instance];
  if (subgrid >= I.nsub)
    return fail(CMI_ERR_INVALID_ARGUMENT, "subgrid %u out of range [0, %u)", subgrid, I.nsub);
  if (mode != CMI_WALK_PROPAGATE && mode != CMI_WALK_OPTICAL_DEPTH)
    return fail(CMI_ERR_INVALID_ARGUMENT, "mode must be CMI_WALK_PROPAGATE or "
                                          "CMI_WALK_OPTICAL_DEPTH");
  if (n == 0) return CMI_OK;
  if (!photons || !input_directions || !output_directions)
    return fail(CMI_ERR_INVALID_ARGUMENT, "null argument");
  for (uint32_t i = 0; i < n; ++i)
    if (input_directions[i] < 0 || input_directions[i] >= kNumDirections)
      return fail(CMI_ERR_INVALID_ARGUMENT, "input direction %d out of range",
                  input_directions[i]);
  const size_t pk_bytes = (sizeof(Packet64) * (size_t)n + 255) & ~(size_t)255;
  CMI_TRY(ensure_stage(c, pk_bytes + 2 * sizeof(int32_t) * (size_t)n + 256));
  char *base = reinterpret_cast<char *>(c->d_stage);
  Packet64 *d_pk = reinterpret_cast<Packet64 *>(base);
  int32_t *d_in = reinterpret_cast<int32_t *>(base + pk_bytes);
  int32_t *d_out = d_in + n;
  CMI_CUDA(cudaMemcpyAsync(d_pk, photons, sizeof(Packet64) * n, cudaMemcpyHostToDevice,
                           c->stream));
  CMI_CUDA(cudaMemcpyAsync(d_in, input_directions, sizeof(int32_t) * n, cudaMemcpyHostToDevice,
                           c->stream));
  const unsigned grid = (n + 127) / 128;
  if (mode == CMI_WALK_PROPAGATE)
    k_walk_photons<kPropagate><<<grid, 128, 0, c->stream>>>(
        c->d_sub, I.first_sub + subgrid, c->d_nH, c->d_xH, c->tables, d_pk, d_in, n, d_out);
  else
    k_walk_photons<kDepth><<<grid, 128, 0, c->stream>>>(
        c->d_sub, I.first_sub + subgrid, c->d_nH, c->d_xH, c->tables, d_pk, d_in, n, d_out);
  CMI_CUDA(cudaGetLastError());
  CMI_CUDA(cudaMemcpyAsync(photons, d_pk, sizeof(Packet64) * n, cudaMemcpyDeviceToHost,
                           c->stream));
  CMI_CUDA(cudaMemcpyAsync(output_directions, d_out, sizeof(int32_t) * n,
                           cudaMemcpyDeviceToHost, c->stream));
  CMI_CUDA(cudaStreamSynchronize(c->stream));
  for (uint32_t i = 0; i < n; ++i)
    if (output_directions[i] < 0)
      return fail(CMI_ERR_INVARIANT, "photon %u: walk step bound exceeded", i);
  return CMI_OK;
}

extern "C" int cmi_dust_run(cmi_context *c, int32_t instance, uint64_t num_photon, uint64_t seed,
                            uint32_t iteration, double albedo, const double source[3],
                            int32_t npix_x, int32_t npix_y, double *image,
                            cmi_dust_stats *stats) {
  CMI_TRY(check_ctx(c));
  CMI_TRY(check_instance(c, instance));
  if (num_photon == 0 || num_photon > (1ull << 30))
    return fail(CMI_ERR_INVALID_ARGUMENT, "num_photon must be in [1, 2^30]");
  if (!(albedo >= 0. && albedo < 1.))
    return fail(CMI_ERR_INVALID_ARGUMENT, "albedo must be in [0, 1)");
  if (npix_x < 1 || npix_y < 1 || npix_x > 65536 || npix_y > 65536 ||
      (int64_t)npix_x * npix_y > (1ll << 26))
    return fail(CMI_ERR_INVALID_ARGUMENT, "image size out of range");
  if (!source || !image) return fail(CMI_ERR_INVALID_ARGUMENT, "null argument");
  const HostInstance &I = c->inst[instance];
  const double *box = I.desc.box;
  // Source::get_subgrid_index: the subgrid holding the source
  int si[3];
  for (int a = 0; a < 3; ++a) {
    if (!(source[a] >= box[a] && source[a] <= box[a] + box[3 + a]))
      return fail(CMI_ERR_INVALID_ARGUMENT, "the source lies outside the box");
    si[a] = (int)((source[a] - box[a]) / box[3 + a] * I.desc.num_subgrid[a]);
    si[a] = std::min(si[a], I.desc.num_subgrid[a] - 1);
  }
  const uint32_t n = (uint32_t)num_photon;
  const size_t npix = (size_t)npix_x * npix_y;
  // the buffers grow to the largest call and stay with the context (about
  // 290 bytes per packet); a failed allocation leaves no buffers behind
  if (!c->dust || c->dust_capacity < n || c->dust_pixels < npix) {
    CMI_CUDA(cudaStreamSynchronize(c->stream));
    free_dust_buffers(c->dust);
    c->dust = nullptr;
    c->dust_capacity = 0;
    c->dust_pixels = 0;
    DustBuffers *nb = new DustBuffers();
    const uint64_t cap = std::max<uint64_t>(n, 1024);
    const size_t pix = std::max<size_t>(npix, 101 * 101);
    int rc = CMI_OK;
    for (int k = 0; k < 2; ++k) {
      if (rc == CMI_OK) rc = dev_alloc(&nb->pk[k], cap);
      if (rc == CMI_OK) rc = dev_alloc(&nb->sub[k], cap);
      if (rc == CMI_OK) rc = dev_alloc(&nb->id[k], cap);
      if (rc == CMI_OK) rc = dev_alloc(&nb->gen[k], cap);
    }
    if (rc == CMI_OK) rc = dev_alloc(&nb->peel, cap);
    if (rc == CMI_OK) rc = dev_alloc(&nb->peel_sub, cap);
    if (rc == CMI_OK) rc = dev_alloc(&nb->status, cap);
    if (rc == CMI_OK) rc = dev_alloc(&nb->counts, 4);
    if (rc == CMI_OK) rc = dev_alloc(&nb->counters, 8);
    if (rc == CMI_OK) rc = dev_alloc(&nb->image, pix);
    if (rc != CMI_OK) {
      free_dust_buffers(nb);
      return rc;
    }
    c->dust = nb;
    c->dust_capacity = cap;
    c->dust_pixels = pix;
  }
  DustBuffers &B = *c->dust;
  cudaStream_t st = c->stream;
  CMI_CUDA(cudaMemsetAsync(B.counters, 0, sizeof(unsigned long long) * 8, st));
  CMI_CUDA(cudaMemsetAsync(B.image, 0, sizeof(double) * npix, st));
  // counts: [0] live packets of pass 0, [1] of pass 1
  const uint32_t counts0[4] = {n, 0u, 0u, 0u};
  CMI_CUDA(cudaMemcpyAsync(B.counts, counts0, sizeof(counts0), cudaMemcpyHostToDevice, st));

  DustParams p{};
  p.subs = c->d_sub;
  p.nH = c->d_nH;
  p.xH = c->d_xH;
  p.tables = c->tables;
  p.status = B.status;
  p.seed = seed;
  p.instance = (uint32_t)instance;
  p.iteration = iteration;
  for (int a = 0; a < 3; ++a) p.src[a] = source[a];
  p.src_sub = I.first_sub + (uint32_t)((si[0] * I.desc.num_subgrid[1] + si[1]) *
                                           I.desc.num_subgrid[2] + si[2]);
  p.counters = B.counters;
  auto pass = [&](int k) {
    p.pk = B.pk[k];
    p.sub = B.sub[k];
    p.id = B.id[k];
    p.gen = B.gen[k];
    p.count = B.counts + k;
  };
  const unsigned wb = dust_blocks(n, 128);
  // 1. TAU packets to the box edge, 2. forced-scattering relaunch
  pass(0);
  k_dust_emit<<<dust_blocks(n, 256), 256, 0, st>>>(p, n);
  k_dust_walk<kDepth><<<wb, 128, 0, st>>>(p);
  k_dust_relaunch<<<dust_blocks(n, 256), 256, 0, st>>>(p);
  CMI_CUDA(cudaGetLastError());
  uint32_t generations = 0;
  int cur = 0;
  for (uint32_t g = 0; g < 4096u; ++g) {
    // 3. DIRECT packets to absorption or out of the box
    pass(cur);
    k_dust_walk<kPropagate><<<wb, 128, 0, st>>>(p);
    // 4. scattering + peel-off copies into the other pass
    CMI_CUDA(cudaMemsetAsync(B.counts + (1 - cur), 0, sizeof(uint32_t), st));
    DustScatterParams q{};
    q.pk = B.pk[cur];
    q.sub = B.sub[cur];
    q.id = B.id[cur];
    q.gen = B.gen[cur];
    q.status = B.status;
    q.count = B.counts + cur;
    q.out_pk = B.pk[1 - cur];
    q.out_sub = B.sub[1 - cur];
    q.out_id = B.id[1 - cur];
    q.out_gen = B.gen[1 - cur];
    q.peel_pk = B.peel;
    q.peel_sub = B.peel_sub;
    q.out_count = B.counts + (1 - cur);
    q.seed = seed;
    q.instance = (uint32_t)instance;
    q.iteration = iteration;
    q.albedo = albedo;
    q.counters = B.counters;
    k_dust_scatter<<<dust_blocks(n, 256), 256, 0, st>>>(q);
    ++generations;
    uint32_t m = 0;
    CMI_CUDA(cudaMemcpyAsync(&m, B.counts + (1 - cur), sizeof(uint32_t), cudaMemcpyDeviceToHost,
                             st));
    CMI_CUDA(cudaStreamSynchronize(st));
    if (m == 0u) break;
    // peel-offs (one per scattered packet) to the box edge, into the image
    DustParams pp = p;
    pp.pk = B.peel;
    pp.sub = B.peel_sub;
    pp.id = nullptr;
    pp.gen = nullptr;
    pp.count = B.counts + (1 - cur);
    k_dust_walk<kDepth><<<dust_blocks(m, 128), 128, 0, st>>>(pp);
    k_dust_image<<<dust_blocks(m, 256), 256, 0, st>>>(B.peel, B.status, B.counts + (1 - cur),
                                                      box[0], box[3], box[1], box[4], npix_x,
                                                      npix_y, B.image, B.counters + 6);
    CMI_CUDA(cudaGetLastError());
    cur = 1 - cur;
  }
  std::vector<double> img(npix);
  unsigned long long ctr[8];
  CMI_CUDA(cudaMemcpyAsync(img.data(), B.image, sizeof(double) * npix, cudaMemcpyDeviceToHost, st));
  CMI_CUDA(cudaMemcpyAsync(ctr, B.counters, sizeof(ctr), cudaMemcpyDeviceToHost, st));
  CMI_CUDA(cudaStreamSynchronize(st));
  // the driver's image.dat holds the sums divided by the packet count
  for (size_t k = 0; k < npix; ++k) image[k] = img[k] / (double)num_photon;
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->emitted = num_photon;
    stats->cell_crossings = ctr[0];
    stats->subgrid_transits = ctr[1];
    stats->absorbed = ctr[3];
    stats->escaped = ctr[4];
    stats->scatterings = ctr[5];
    stats->peeloffs_off_image = ctr[6];
    stats->generations = generations;
    stats->error_flags = ctr[2] ? (uint32_t)kFlagWalkLimit : 0u;
  }
  if (ctr[2]) return fail(CMI_ERR_INVARIANT, "dust walk: step or visit bound exceeded");
  return CMI_OK;
}

// ===========================================================================
// Allocation-free buffer traversal (cmi_traverse_buffer_noalloc)
// ===========================================================================
namespace {

// Layout of the fixed device array: walked photons, their exit directions,
// the 27 output flags and an error word.
constexpr size_t kNoAllocPhotonBytes = sizeof(Packet64) * CMI_NOALLOC_MAX_PHOTONS;
constexpr size_t kNoAllocDirOffset = kNoAllocPhotonBytes;
constexpr size_t kNoAllocFlagsOffset = kNoAllocDirOffset + sizeof(int32_t) * CMI_NOALLOC_MAX_PHOTONS;
constexpr size_t kNoAllocErrOffset = kNoAllocFlagsOffset + 32;
constexpr size_t kNoAllocBytes = kNoAllocErrOffset + 256;

}  // namespace

// The one scratch array of the allocation-free entry point.  In host code
// this name is only a handle: its device address comes from
// cudaGetSymbolAddress (see noalloc_scratch below).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

namespace {

std::mutex g_noalloc_mutex;
constexpr int kNoAllocMaxDevices = 64;
unsigned char *g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once
// per device with that device current.
int noalloc_scratch(unsigned char **out) {
  int dev = -1;
  CMI_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices)
    return fail(CMI_ERR_NOT_SUPPORTED, "device %d beyond the supported %d", dev,
                kNoAllocMaxDevices);
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(CMI_ERR_CUDA, "cudaGetSymbolAddress of the traversal scratch failed: %s",
                  cudaGetErrorString(e));
    g_noalloc_ptr[dev] = static_cast<unsigned char *>(p);
  }
  *out = g_noalloc_ptr[dev];
  return CMI_OK;
}

struct NoAllocParams {
  DevSubgrid sub;  // geometry by value: no device-side subgrid table
  uint8_t enabled[32];
  uint8_t *enabled_out;  // flags for k_partition, written by block 0
  int32_t input_direction;
  const Packet64 *in;
  uint32_t n;
  const double *nH, *xH;
  double *J;
  Packet64 *walked;
  int32_t *dir;
  uint32_t *err;
  DirectionTables tables;
};

// The reference FP64 walk of every photon through one subgrid (one photon
// per thread), fields staged in shared memory, tallies flushed to J.
__global__ void __launch_bounds__(256) k_traverse_noalloc(NoAllocParams prm) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ DirectionTables tab;
  const DevSubgrid &S = prm.sub;
  const int P = S.padded_cells;
  double *s_n = reinterpret_cast<double *>(smem_raw);
  double *s_x = s_n + P;
  double *s_J = s_x + P;
  if (threadIdx.x < sizeof(DirectionTables) / 4) {
    reinterpret_cast<uint32_t *>(&tab)[threadIdx.x] =
        reinterpret_cast<const uint32_t *>(&prm.tables)[threadIdx.x];
  }
  if (blockIdx.x == 0 && threadIdx.x < 32) prm.enabled_out[threadIdx.x] = prm.enabled[threadIdx.x];
  for (int c = threadIdx.x; c < S.ncells; c += blockDim.x) {
    s_n[c] = prm.nH[c];
    s_x[c] = prm.xH[c];
    s_J[c] = 0.;
  }
  __syncthreads();
  View64 v;
  for (int a = 0; a < 3; ++a) {
    v.n[a] = S.ncell[a];
    v.anchor[a] = S.anchor[a];
    v.cs[a] = S.cell_size[a];
    v.inv_cs[a] = S.inv_cell_size[a];
  }
  v.nyz = S.ncell[1] * S.ncell[2];
  v.nH = s_n;
  v.xH = s_x;
  v.J = s_J;
  const int limit = S.ncell[0] + S.ncell[1] + S.ncell[2] + 3;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < prm.n) {
    Packet64 ph = prm.in[i];
    ph.meta = (uint32_t)prm.input_direction;
    Walk64 w;
    int status = w.begin(ph, v, tab.sign_code);
    while (status == kRun) {
      status = w.step(v);
      if (status == kRun && w.steps > limit) status = kDrop;
    }
    int result = kInside;
    ph = w.packet(v, 0u);
    if (status == kExited) result = tab.mask_dir[w.exit_mask(v)];
    if (status == kDrop || result >= kNumDirections) {
      atomicOr(prm.err, kFlagWalkLimit);
      result = kInside;
    }
    ph.meta = 0u;
    prm.walked[i] = ph;
    prm.dir[i] = result;
  }
  __syncthreads();
  for (int c = threadIdx.x; c < S.ncells; c += blockDim.x) {
    if (s_J[c] != 0.) atomicAdd(&prm.J[c], s_J[c]);
  }
}

}  // namespace

extern "C" int cmi_traverse_buffer_noalloc(const double box[6], const int32_t ncell[3],
                                           const double *d_nH, const double *d_xH, double *d_J,
                                           int32_t input_direction, const cmi_photon *d_in,
                                           uint32_t n, const uint8_t *output_enabled,
                                           cmi_photon *d_out, uint32_t *d_out_count,
                                           uint32_t *d_num_done, void *stream) {
  if (!box || !ncell || !d_nH || !d_xH || !d_J || !d_out_count || !d_num_done)
    return fail(CMI_ERR_INVALID_ARGUMENT, "null argument");
  if (n > 0 && (!d_in || !d_out)) return fail(CMI_ERR_INVALID_ARGUMENT, "null photon buffer");
  if (n > CMI_NOALLOC_MAX_PHOTONS)
    return fail(CMI_ERR_CAPACITY,
                "%u photons exceed the allocation-free scratch of %d photons; split the "
                "buffer or use cmi_traverse_buffer",
                n, CMI_NOALLOC_MAX_PHOTONS);
  if (input_direction < 0 || input_direction >= kNumDirections)
    return fail(CMI_ERR_INVALID_ARGUMENT, "input direction %d out of range", input_direction);
  DevSubgrid S{};
  int64_t cells = 1;
  for (int a = 0; a < 3; ++a) {
    if (ncell[a] <= 0 || !(box[3 + a] > 0.))
      return fail(CMI_ERR_INVALID_ARGUMENT, "cells and box sides must be positive");
    cells *= ncell[a];
    // DensitySubGrid(box, ncell), DensitySubGrid.hpp:516-527
    S.anchor[a] = box[a];
    S.cell_size[a] = box[3 + a] / ncell[a];
    S.inv_cell_size[a] = ncell[a] / box[3 + a];
    S.cell_size_f[a] = (float)S.cell_size[a];
    S.ncell[a] = ncell[a];
  }
  if (cells > 4096)
    return fail(CMI_ERR_NOT_SUPPORTED, "%lld cells per subgrid exceed 4096",
                (long long)cells);
  S.ncells = (int32_t)cells;
  S.padded_cells = (S.ncells + 3) & ~3;
  for (int d = 0; d < kNumDirections; ++d) S.ngb[d] = kOutside;

  unsigned char *scratch = nullptr;
  CMI_TRY(noalloc_scratch(&scratch));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Packet64 *walked = reinterpret_cast<Packet64 *>(scratch);
  int32_t *dir = reinterpret_cast<int32_t *>(scratch + kNoAllocDirOffset);
  uint8_t *flags = scratch + kNoAllocFlagsOffset;
  uint32_t *err = reinterpret_cast<uint32_t *>(scratch + kNoAllocErrOffset);
  // the previous call's contents stay in the array: the error word is reset
  // to zero here, the output flags are rewritten by the walk kernel, and
  // walked/dir entries are written before they are read
  CMI_CUDA(cudaMemsetAsync(err, 0, sizeof(uint32_t), s));
  {
    NoAllocParams prm{};
    for (int d = 0; d < 32; ++d)
      prm.enabled[d] = (d < kNumDirections) ? (output_enabled ? output_enabled[d] : 1) : 0;
    prm.enabled_out = flags;
    prm.sub = S;
    prm.input_direction = input_direction;
    prm.in = reinterpret_cast<const Packet64 *>(d_in);
    prm.n = n;
    prm.nH = d_nH;
    prm.xH = d_xH;
    prm.J = d_J;
    prm.walked = walked;
    prm.dir = dir;
    prm.err = err;
    prm.tables = make_direction_tables();
    const size_t smem = 24 * (size_t)S.padded_cells;
    CMI_CUDA(cudaFuncSetAttribute(k_traverse_noalloc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem));
    k_traverse_noalloc<<<n > 0 ? (n + 255) / 256 : 1, 256, smem, s>>>(prm);
    CMI_CUDA(cudaGetLastError());
  }
  k_partition<<<1, 256, 0, s>>>(walked, dir, n, flags, reinterpret_cast<Packet64 *>(d_out),
                                d_out_count, d_num_done);
  CMI_CUDA(cudaGetLastError());
  uint32_t herr = 0;
  CMI_CUDA(cudaMemcpyAsync(&herr, err, sizeof(herr), cudaMemcpyDeviceToHost, s));
  CMI_CUDA(cudaStreamSynchronize(s));
  if (herr & kFlagWalkLimit) return fail(CMI_ERR_INVARIANT, "walk step bound exceeded");
  return CMI_OK;
}
