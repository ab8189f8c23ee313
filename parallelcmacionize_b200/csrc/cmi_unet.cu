// Learned warm start: a 3-level 3D convolutional U-Net that maps
// [log n_H, log source flux] on a grid to log10 x_H, with hand-written BF16
// kernels (FP32 accumulation) for inference and training.  No reference
// counterpart: the reference starts every run from x_H = 1e-6
// (DensitySubGrid.hpp:544-551); the network only chooses the starting field,
// the plain Monte Carlo iteration still decides convergence.
//
// Tensors are channels-last BF16 [batch][Z][Y][X][C] with C a multiple of 16;
// channels beyond a tensor's real count are zero.  One sample's voxel order is
// the engine's cube layout ((ix * ny + iy) * nz + iz, with Z = ix, X = iz).
//
// Kernels
//  * k_conv3_tc: 3x3x3 convolution, zero padding, as an implicit GEMM on the
//    5th-generation tensor cores.  A tile is 128 voxels of one sample (8x16x1,
//    or 8x8x2 when Y is not a multiple of 16) = the 128 TMEM lanes of an
//    M = 128 tcgen05.mma; N = output channels; one K step = one kernel tap x
//    16 input channels.  The kernel is persistent (one CTA per SM walks the
//    tiles) and warp-specialised: one thread loads each tile's input box
//    with a one-voxel halo by TMA (out-of-range voxels read as zero: the
//    padding), each 16-channel chunk as two 8-channel halves, unswizzled
//    (8x8x2 tiles: three copies of the halo shifted by -1, 0, +1 in y, so
//    that the 8-voxel rows of both z slices lie one row stride apart), into
//    one of two buffers, so that the next tile loads while this one computes.
//    The A operand of a tap is the halo at its offset (K-major, 16-byte rows,
//    8-row groups one row stride apart, the two channel halves one
//    half-region apart).  The weights (32-byte swizzled K-major) are loaded
//    once per CTA and stay in shared memory when they fit, else they stream
//    through a ring of whole-tap stages.  One thread issues the MMAs into one
//    of two TMEM accumulators; four warps read the other one with tcgen05.ld,
//    add bias, apply leaky ReLU and store BF16.
//    The input gradient of a convolution is the same kernel run on dy with
//    the weights flipped in space and transposed in channels.
//  * k_conv3_wgrad_tc: weight gradient dW[co][tap][ci] = sum_v dy[v][co] *
//    x[v + tap][ci], a reduction over all voxels, on the tensor cores: GEMMs
//    with M = 128 output-channel rows, K = voxels and N = 48 = three taps
//    along x x 16 input channels (the B operand's column groups one voxel
//    apart).  A CTA owns a group of such units, one TMEM accumulator each,
//    and walks the tiles; per tile it loads dy and the input with its halo by
//    TMA (the input box of the forward kernel); four warps move dy into TMEM
//    transposed (lane = output channel), the A operand that every unit's MMAs
//    share, and the B operand of a unit is the halo at its offset (MN-major).
//    At the end the accumulators are read with tcgen05.ld and added to dW
//    with FP32 atomics.
//  * pooling, upsampling, activation backward, the 1x1 output head fused
//    with the MSE loss and its gradient, Adam, weight packing, features.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "cmacionize_b200.h"

namespace cmiu {

using bf16 = __nv_bfloat16;

constexpr long long kWaitCycles = 4000000000ll;
constexpr uint32_t kErrTimeout = 1u;
constexpr int kFeatures = 3;  // input channels of the network

// ---------------------------------------------------------------------------
// error reporting (the engine's cmi_last_error_string is per thread; the
// network keeps its own)
// ---------------------------------------------------------------------------
thread_local char g_err[512];

int fail(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

#define UN_CUDA(call)                                                                      \
  do {                                                                                     \
    const cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) {                                                               \
      (void)cudaGetLastError();                                                            \
      return fail(e_ == cudaErrorMemoryAllocation ? CMI_ERR_OUT_OF_MEMORY : CMI_ERR_CUDA, \
                  "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__,       \
                  __LINE__);                                                               \
    }                                                                                      \
  } while (0)

#define UN_TRY(expr)            \
  do {                          \
    const int rc_ = (expr);     \
    if (rc_ != CMI_OK) return rc_; \
  } while (0)

// ---------------------------------------------------------------------------
// device helpers: mbarrier, TMA, tcgen05
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count));
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait: false (and the error flag) after kWaitCycles SM clock cycles
// (about 2 s); the SM's own cycle counter is cheap to read in the spin loop
__device__ __forceinline__ bool mbar_wait(uint64_t *b, uint32_t parity, uint32_t *err) {
  if (mbar_try(b, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try(b, parity)) {
    if (clock64() - t0 > kWaitCycles) {
      atomicOr(err, kErrTimeout);
      return false;
    }
  }
  return true;
}
__device__ __forceinline__ void tma_load_5d(void *dst, const CUtensorMap *map, int c0, int c1,
                                            int c2, int c3, int c4, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4),
      "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes,
                                          uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// shared-memory matrix descriptor: K-major, 32-byte swizzle, 8-row groups
// 256 bytes apart (start address >> 4 | LBO 16 B | SBO 256 B | version 1 |
// layout SWIZZLE_32B)
__device__ __forceinline__ uint64_t sw32_desc(const void *p) {
  const uint64_t a = (smem_u32(p) & 0x3FFFFu) >> 4;
  return a | (1ull << 16) | ((uint64_t)(256 >> 4) << 32) | (1ull << 46) | (6ull << 61);
}
// shared-memory matrix descriptor, 32-byte swizzle, with the given byte offsets
// (K-major: sbo between 8-row groups; MN-major: lbo between 16-element column
// groups, sbo between 8-row K groups)
__device__ __forceinline__ uint64_t sw32_desc_off(const void *p, uint32_t lbo, uint32_t sbo) {
  const uint64_t a = (smem_u32(p) & 0x3FFFFu) >> 4;
  return a | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) | (1ull << 46) |
         (6ull << 61);
}
// instruction descriptor: BF16 x BF16 -> F32, A and B K-major, M = 128
__host__ __device__ constexpr uint32_t idesc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(128 >> 4) << 24);
}

// ---------------------------------------------------------------------------
// convolution tiles
// ---------------------------------------------------------------------------
// A tile is kMT sub-tiles of 128 voxels, each the M = 128 rows of its own MMAs
// and TMEM accumulator, row r = x + 8 (y + TY z):
//  * TY = 16: 8 x 16 x KZ voxels (KZ = kMT z slices of 8 x 16); the input box
//    with its one-voxel halo is one copy of 10 x 18 x (KZ + 2) voxels, shared by
//    the sub-tiles (the deeper the tile, the fewer halo voxels per output);
//  * TY = 8:  8 x 8 x 2 voxels, one sub-tile (grids whose Y is not a multiple
//    of 16); the halo is three copies of 10 x 8 x 4 voxels shifted by -1, 0, +1
//    in y, so that in a copy the 8-voxel rows of both z slices lie one row
//    stride apart.
// Each 16-channel chunk of the input is stored in its own region, one 32-byte
// row per voxel (x fastest), with the 32-byte swizzle of the tensor cores
// (address bit 4 ^= bit 7) that TMA applies as it writes.  An A operand (K-major,
// SWIZZLE_32B: 8 voxel rows x 16 channels per atom) is then the halo at the tap's
// offset with its 8-voxel groups kRowBytes apart (SBO): the swizzle is a function
// of the shared-memory address, so an operand may start at any voxel row.  The
// weight-gradient kernel reads the same regions as MN-major B operands (16
// channels per row, 8-voxel K groups kRowBytes apart, chunks kChunkBytes apart).
template <int TY, int KZ = 1>
struct ConvTile {
  static_assert(TY == 16 || KZ == 1, "8 x 8 x 2 tiles have one sub-tile");
  static constexpr int kMT = KZ;                         // sub-tiles (M = 128 each)
  static constexpr int kTX = 8, kTY = TY, kTZ = (TY == 16) ? KZ : 2;
  static constexpr int kHX = kTX + 2, kHZ = kTZ + 2;
  static constexpr int kCopies = (TY == 16) ? 1 : 3;
  static constexpr int kCopyRows = (TY == 16) ? kTY + 2 : kTY;  // y rows per z slice
  static constexpr int kCopyBytes = kHX * kCopyRows * kHZ * 32;
  static constexpr int kChunkBytes = (kCopies * kCopyBytes + 1023) / 1024 * 1024;
  static constexpr int kRowBytes = kHX * 32;  // from one 8-voxel row to the next
  static_assert(kCopies == 1 || kCopyBytes % 1024 == 0, "copies start on 1024-byte boundaries");
  // A operand of sub-tile st and tap (hz, hy, hx) (halo offsets 0..2), from the
  // start of a chunk
  static __host__ __device__ constexpr int tap_offset(int st, int hz, int hy, int hx) {
    return (kCopies == 1) ? (((hz + st) * kCopyRows + hy) * kHX + hx) * 32
                          : hy * kCopyBytes + (hz * kCopyRows * kHX + hx) * 32;
  }
  // the TMA loads of one 16-channel chunk of the halo (c0: first channel)
  static __device__ __forceinline__ void load_chunk(unsigned char *dst, const CUtensorMap *map,
                                                    int c0, int x0, int y0, int z0, int n,
                                                    uint64_t *bar) {
#pragma unroll
    for (int d = 0; d < kCopies; ++d)
      tma_load_5d(dst + d * kCopyBytes, map, c0, x0 - 1, y0 - 1 + (kCopies == 1 ? 0 : d),
                  z0 - 1, n, bar);
  }
  static __device__ __forceinline__ void tile_origin(int t, const int dims[3], int &x0, int &y0,
                                                     int &z0, int &n) {
    const int tx = dims[0] / kTX, ty = dims[1] / kTY, tz = dims[2] / kTZ;
    const int bx = t % tx;
    t /= tx;
    const int by = t % ty;
    t /= ty;
    const int bz = t % tz;
    n = t / tz;
    x0 = bx * kTX;
    y0 = by * kTY;
    z0 = bz * kTZ;
  }
  static __host__ __device__ int num_tiles(int batch, const int dims[3]) {
    return batch * (dims[0] / kTX) * (dims[1] / kTY) * (dims[2] / kTZ);
  }
};

// bounded wait that also gives up once another role of the CTA has given up
__device__ __forceinline__ bool role_wait(uint64_t *b, uint32_t parity, uint32_t *err,
                                          volatile int *abort) {
  if (*abort) return false;
  if (!mbar_wait(b, parity, err)) {
    *abort = 1;
    return false;
  }
  return true;
}

// BF16 vectors of 8 channels (16 bytes)
struct Bf8 {
  float v[8];
};
__device__ __forceinline__ Bf8 load8(const bf16 *p) {
  const uint4 q = *reinterpret_cast<const uint4 *>(p);
  const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&q);
  Bf8 r;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float2 f = __bfloat1622float2(h[k]);
    r.v[2 * k] = f.x;
    r.v[2 * k + 1] = f.y;
  }
  return r;
}
__device__ __forceinline__ void store8(bf16 *p, const Bf8 &r) {
  uint4 q;
  __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&q);
#pragma unroll
  for (int k = 0; k < 4; ++k) h[k] = __floats2bfloat162_rn(r.v[2 * k], r.v[2 * k + 1]);
  *reinterpret_cast<uint4 *>(p) = q;
}
// leaky ReLU derivative from the activation output y (same sign as its input)
__device__ __forceinline__ void gate8(Bf8 &d, const bf16 *y, float slope) {
  const Bf8 g = load8(y);
#pragma unroll
  for (int k = 0; k < 8; ++k)
    if (!(g.v[k] > 0.f)) d.v[k] *= slope;
}

// ---------------------------------------------------------------------------
// 3x3x3 convolution on tensor cores: persistent, warp-specialised
// ---------------------------------------------------------------------------
struct ConvArgs {
  const bf16 *wpack;     // [steps][npad][16], 32-byte swizzled rows
  const float *bias;     // [npad] (may be null)
  bf16 *out;             // output tensor base
  int out_ctot, out_c0;  // its channel count and this convolution's first channel
  int npad;              // output channels (multiple of 16, <= 256)
  int nchunk;            // 16-channel chunks of the input
  int nbuf;              // halo buffers (2: the next tile's halo loads during this one)
  int wstages;           // weight stages of one tap each; 27: all weights stay resident
  int kq;                // k_conv3_xf: K steps per weight stage (divides nchunk)
  int dims[3];           // X, Y, Z
  int batch;
  int act;               // 1: leaky ReLU
  float slope;
  const bf16 *gate;      // input-gradient convolutions: out *= leaky'(gate) (may be null)
  int gate_ctot, gate_c0;
  uint32_t *err;
};
constexpr int kConvWarps = 6;               // 0-3 epilogue, 4 loads, 5 MMAs
constexpr int kConvThreads = kConvWarps * 32;
constexpr int kMaxWStages = 27;            // one per tap: resident weights

// A CTA walks tiles blockIdx.x, + gridDim.x, ...: warp 4 loads each tile's halo
// (into buffer i % nbuf) and the weights, one stage per tap (nchunk K steps);
// with 27 stages the weights are loaded once and stay for all tiles of the CTA,
// else they stream through a ring of wstages.  Warp 5 issues the MMAs of tile i
// into TMEM accumulator set i % 2 (one accumulator per sub-tile); warps 0-3 read
// set i % 2, add bias, apply the activation and store BF16 while the MMAs of
// tile i + 1 run.  With resident weights the MMA loop is fully unrolled over the
// taps and sub-tiles, so that one tcgen05.mma follows the next with only a
// descriptor add between them.
template <int TY, int KZ>
__global__ void __launch_bounds__(kConvThreads) k_conv3_tc(const __grid_constant__ CUtensorMap in,
                                                           ConvArgs a) {
  using T = ConvTile<TY, KZ>;
  extern __shared__ __align__(1024) unsigned char sm_raw[];
  unsigned char *sm = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(sm_raw) + 1023) & ~(uintptr_t)1023);
  const int bbytes = a.npad * 32;                             // one K step's weights
  const int tbytes = a.nchunk * bbytes;                        // one tap's weights
  const int S = a.wstages;
  const bool resident = S == 27;
  const size_t hbytes = (size_t)a.nchunk * T::kChunkBytes;    // one halo buffer
  unsigned char *sH = sm;                                      // [nbuf][nchunk][chunk]
  unsigned char *sB = sH + a.nbuf * hbytes;                    // [S][nchunk][npad * 32]
  float *sbias = reinterpret_cast<float *>(sB + (size_t)S * tbytes);
  uint64_t *b_full = reinterpret_cast<uint64_t *>(sbias + a.npad);
  uint64_t *b_empty = b_full + kMaxWStages;
  uint64_t *h_full = b_empty + kMaxWStages;  // [2]
  uint64_t *h_empty = h_full + 2;          // [2]
  uint64_t *a_full = h_empty + 2;          // [2]
  uint64_t *a_empty = a_full + 2;          // [2]
  uint64_t *drain = a_empty + 2;           // the MMAs in flight when the CTA ends
  uint32_t *tslot = reinterpret_cast<uint32_t *>(drain + 1);
  __shared__ int s_abort;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tiles = T::num_tiles(a.batch, a.dims);
  const int nmine = (blockIdx.x < tiles) ? (tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const uint32_t acols = a.npad <= 32 ? 32u : a.npad <= 64 ? 64u : a.npad <= 128 ? 128u : 256u;
  const uint32_t scols = T::kMT * acols;  // one accumulator set

  for (int c = tid; c < a.npad; c += kConvThreads) sbias[c] = a.bias ? a.bias[c] : 0.f;
  if (tid == 0) {
    s_abort = 0;
    for (int s = 0; s < S; ++s) {
      mbar_init(&b_full[s], 1);
      mbar_init(&b_empty[s], 1);
    }
    for (int s = 0; s < 2; ++s) {
      mbar_init(&h_full[s], 1);
      mbar_init(&h_empty[s], 1);
      mbar_init(&a_full[s], 1);
      mbar_init(&a_empty[s], 4);  // one arrival per epilogue warp
    }
    mbar_init(drain, 1);
    fence_mbar_init();
  }
  if (warp == 5) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tslot)),
                 "r"(2 * scols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  volatile int *abort = &s_abort;

  if (warp == 4 && lane == 0) {
    // loads: resident weights once, in one copy; then per tile its halo and,
    // when the weights stream, one stage per tap
    int tiles_issued = 0, stages_issued = 0;
    if (resident && nmine > 0) {
      mbar_expect_tx(&b_full[0], (uint32_t)(27 * tbytes));
      bulk_load(sB, a.wpack, (uint32_t)(27 * tbytes), &b_full[0]);
    }
    for (int i = 0; i < nmine && !*abort; ++i) {
      int x0, y0, z0, n;
      T::tile_origin(blockIdx.x + i * gridDim.x, a.dims, x0, y0, z0, n);
      const int hb = i % a.nbuf, hu = i / a.nbuf;
      if (hu > 0 && !role_wait(&h_empty[hb], (uint32_t)(hu - 1) & 1u, a.err, abort)) break;
      mbar_expect_tx(&h_full[hb], (uint32_t)(a.nchunk * T::kCopies * T::kCopyBytes));
      unsigned char *h = sH + hb * hbytes;
      for (int c = 0; c < a.nchunk; ++c)
        T::load_chunk(h + (size_t)c * T::kChunkBytes, &in, c * 16, x0, y0, z0, n, &h_full[hb]);
      tiles_issued = i + 1;
      if (resident) continue;
      for (int tap = 0; tap < 27; ++tap) {
        const int g = i * 27 + tap, s = g % S, u = g / S;
        if (u > 0 && !role_wait(&b_empty[s], (uint32_t)(u - 1) & 1u, a.err, abort)) break;
        mbar_expect_tx(&b_full[s], (uint32_t)tbytes);
        bulk_load(sB + (size_t)s * tbytes, a.wpack + (size_t)tap * a.nchunk * a.npad * 16,
                  (uint32_t)tbytes, &b_full[s]);
        stages_issued = g + 1;
      }
    }
    // the last copy into every buffer has landed before the CTA ends (they have
    // all been consumed, unless a role gave up)
    for (int i = max(0, tiles_issued - a.nbuf); i < tiles_issued; ++i)
      mbar_wait(&h_full[i % a.nbuf], (uint32_t)(i / a.nbuf) & 1u, a.err);
    for (int g = max(0, stages_issued - S); g < stages_issued; ++g)
      mbar_wait(&b_full[g % S], (uint32_t)(g / S) & 1u, a.err);
    if (resident && nmine > 0) mbar_wait(&b_full[0], 0u, a.err);
  } else if (warp == 5 && lane == 0) {
    const uint32_t idesc = idesc_bf16(a.npad);
    // descriptors advance by (byte offset >> 4) in their low 14-bit address
    // field; every operand lies below 256 KB, so the sums never carry out of it
    const uint64_t bdesc0 = sw32_desc_off(sB, 16u, 256u);
    const uint32_t cstep = (uint32_t)T::kChunkBytes >> 4;  // next 16-channel chunk
    const uint32_t bstep = (uint32_t)bbytes >> 4;           // next K step's weights
    const int nchunk = a.nchunk;
    const uint64_t tstep = (uint64_t)nchunk * bstep;        // next tap's weights
    bool ok = true;
    if (resident && nmine > 0) {
      ok = role_wait(&b_full[0], 0u, a.err, abort);
      tc_fence_after();
    }
    int s = 0;            // weight stage of the next tap (streaming)
    uint32_t sphase = 0;  // its parity
    for (int i = 0; i < nmine && ok && !*abort; ++i) {
      const int ab = i & 1, au = i >> 1;
      const int hb = i % a.nbuf, hu = i / a.nbuf;
      if (au > 0 && !role_wait(&a_empty[ab], (uint32_t)(au - 1) & 1u, a.err, abort)) break;
      if (!role_wait(&h_full[hb], (uint32_t)hu & 1u, a.err, abort)) break;
      tc_fence_after();
      const uint64_t adesc0 = sw32_desc_off(sH + hb * hbytes, 16u, (uint32_t)T::kRowBytes);
      const uint32_t d0 = tmem + (uint32_t)ab * scols;
      if (resident) {
        // registers only in this loop: the MMA statements carry no memory
        // clobber (they are ordered by being volatile, and the data they read
        // was published by the barrier waits above)
        uint64_t bd = bdesc0;
        const int nch = nchunk;
        if (nch == 1) {
          // one 16-channel chunk: one MMA per tap and sub-tile
          for (int tap = 0; tap < 27; ++tap) {
            const uint64_t at =
                adesc0 + ((uint32_t)T::tap_offset(0, tap / 9, (tap / 3) % 3, tap % 3) >> 4);
            const uint32_t acc = tap > 0 ? 1u : 0u;
#pragma unroll
            for (int st = 0; st < T::kMT; ++st)
              asm volatile(
                  "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                  " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(
                      d0 + (uint32_t)st * acols),
                  "l"(at + (uint32_t)(T::tap_offset(st, 0, 0, 0) >> 4)), "l"(bd), "r"(idesc),
                  "r"(acc));
            bd += bstep;
          }
        } else {
          for (int tap = 0; tap < 27; ++tap) {
            // tap (dz, dy, dx) reads the input at (x + dx, y + dy, z + dz)
            uint64_t at =
                adesc0 + ((uint32_t)T::tap_offset(0, tap / 9, (tap / 3) % 3, tap % 3) >> 4);
            uint64_t bc = bd;
            for (int c = 0; c < nch; ++c) {
              const uint32_t acc = (tap > 0 || c > 0) ? 1u : 0u;
#pragma unroll
              for (int st = 0; st < T::kMT; ++st)
                asm volatile(
                    "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                    " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(
                        d0 + (uint32_t)st * acols),
                    "l"(at + (uint32_t)(T::tap_offset(st, 0, 0, 0) >> 4)), "l"(bc),
                    "r"(idesc), "r"(acc));
              at += cstep;
              bc += bstep;
            }
            bd += tstep;
          }
        }
      } else {
        for (int tap = 0; tap < 27; ++tap) {
          if (!role_wait(&b_full[s], sphase, a.err, abort)) {
            ok = false;
            break;
          }
          tc_fence_after();
          uint64_t bc = bdesc0 + (uint32_t)(s * nchunk) * bstep;
          uint64_t at =
              adesc0 + ((uint32_t)T::tap_offset(0, tap / 9, (tap / 3) % 3, tap % 3) >> 4);
          for (int c = 0; c < nchunk; ++c) {
            const uint32_t acc = (tap > 0 || c > 0) ? 1u : 0u;
#pragma unroll
            for (int st = 0; st < T::kMT; ++st)
              asm volatile(
                  "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                  " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(
                      d0 + (uint32_t)st * acols),
                  "l"(at + (uint32_t)(T::tap_offset(st, 0, 0, 0) >> 4)), "l"(bc), "r"(idesc),
                  "r"(acc));
            at += cstep;
            bc += bstep;
          }
          asm volatile(
              "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                  smem_u32(&b_empty[s]))
              : "memory");
          if (++s == S) {
            s = 0;
            sphase ^= 1u;
          }
        }
        if (!ok) break;
      }
      // the halo buffer and the accumulators are released once these MMAs complete
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
              smem_u32(&h_empty[hb]))
          : "memory");
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
              smem_u32(&a_full[ab]))
          : "memory");
    }
    // every MMA issued has completed before TMEM is released
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            smem_u32(drain))
        : "memory");
    mbar_wait(drain, 0, a.err);
  } else if (warp < 4) {
    for (int i = 0; i < nmine; ++i) {
      const int ab = i & 1;
      // one lane waits, then the warp reads its 32 TMEM lanes of every sub-tile
      bool ok0 = true;
      if (lane == 0) ok0 = role_wait(&a_full[ab], (uint32_t)(i >> 1) & 1u, a.err, abort);
      if (!__shfl_sync(0xffffffffu, ok0, 0)) break;
      tc_fence_after();
      int x0, y0, z0, n;
      T::tile_origin(blockIdx.x + i * gridDim.x, a.dims, x0, y0, z0, n);
      // row r of sub-tile st = voxel (x0 + r % 8, y0 + (r / 8) % TY, z)
      const int r = warp * 32 + lane;
      const int vx = x0 + (r & 7), vy = y0 + ((r >> 3) % T::kTY);
#pragma unroll
      for (int st = 0; st < T::kMT; ++st) {
        const int vz = z0 + (T::kCopies == 1 ? st : r / (8 * T::kTY));
        const size_t vox = (((size_t)n * a.dims[2] + vz) * a.dims[1] + vy) * a.dims[0] + vx;
        bf16 *dst = a.out + vox * a.out_ctot + a.out_c0;
        for (int j = 0; j < a.npad; j += 16) {
          uint32_t v[16];
          const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)ab * scols +
                                 (uint32_t)st * acols + (uint32_t)j;
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,"
              "%12,%13,%14,%15}, [%16];"
              : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
              : "r"(taddr));
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
          __align__(16) bf16 o[16];
          float gy[16];
          if (a.gate) {
            const bf16 *gp = a.gate + vox * a.gate_ctot + a.gate_c0 + j;
            const Bf8 g0 = load8(gp), g1 = load8(gp + 8);
#pragma unroll
            for (int e = 0; e < 8; ++e) {
              gy[e] = g0.v[e];
              gy[e + 8] = g1.v[e];
            }
          }
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            float f = __uint_as_float(v[e]) + sbias[j + e];
            if (a.act) f = f > 0.f ? f : f * a.slope;
            if (a.gate) {
              // the stored BF16 gradient times the activation derivative
              f = __bfloat162float(__float2bfloat16_rn(f));
              if (!(gy[e] > 0.f)) f *= a.slope;
            }
            o[e] = __float2bfloat16_rn(f);
          }
          uint4 *d4 = reinterpret_cast<uint4 *>(dst + j);
          d4[0] = reinterpret_cast<const uint4 *>(o)[0];
          d4[1] = reinterpret_cast<const uint4 *>(o)[1];
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(
                                      smem_u32(&a_empty[ab]))
                                  : "memory");
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 5) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(2 * scols)
                 : "memory");
  }
}

// ---------------------------------------------------------------------------
// 3x3x3 convolution with the x taps folded into N
// ---------------------------------------------------------------------------
// The MMA rows are u = 16 x 8 voxels (x fastest) and N = 3 x npad columns: for
// a (dz, dy) tap row, column g npad + c of row u accumulates sum over the input
// channels of x(u + (0, dy, dz)) W(dz, dy, dx = g)[c].  The output at v is then
// D(v - 1)[0] + D(v)[1] + D(v + 1)[2]: the neighbours along x are the lanes
// either side in the warp, so the epilogue combines them with two shuffles.  A
// tile yields the 14 x 8 outputs of its u columns 1 .. 14 (tiles overlap by two
// columns; the last one along x is cut at the grid's edge).  Each (dz, dy, chunk)
// is one MMA of N = 3 npad instead of three of N = npad, and the input box needs
// no halo in x: 16 x 10 x (KZ + 2) voxels.
template <int KZ>
struct XTile {
  static constexpr int kUX = 16, kUY = 8;            // MMA rows: 16 x 8 voxels
  static constexpr int kOX = 14;                     // outputs per tile along x
  static constexpr int kHY = kUY + 2, kHZ = KZ + 2;  // input rows, slices
  static constexpr int kCopyBytes = kUX * kHY * kHZ * 32;
  static constexpr int kChunkBytes = (kCopyBytes + 1023) / 1024 * 1024;
  // A operand of sub-tile st and tap row (dz, dy): 128 consecutive voxel rows
  static __host__ __device__ constexpr int tap_offset(int st, int dz, int dy) {
    return ((st + dz) * kHY + dy) * kUX * 32;
  }
  static __device__ __forceinline__ void origin(int t, const int dims[3], int &x0, int &y0,
                                                int &z0, int &n) {
    const int tx = (dims[0] + kOX - 1) / kOX, ty = dims[1] / kUY, tz = dims[2] / KZ;
    const int bx = t % tx;
    t /= tx;
    const int by = t % ty;
    t /= ty;
    const int bz = t % tz;
    n = t / tz;
    x0 = bx * kOX - 1;
    y0 = by * kUY;
    z0 = bz * KZ;
  }
  static __host__ __device__ int num_tiles(int batch, const int dims[3]) {
    return batch * ((dims[0] + kOX - 1) / kOX) * (dims[1] / kUY) * (dims[2] / KZ);
  }
};

// A persistent, warp-specialised CTA like k_conv3_tc's, with kXfEpiWarps + 2
// warps: warp kXfEpiWarps loads (the weights once when resident, else kq K
// steps per ring stage; each tile's input box into a ring of up to kMaxInBufs
// buffers, as many as shared memory holds), warp kXfEpiWarps + 1 issues the
// MMAs (the whole warp, one elected lane issuing), warps 0 .. kXfEpiWarps - 1
// combine the x taps, add bias, apply the activation or the derivative gate
// and store.
constexpr int kMaxInBufs = 8;
constexpr int kXfEpiWarps = 8;                      // two per quarter of the TMEM lanes
constexpr int kXfThreads = (kXfEpiWarps + 2) * 32;  // + loads + MMAs
// tcgen05.mma and tcgen05.commit issued by one elected lane of a converged warp:
// the x-folded kernel's MMA role runs its loops on the whole warp, whose
// branches are then uniform (a branch inside a one-lane region costs more than
// an MMA).  elect.sync picks the same lane every time, so the commits track the
// MMAs that lane issued.  No memory clobber on the MMA: the statements are
// ordered by being volatile, and their operands were published by the barrier
// waits before them.
__device__ __forceinline__ void mma_el(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc,
                                       uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p, e;\n elect.sync _|e, 0xffffffff;\n setp.ne.b32 p, %4, 0;\n"
      " @e tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void commit_el(uint64_t *bar) {
  asm volatile(
      "{\n .reg .pred e;\n elect.sync _|e, 0xffffffff;\n"
      " @e tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n}" ::"r"(
          smem_u32(bar))
      : "memory");
}
// bounded wait of a whole warp with one outcome for all its lanes
__device__ __forceinline__ bool warp_wait(uint64_t *b, uint32_t parity, uint32_t *err,
                                          volatile int *abort) {
  return __all_sync(0xffffffffu, role_wait(b, parity, err, abort));
}

// The MMAs of one tile with resident weights, fully unrolled (NCH input chunks),
// so that they follow one another with only descriptor adds between them.
template <int KZ, int NCH>
__device__ __forceinline__ void xf_mma_tile(uint32_t d0, uint32_t acols, uint64_t adesc0,
                                            uint64_t bdesc0, uint32_t idesc, uint32_t bstep) {
  using T = XTile<KZ>;
  uint64_t bd = bdesc0;
#pragma unroll
  for (int t9 = 0; t9 < 9; ++t9)
#pragma unroll
    for (int c = 0; c < NCH; ++c) {
#pragma unroll
      for (int st = 0; st < KZ; ++st)
        mma_el(d0 + (uint32_t)st * acols,
               adesc0 + (uint32_t)((T::tap_offset(st, t9 / 3, t9 % 3) + c * T::kChunkBytes) >> 4),
               bd, idesc, (t9 > 0 || c > 0) ? 1u : 0u);
      bd += bstep;
    }
}

// The MMAs of one tap row (NCH input chunks) from one weight stage, unrolled;
// acc0 = 0 starts the accumulators
template <int KZ, int NCH>
__device__ __forceinline__ void xf_mma_row(uint32_t d0, uint32_t acols, uint64_t at, uint64_t bd,
                                           uint32_t idesc, uint32_t bstep, uint32_t acc0) {
  using T = XTile<KZ>;
#pragma unroll
  for (int c = 0; c < NCH; ++c) {
#pragma unroll
    for (int st = 0; st < KZ; ++st)
      mma_el(d0 + (uint32_t)st * acols,
             at + (uint32_t)((T::tap_offset(st, 0, 0) + c * T::kChunkBytes) >> 4), bd, idesc,
             c > 0 ? 1u : acc0);
    bd += bstep;
  }
}

// NCH > 0: the kernel for NCH input chunks (resident weights, or a stage per
// tap row, fully unrolled); 0: any chunk count
template <int KZ, int NCH>
__global__ void __launch_bounds__(kXfThreads, 1) k_conv3_xf(const __grid_constant__ CUtensorMap in,
                                                           ConvArgs a) {
  using T = XTile<KZ>;
  extern __shared__ __align__(1024) unsigned char sm_raw[];
  unsigned char *sm = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(sm_raw) + 1023) & ~(uintptr_t)1023);
  const int nrow = 3 * a.npad;                                // MMA N
  const int bbytes = nrow * 32;                               // one K step's weights
  const int tbytes = a.nchunk * bbytes;                       // one tap row's weights
  const int qbytes = a.kq * bbytes;                           // one weight stage
  const int kst = 9 * a.nchunk / a.kq;                        // weight stages per tile
  const int S = a.wstages;
  const bool resident = S == kst && a.kq == a.nchunk;
  const size_t hbytes = (size_t)a.nchunk * T::kChunkBytes;   // one input buffer
  unsigned char *sH = sm;                                     // [nbuf][nchunk][chunk]
  unsigned char *sB = sH + a.nbuf * hbytes;                   // [S][kq][3 npad * 32]
  float *sbias = reinterpret_cast<float *>(sB + (size_t)S * qbytes);
  uint64_t *b_full = reinterpret_cast<uint64_t *>(sbias + a.npad);
  uint64_t *b_empty = b_full + kMaxWStages;
  uint64_t *h_full = b_empty + kMaxWStages;  // [kMaxInBufs]
  uint64_t *h_empty = h_full + kMaxInBufs;   // [kMaxInBufs]
  uint64_t *a_full = h_empty + kMaxInBufs;   // [2]
  uint64_t *a_empty = a_full + 2;            // [2]
  uint64_t *drain = a_empty + 2;             // the MMAs in flight when the CTA ends
  uint32_t *tslot = reinterpret_cast<uint32_t *>(drain + 1);
  __shared__ int s_abort;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tiles = T::num_tiles(a.batch, a.dims);
  const int nmine = (blockIdx.x < tiles) ? (tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const uint32_t acols = nrow <= 64 ? 64u : nrow <= 128 ? 128u : 256u;
  const uint32_t scols = KZ * acols;  // one accumulator set

  for (int c = tid; c < a.npad; c += kXfThreads) sbias[c] = a.bias ? a.bias[c] : 0.f;
  if (tid == 0) {
    s_abort = 0;
    for (int s = 0; s < S; ++s) {
      mbar_init(&b_full[s], 1);
      mbar_init(&b_empty[s], 1);
    }
    for (int s = 0; s < a.nbuf; ++s) {
      mbar_init(&h_full[s], 1);
      mbar_init(&h_empty[s], 1);
    }
    for (int s = 0; s < 2; ++s) {
      mbar_init(&a_full[s], 1);
      mbar_init(&a_empty[s], kXfEpiWarps);  // one arrival per epilogue warp
    }
    mbar_init(drain, 1);
    fence_mbar_init();
  }
  if (warp == kXfEpiWarps + 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tslot)),
                 "r"(2 * scols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  volatile int *abort = &s_abort;

  if (warp == kXfEpiWarps && lane == 0) {
    int tiles_issued = 0, stages_issued = 0;
    if (resident && nmine > 0) {
      mbar_expect_tx(&b_full[0], (uint32_t)(9 * tbytes));
      bulk_load(sB, a.wpack, (uint32_t)(9 * tbytes), &b_full[0]);
    }
    for (int i = 0; i < nmine && !*abort; ++i) {
      int x0, y0, z0, n;
      T::origin(blockIdx.x + i * gridDim.x, a.dims, x0, y0, z0, n);
      const int hb = i % a.nbuf, hu = i / a.nbuf;
      if (hu > 0 && !role_wait(&h_empty[hb], (uint32_t)(hu - 1) & 1u, a.err, abort)) break;
      mbar_expect_tx(&h_full[hb], (uint32_t)(a.nchunk * T::kCopyBytes));
      unsigned char *h = sH + hb * hbytes;
      for (int c = 0; c < a.nchunk; ++c)
        tma_load_5d(h + (size_t)c * T::kChunkBytes, &in, c * 16, x0, y0 - 1, z0 - 1, n,
                    &h_full[hb]);
      tiles_issued = i + 1;
      if (resident) continue;
      for (int k = 0; k < kst; ++k) {
        const int g = i * kst + k, s = g % S, u = g / S;
        if (u > 0 && !role_wait(&b_empty[s], (uint32_t)(u - 1) & 1u, a.err, abort)) break;
        mbar_expect_tx(&b_full[s], (uint32_t)qbytes);
        bulk_load(sB + (size_t)s * qbytes, a.wpack + (size_t)k * a.kq * nrow * 16,
                  (uint32_t)qbytes, &b_full[s]);
        stages_issued = g + 1;
      }
    }
    // the last copy into every buffer has landed before the CTA ends
    for (int i = max(0, tiles_issued - a.nbuf); i < tiles_issued; ++i)
      mbar_wait(&h_full[i % a.nbuf], (uint32_t)(i / a.nbuf) & 1u, a.err);
    for (int g = max(0, stages_issued - S); g < stages_issued; ++g)
      mbar_wait(&b_full[g % S], (uint32_t)(g / S) & 1u, a.err);
    if (resident && nmine > 0) mbar_wait(&b_full[0], 0u, a.err);
  } else if (warp == kXfEpiWarps + 1) {
    const uint32_t idesc = idesc_bf16(nrow);
    // descriptors advance by (byte offset >> 4) in their low 14-bit address
    // field; every operand lies below 256 KB, so the sums never carry out of it
    const uint64_t bdesc0 = sw32_desc_off(sB, 16u, 256u);
    const uint32_t cstep = (uint32_t)T::kChunkBytes >> 4;  // next 16-channel chunk
    const uint32_t bstep = (uint32_t)bbytes >> 4;           // next K step's weights
    const int nchunk = a.nchunk;
    bool ok = true;
    if (resident && nmine > 0) {
      ok = warp_wait(&b_full[0], 0u, a.err, abort);
      tc_fence_after();
    }
    int s = 0;            // weight stage of the next K steps (streaming)
    uint32_t sphase = 0;  // its parity
    int hb = 0;           // input buffer of tile i
    uint32_t hphase = 0;  // its parity
    for (int i = 0; i < nmine && ok; ++i) {
      const int ab = i & 1;
      if (i >= 2 && !warp_wait(&a_empty[ab], (uint32_t)((i >> 1) - 1) & 1u, a.err, abort)) break;
      if (!warp_wait(&h_full[hb], hphase, a.err, abort)) break;
      tc_fence_after();
      const uint64_t adesc0 = sw32_desc_off(sH + hb * hbytes, 16u, 256u);
      const uint32_t d0 = tmem + (uint32_t)ab * scols;
      if (NCH > 0 && resident) {
        xf_mma_tile<KZ, (NCH > 0 ? NCH : 1)>(d0, acols, adesc0, bdesc0, idesc, bstep);
      } else if (resident) {
        // registers only: see xf_mma_tile
        uint64_t bd = bdesc0;
        for (int t9 = 0; t9 < 9; ++t9) {
          uint64_t at = adesc0 + ((uint32_t)T::tap_offset(0, t9 / 3, t9 % 3) >> 4);
          for (int c = 0; c < nchunk; ++c) {
            const uint32_t acc = (t9 > 0 || c > 0) ? 1u : 0u;
#pragma unroll
            for (int st = 0; st < KZ; ++st)
              mma_el(d0 + (uint32_t)st * acols, at + (uint32_t)(T::tap_offset(st, 0, 0) >> 4), bd,
                     idesc, acc);
            at += cstep;
            bd += bstep;
          }
        }
      } else {
        // stage k holds K steps k kq .. k kq + kq - 1 (tap row t9 = step / nchunk)
        for (int k = 0; k < kst; ++k) {
          if (!warp_wait(&b_full[s], sphase, a.err, abort)) {
            ok = false;
            break;
          }
          tc_fence_after();
          uint64_t bd = bdesc0 + (uint32_t)(s * a.kq) * bstep;
          if (NCH > 0 && a.kq == NCH) {
            // one tap row per stage
            xf_mma_row<KZ, (NCH > 0 ? NCH : 1)>(
                d0, acols, adesc0 + ((uint32_t)T::tap_offset(0, k / 3, k % 3) >> 4), bd, idesc,
                bstep, k > 0 ? 1u : 0u);
            commit_el(&b_empty[s]);
            if (++s == S) {
              s = 0;
              sphase ^= 1u;
            }
            continue;
          }
          const int step0 = k * a.kq, t9 = step0 / nchunk, c0 = step0 - t9 * nchunk;
          uint64_t at = adesc0 + ((uint32_t)(T::tap_offset(0, t9 / 3, t9 % 3) +
                                             c0 * T::kChunkBytes) >> 4);
          for (int c = 0; c < a.kq; ++c) {
            const uint32_t acc = (step0 + c > 0) ? 1u : 0u;
#pragma unroll
            for (int st = 0; st < KZ; ++st)
              mma_el(d0 + (uint32_t)st * acols, at + (uint32_t)(T::tap_offset(st, 0, 0) >> 4), bd,
                     idesc, acc);
            at += cstep;
            bd += bstep;
          }
          commit_el(&b_empty[s]);
          if (++s == S) {
            s = 0;
            sphase ^= 1u;
          }
        }
        if (!ok) break;
      }
      // the input buffer and the accumulators are released once these MMAs complete
      commit_el(&h_empty[hb]);
      commit_el(&a_full[ab]);
      if (++hb == a.nbuf) {
        hb = 0;
        hphase ^= 1u;
      }
    }
    // every MMA issued has completed before TMEM is released
    commit_el(drain);
    mbar_wait(drain, 0, a.err);
  } else if (warp < kXfEpiWarps) {
    for (int i = 0; i < nmine; ++i) {
      const int ab = i & 1;
      bool ok0 = true;
      if (lane == 0) ok0 = role_wait(&a_full[ab], (uint32_t)(i >> 1) & 1u, a.err, abort);
      if (!__shfl_sync(0xffffffffu, ok0, 0)) break;
      tc_fence_after();
      int x0, y0, z0, n;
      T::origin(blockIdx.x + i * gridDim.x, a.dims, x0, y0, z0, n);
      // row r = u (16 x 8, x fastest); outputs at u columns 1 .. 14 inside the grid.
      // Warps q and q + 4 read TMEM lanes 32 q .. 32 q + 31 and share the
      // (sub-tile, 16-channel group) items of the tile between them.
      const int q = warp & 3, r = q * 32 + lane, ux = r & 15;
      const int vx = x0 + ux, vy = y0 + (r >> 4);
      const bool valid = ux >= 1 && ux <= T::kOX && vx < a.dims[0];
      const int ngrp = a.npad >> 4;
      for (int item = warp >> 2; item < KZ * ngrp; item += kXfEpiWarps / 4) {
        const int st = item / ngrp, j = (item - st * ngrp) * 16;
        const int vz = z0 + st;
        const size_t vox = (((size_t)n * a.dims[2] + vz) * a.dims[1] + vy) * a.dims[0] + vx;
        {
          uint32_t v[3][16];
#pragma unroll
          for (int g = 0; g < 3; ++g) {
            const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)ab * scols +
                                   (uint32_t)st * acols + (uint32_t)(g * a.npad + j);
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,"
                "%12,%13,%14,%15}, [%16];"
                : "=r"(v[g][0]), "=r"(v[g][1]), "=r"(v[g][2]), "=r"(v[g][3]), "=r"(v[g][4]),
                  "=r"(v[g][5]), "=r"(v[g][6]), "=r"(v[g][7]), "=r"(v[g][8]), "=r"(v[g][9]),
                  "=r"(v[g][10]), "=r"(v[g][11]), "=r"(v[g][12]), "=r"(v[g][13]),
                  "=r"(v[g][14]), "=r"(v[g][15])
                : "r"(taddr));
          }
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
          float f[16];
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            // x tap -1 from the lane before, +1 from the lane after
            const float left = __shfl_up_sync(0xffffffffu, __uint_as_float(v[0][e]), 1);
            const float right = __shfl_down_sync(0xffffffffu, __uint_as_float(v[2][e]), 1);
            f[e] = left + __uint_as_float(v[1][e]) + right;
          }
          if (valid) {
            bf16 *dst = a.out + vox * a.out_ctot + a.out_c0 + j;
            float gy[16];
            if (a.gate) {
              const bf16 *gp = a.gate + vox * a.gate_ctot + a.gate_c0 + j;
              const Bf8 g0 = load8(gp), g1 = load8(gp + 8);
#pragma unroll
              for (int e = 0; e < 8; ++e) {
                gy[e] = g0.v[e];
                gy[e + 8] = g1.v[e];
              }
            }
            // leaky ReLU as max(x, slope x): the same for 0 <= slope < 1
            __align__(16) __nv_bfloat162 o[8];
#pragma unroll
            for (int e = 0; e < 16; e += 2) {
              float x0 = f[e] + sbias[j + e], x1 = f[e + 1] + sbias[j + e + 1];
              if (a.act) {
                x0 = fmaxf(x0, x0 * a.slope);
                x1 = fmaxf(x1, x1 * a.slope);
              }
              if (a.gate) {
                x0 = __bfloat162float(__float2bfloat16_rn(x0));
                x1 = __bfloat162float(__float2bfloat16_rn(x1));
                if (!(gy[e] > 0.f)) x0 *= a.slope;
                if (!(gy[e + 1] > 0.f)) x1 *= a.slope;
              }
              o[e / 2] = __floats2bfloat162_rn(x0, x1);
            }
            uint4 *d4 = reinterpret_cast<uint4 *>(dst);
            d4[0] = reinterpret_cast<const uint4 *>(o)[0];
            d4[1] = reinterpret_cast<const uint4 *>(o)[1];
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(
                                      smem_u32(&a_empty[ab]))
                                  : "memory");
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kXfEpiWarps + 1) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(2 * scols)
                 : "memory");
  }
}

// ---------------------------------------------------------------------------
// weight gradient on the tensor cores
// ---------------------------------------------------------------------------
struct WgradTcArgs {
  int cout;                  // dy channels (storage, multiple of 16, <= 128)
  int nchunk;                // 16-channel chunks of the input
  int nbuf;                  // tile buffers (2: the next tile loads during this one)
  int dims[3];
  int batch;
  int units_per_cta;         // units (dz x dy chunk x input chunk) of a CTA;
                             // blockIdx.y selects a group of units
  uint32_t tmem_cols;        // power of two >= units_per_cta * kUnitCols
  int bar_off;               // bytes from the buffers' start to the barriers (past every
                             // byte an MMA may read)
  float *dw;                 // [cout_real][27][cin_real] (FP32, accumulated)
  float *db;                 // [cout_real] bias gradient: sum of dy (accumulated; may be null)
  const int *ci_map;         // storage input channel -> real input channel or -1
  int cin_real, cout_real;
  // the CTAs' sums, reduced into dw by k_wgrad_reduce (null: FP32 atomics into
  // dw): [group][cta][unit][dx tap g][accumulator row < 48][16 input channels]
  float *part;
  uint32_t *err;
};
constexpr int kWgradWarps = 6;            // 0-3 bias sums and readout, 4 loads, 5 MMAs
constexpr int kWgradThreads = kWgradWarps * 32;
constexpr int kUnitCols = 48;             // one unit's accumulator: taps dx = -1, 0, 1 x 16
constexpr int kWgradUnitsPerCta = 10;     // 10 x 48 <= 512 TMEM columns
constexpr int kWgMaxBufs = 4;             // tile buffers in flight at most

// dy of a tile with one extra voxel row on either side in y, 16 channels per
// 32-byte voxel row (32-byte swizzle), x fastest:
//  * 8 x 16 x 1 tiles: one box of 8 x 18 rows (rows y0 - 1 .. y0 + 16);
//  * 8 x 8 x 2 tiles: three copies of 8 x 8 x 2 voxels shifted by -1, 0, +1 in y.
// The voxels of the tile shifted by t - 1 rows in y then start kMStride bytes x t
// after the start of the first row (copy).
template <int TY>
struct DyTile {
  static constexpr int kCopies = (TY == 16) ? 1 : 3;
  static constexpr int kRows = (TY == 16) ? TY + 2 : TY;  // y rows of a box
  static constexpr int kTZ = 128 / (8 * TY);
  static constexpr int kCopyBytes = 8 * kRows * kTZ * 32;
  static constexpr int kChunkBytes = (kCopies * kCopyBytes + 1023) / 1024 * 1024;
  static constexpr int kMStride = (TY == 16) ? 8 * 32 : kCopyBytes;
  // bytes past a chunk's start that an MMA's A operand may read: M group 7 of the
  // last K step (voxels 112 .. 127)
  static constexpr int kReach = 7 * kMStride + 7 * 512 + 512;
  static __device__ __forceinline__ void load_chunk(unsigned char *dst, const CUtensorMap *map,
                                                    int c0, int x0, int y0, int z0, int n,
                                                    uint64_t *bar) {
#pragma unroll
    for (int d = 0; d < kCopies; ++d)
      tma_load_5d(dst + d * kCopyBytes, map, c0, x0, y0 - 1 + (kCopies == 1 ? 0 : d), z0, n, bar);
  }
  // byte offset of tile voxel r (r = x + 8 (y + TY z)) in the unshifted rows
  static __device__ __forceinline__ int own_offset(int r) {
    return (kCopies == 1) ? (r + 8) * 32 : kCopyBytes + r * 32;
  }
};

// The work of a tile is 3 x (cout / 16) x nchunk units: one z tap row (dz) x one
// 16-output-channel chunk of dy x one 16-channel input chunk, 8 MMAs (K = 16
// voxels each) that cover all 9 (dy, dx) taps of the row at once:
//  * B (the input halo at dz and the centre y row, MN-major) has its three
//    16-channel column groups one voxel (32 bytes) apart: column group g reads
//    the input shifted by dx = g - 1;
//  * A (dy, MN-major, M = 128 rows in 8 groups of 16 output channels) has its M
//    groups kMStride apart: group t reads dy shifted by t - 1 rows in y, which
//    pairs dy(v) with the input at v + (1 - t) rows.  Groups 3 .. 7 read
//    whatever follows and feed accumulator rows that are never read.
// Over all tiles every voxel meets every tap once: the rows a shifted tile
// misses at the grid's edge pair with input outside the grid (zero).
// A CTA owns a group of units (one TMEM accumulator each) and the tiles
// blockIdx.x, + gridDim.x, ...: warp 4 loads tile i's dy and input halo into
// buffer i % nbuf (up to kWgMaxBufs) by TMA; warp 5 issues the MMAs (the whole
// warp, one elected lane issuing); warps 0-3 sum dy for the bias gradient (the
// CTAs of the first group) and at the end read the TMEM lanes: into the
// scratch rows that k_wgrad_reduce sums over the CTAs, or with FP32 atomics
// straight into dW when no scratch is given.
template <int TY>
__global__ void __launch_bounds__(kWgradThreads) k_conv3_wgrad_tc(
    const __grid_constant__ CUtensorMap xmap, const __grid_constant__ CUtensorMap dymap,
    WgradTcArgs a) {
  using T = ConvTile<TY>;
  using D = DyTile<TY>;
  extern __shared__ __align__(1024) unsigned char sm_raw[];
  unsigned char *sm = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(sm_raw) + 1023) & ~(uintptr_t)1023);
  const int ncc = a.cout / 16;
  const size_t dybytes = (size_t)ncc * D::kChunkBytes;
  const size_t hbytes = (size_t)a.nchunk * T::kChunkBytes;
  const size_t bufbytes = dybytes + hbytes;  // [dy chunks][input halo] per buffer
  uint64_t *full = reinterpret_cast<uint64_t *>(sm + a.bar_off);  // [kWgMaxBufs]
  uint64_t *empty = full + kWgMaxBufs;  // the MMAs done (1) and dy summed (4 warps)
  uint64_t *drain = empty + kWgMaxBufs;  // the MMAs in flight when the CTA ends
  uint32_t *tslot = reinterpret_cast<uint32_t *>(drain + 1);
  __shared__ float s_db[128];  // the CTA's bias-gradient sums
  __shared__ int s_abort;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nunits = 3 * ncc * a.nchunk;
  const int u0 = blockIdx.y * a.units_per_cta;
  const int nunit = min(a.units_per_cta, nunits - u0);
  const int tiles = a.batch * (a.dims[0] / T::kTX) * (a.dims[1] / T::kTY) * (a.dims[2] / T::kTZ);
  const int nmine = (blockIdx.x < tiles && nunit > 0)
                        ? (tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;

  for (int c = tid; c < 128; c += kWgradThreads) s_db[c] = 0.f;
  if (tid == 0) {
    s_abort = 0;
    for (int s = 0; s < a.nbuf; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 5);
    }
    mbar_init(drain, 1);
    fence_mbar_init();
  }
  if (warp == 5) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tslot)),
                 "r"(a.tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  volatile int *abort = &s_abort;
  const uint32_t bytes = (uint32_t)((size_t)ncc * D::kCopies * D::kCopyBytes +
                                    (size_t)a.nchunk * T::kCopies * T::kCopyBytes);

  if (warp == 4 && lane == 0) {
    int issued = 0;
    for (int i = 0; i < nmine && !*abort; ++i) {
      int x0, y0, z0, n;
      T::tile_origin(blockIdx.x + i * gridDim.x, a.dims, x0, y0, z0, n);
      const int b = i % a.nbuf, u = i / a.nbuf;
      if (u > 0 && !role_wait(&empty[b], (uint32_t)(u - 1) & 1u, a.err, abort)) break;
      unsigned char *buf = sm + b * bufbytes;
      mbar_expect_tx(&full[b], bytes);
      for (int g = 0; g < ncc; ++g)
        D::load_chunk(buf + g * D::kChunkBytes, &dymap, g * 16, x0, y0, z0, n, &full[b]);
      for (int c = 0; c < a.nchunk; ++c)
        T::load_chunk(buf + dybytes + (size_t)c * T::kChunkBytes, &xmap, c * 16, x0, y0, z0, n,
                      &full[b]);
      issued = i + 1;
    }
    // the last copy into every buffer has landed before the CTA ends
    for (int i = max(0, issued - a.nbuf); i < issued; ++i)
      mbar_wait(&full[i % a.nbuf], (uint32_t)(i / a.nbuf) & 1u, a.err);
  } else if (warp == 5) {
    // the whole warp runs the loop (uniform branches), one elected lane issues.
    // BF16 x BF16 -> F32, A and B MN-major, M = 128, N = 48
    const uint32_t idesc = idesc_bf16(kUnitCols) | (1u << 15) | (1u << 16);
    const uint32_t kstep_a = (uint32_t)(16 * 32) >> 4;           // the next 16 voxels of dy
    const uint32_t kstep_b = (uint32_t)(2 * T::kRowBytes) >> 4;  // ... of the halo
    // descriptor offsets of the CTA's units (dz, dy chunk cc, input chunk c)
    const int per_dz = ncc * a.nchunk;
    uint32_t aoff[kWgradUnitsPerCta], boff[kWgradUnitsPerCta];
#pragma unroll
    for (int j = 0; j < kWgradUnitsPerCta; ++j) {
      const int u = u0 + min(j, max(nunit - 1, 0)), dz = u / per_dz, rem = u - dz * per_dz;
      const int cc = rem / a.nchunk, c = rem - cc * a.nchunk;
      aoff[j] = (uint32_t)(cc * D::kChunkBytes) >> 4;
      boff[j] = (uint32_t)(c * T::kChunkBytes + T::tap_offset(0, dz, 1, 0)) >> 4;
    }
    int b = 0;           // buffer of tile i
    uint32_t bph = 0;    // its parity
    for (int i = 0; i < nmine; ++i) {
      if (!warp_wait(&full[b], bph, a.err, abort)) break;
      tc_fence_after();
      const unsigned char *buf = sm + b * bufbytes;
      // A: LBO along M (the next 16 rows: dy one voxel row further in y), SBO
      // along K (the next 8 voxels); B: LBO along N (the next 16 columns: the
      // next voxel in x), SBO along K (the next 8-voxel row)
      const uint64_t adesc = sw32_desc_off(buf, (uint32_t)D::kMStride, 256u);
      const uint64_t hdesc = sw32_desc_off(buf + dybytes, 32u, (uint32_t)T::kRowBytes);
      const uint32_t acc0 = i > 0 ? 1u : 0u;
#pragma unroll
      for (int j = 0; j < kWgradUnitsPerCta; ++j) {
        if (j < nunit) {
          const uint64_t ad = adesc + aoff[j], bd = hdesc + boff[j];
          const uint32_t dt = tmem + (uint32_t)(j * kUnitCols);
          mma_el(dt, ad, bd, idesc, acc0);
#pragma unroll
          for (int k = 1; k < 8; ++k)
            mma_el(dt, ad + (uint32_t)k * kstep_a, bd + (uint32_t)k * kstep_b, idesc, 1u);
        }
      }
      // the buffer is free once these MMAs complete
      commit_el(&empty[b]);
      if (++b == a.nbuf) {
        b = 0;
        bph ^= 1u;
      }
    }
    // every MMA issued has completed before the readout and the release of TMEM
    commit_el(drain);
    mbar_wait(drain, 0, a.err);
  } else if (warp < 4) {
    // bias gradient: dy[v][co] summed over the CTA's tiles (the first group's
    // CTAs; the others only release the buffers).  The 16-byte halves of the
    // dy rows (8 channels each; 2 per 16-channel chunk) are spread over the
    // 128 threads: thread t reads half p = t % pairs of rows t / pairs,
    // + 128 / pairs, ...; its 8 sums go to shared memory at the end.
    const bool sum = a.db && blockIdx.y == 0;  // CTA-uniform
    const int pairs = 2 * ncc, tpp = 128 / pairs, p = tid % pairs, r0 = tid / pairs;
    const bool mine = sum && r0 < tpp;
    float bsum[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int i = 0; i < nmine; ++i) {
      const int b = i % a.nbuf;
      bool ok0 = true;
      if (lane == 0) ok0 = role_wait(&full[b], (uint32_t)(i / a.nbuf) & 1u, a.err, abort);
      if (!__shfl_sync(0xffffffffu, ok0, 0)) break;
      if (mine) {
        // the 32-byte swizzle: 16-byte half h of the row at byte offset o sits
        // at half h ^ ((o >> 7) & 1)
        const unsigned char *dy = sm + b * bufbytes + (p >> 1) * D::kChunkBytes;
        const int h = p & 1;
        for (int r = r0; r < 128; r += tpp) {
          const int o = D::own_offset(r);
          const Bf8 v = load8(reinterpret_cast<const bf16 *>(dy + o + ((h ^ ((o >> 7) & 1)) << 4)));
#pragma unroll
          for (int e = 0; e < 8; ++e) bsum[e] += v.v[e];
        }
      }
      __syncwarp();
      if (lane == 0)
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&empty[b]))
                     : "memory");
    }
    if (mine) {
#pragma unroll
      for (int e = 0; e < 8; ++e) atomicAdd(&s_db[p * 8 + e], bsum[e]);
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (a.db && blockIdx.y == 0 && nmine > 0 && tid < a.cout_real) atomicAdd(&a.db[tid], s_db[tid]);
  if (a.part && warp < 2 && (nmine == 0 || *abort)) {
    // no tiles: this CTA's share of the sums is zero
    const int lrow = warp * 32 + lane;
    if (lrow < 48)
      for (int j = 0; j < nunit; ++j)
        for (int g = 0; g < 3; ++g) {
          float4 *dst = reinterpret_cast<float4 *>(
              a.part + ((((size_t)blockIdx.y * gridDim.x + blockIdx.x) * a.units_per_cta + j) * 3 +
                        g) * 768 + lrow * 16);
#pragma unroll
          for (int q = 0; q < 4; ++q) dst[q] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
  }
  if (nmine > 0 && !*abort && warp < 2) {
    // TMEM lane 16 t + co (t = 0, 1, 2): dy shifted by t - 1 rows, output
    // channel 16 cc + co; unit j, column 16 g + e: dx = g - 1, input channel
    // 16 c + e; the tap's y offset is 1 - t
    const int lrow = warp * 32 + lane, t = lrow >> 4, col = lrow & 15;
    const int per_dz = ncc * a.nchunk;
    for (int j = 0; j < nunit; ++j) {
      const int u = u0 + j, dz = u / per_dz, rem = u - dz * per_dz;
      const int cc = rem / a.nchunk, c = rem - cc * a.nchunk;
      const int co = cc * 16 + col;
      for (int g = 0; g < 3; ++g) {
        const int tap = dz * 9 + (2 - t) * 3 + g;
        uint32_t v[16];
        const uint32_t taddr =
            tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(j * kUnitCols + g * 16);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,"
            "%13,%14,%15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
              "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
              "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (a.part) {
          // raw sums, 64 bytes per row: reduced over the CTAs by k_wgrad_reduce
          if (t < 3) {
            float4 *dst = reinterpret_cast<float4 *>(
                a.part + ((((size_t)blockIdx.y * gridDim.x + blockIdx.x) * a.units_per_cta + j) *
                              3 + g) * 768 + lrow * 16);
#pragma unroll
            for (int q = 0; q < 4; ++q)
              dst[q] = make_float4(__uint_as_float(v[4 * q]), __uint_as_float(v[4 * q + 1]),
                                   __uint_as_float(v[4 * q + 2]), __uint_as_float(v[4 * q + 3]));
          }
        } else if (t < 3 && co < a.cout_real) {
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            const int ci = a.ci_map[c * 16 + e];
            const float f = __uint_as_float(v[e]);
            if (ci >= 0 && f != 0.f)
              atomicAdd(&a.dw[((size_t)co * 27 + tap) * a.cin_real + ci], f);
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 5) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(a.tmem_cols)
                 : "memory");
  }
}

// dw += the sum over a group's CTAs of their raw weight-gradient sums.  A block
// takes 32 consecutive (unit, dx tap g, accumulator row, input channel)
// outputs, its 8 warps a slice of the CTAs each (coalesced 128-byte reads); the
// slices are added in shared memory and every dw element has one writer.
constexpr int kReduceSlices = 8;
__global__ void __launch_bounds__(32 * kReduceSlices) k_wgrad_reduce(const float *part, int ctas,
                                                                     int units, WgradTcArgs a) {
  __shared__ float s_sum[kReduceSlices][32];
  const int lane = threadIdx.x & 31, sl = threadIdx.x >> 5;
  const int ncc = a.cout / 16, per_dz = ncc * a.nchunk;
  const long long n = (long long)units * 3 * 768;
  const size_t step = (size_t)a.units_per_cta * 3 * 768;
  for (long long b0 = (long long)blockIdx.x * 32; b0 < n; b0 += (long long)gridDim.x * 32) {
    const long long i = b0 + lane;
    const int e = (int)(i & 15), lrow = (int)((i >> 4) % 48);
    const long long ug = i / 768;
    const int g = (int)(ug % 3), u = (int)(ug / 3);
    float sum = 0.f;
    if (i < n) {
      const int y = u / a.units_per_cta, j = u - y * a.units_per_cta;
      const float *src =
          part + (((size_t)y * ctas * a.units_per_cta + j) * 3 + g) * 768 + lrow * 16 + e;
#pragma unroll 4
      for (int x = sl; x < ctas; x += kReduceSlices) sum += src[(size_t)x * step];
    }
    s_sum[sl][lane] = sum;
    __syncthreads();
    if (sl == 0 && i < n) {
      float tot = 0.f;
#pragma unroll
      for (int k = 0; k < kReduceSlices; ++k) tot += s_sum[k][lane];
      const int t = lrow >> 4, dz = u / per_dz, rem = u - dz * per_dz;
      const int cc = rem / a.nchunk, c = rem - cc * a.nchunk;
      const int co = cc * 16 + (lrow & 15), ci = a.ci_map[c * 16 + e];
      const int tap = dz * 9 + (2 - t) * 3 + g;
      if (co < a.cout_real && ci >= 0) a.dw[((size_t)co * 27 + tap) * a.cin_real + ci] += tot;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// elementwise and resampling kernels (channel slices of channels-last tensors).
// Channel counts and slice offsets are multiples of 16, so a thread moves
// groups of 8 channels (16 bytes).
// ---------------------------------------------------------------------------
// 2x2x2 average pooling: out (X/2, Y/2, Z/2) from in (X, Y, Z)
__global__ void k_pool2(const bf16 *in, int ictot, int ic0, bf16 *out, int octot, int oc0, int c,
                        int batch, int X, int Y, int Z) {
  const int Xo = X / 2, Yo = Y / 2, Zo = Z / 2, c8 = c / 8;
  const unsigned n = (unsigned)batch * Xo * Yo * Zo * c8;
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    unsigned g = i / c8;
    const int k = (int)(i - g * c8) * 8;
    const int x = (int)(g % Xo);
    g /= Xo;
    const int y = (int)(g % Yo);
    g /= Yo;
    const int z = (int)(g % Zo);
    const unsigned s = g / Zo;
    Bf8 acc{};
    for (int d = 0; d < 8; ++d) {
      const size_t q = (((size_t)s * Z + 2 * z + (d >> 2)) * Y + 2 * y + ((d >> 1) & 1)) * X +
                       2 * x + (d & 1);
      const Bf8 t = load8(in + q * ictot + ic0 + k);
#pragma unroll
      for (int e = 0; e < 8; ++e) acc.v[e] += t.v[e];
    }
#pragma unroll
    for (int e = 0; e < 8; ++e) acc.v[e] *= 0.125f;
    const size_t o = (((size_t)s * Zo + z) * Yo + y) * Xo + x;
    store8(out + o * octot + oc0 + k, acc);
  }
}

// gradient of pooling, added to din: din[child] += dout[parent] / 8; then, with
// a gate y, din *= leaky'(y) (din is complete: the gradient of the activation y)
__global__ void k_pool2_bwd_add(const bf16 *dout, int octot, int oc0, bf16 *din, int ictot,
                                int ic0, int c, int batch, int X, int Y, int Z, const bf16 *gy,
                                int gctot, int gc0, float slope) {
  const int c8 = c / 8;
  const unsigned n = (unsigned)batch * X * Y * Z * c8;
  const int Xo = X / 2, Yo = Y / 2, Zo = Z / 2;
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    unsigned g = i / c8;
    const int k = (int)(i - g * c8) * 8;
    const int x = (int)(g % X);
    g /= X;
    const int y = (int)(g % Y);
    g /= Y;
    const int z = (int)(g % Z);
    const unsigned s = g / Z;
    const size_t o = (((size_t)s * Zo + z / 2) * Yo + y / 2) * Xo + x / 2;
    const size_t q = (((size_t)s * Z + z) * Y + y) * X + x;
    Bf8 d = load8(din + q * ictot + ic0 + k);
    const Bf8 t = load8(dout + o * octot + oc0 + k);
#pragma unroll
    for (int e = 0; e < 8; ++e) d.v[e] = __bfloat162float(__float2bfloat16_rn(d.v[e] + 0.125f * t.v[e]));
    if (gy) gate8(d, gy + q * gctot + gc0 + k, slope);
    store8(din + q * ictot + ic0 + k, d);
  }
}

// nearest-neighbour upsampling by 2: out (2X, 2Y, 2Z)
__global__ void k_up2(const bf16 *in, int ictot, int ic0, bf16 *out, int octot, int oc0, int c,
                      int batch, int X, int Y, int Z) {
  const int X2 = 2 * X, Y2 = 2 * Y, Z2 = 2 * Z, c8 = c / 8;
  const unsigned n = (unsigned)batch * X2 * Y2 * Z2 * c8;
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    unsigned g = i / c8;
    const int k = (int)(i - g * c8) * 8;
    const int x = (int)(g % X2);
    g /= X2;
    const int y = (int)(g % Y2);
    g /= Y2;
    const int z = (int)(g % Z2);
    const unsigned s = g / Z2;
    const size_t q = (((size_t)s * Z + z / 2) * Y + y / 2) * X + x / 2;
    const size_t o = (((size_t)s * Z2 + z) * Y2 + y) * X2 + x;
    *reinterpret_cast<uint4 *>(out + o * octot + oc0 + k) =
        *reinterpret_cast<const uint4 *>(in + q * ictot + ic0 + k);
  }
}

// gradient of upsampling: dout (X, Y, Z) = sum of the 8 children in din (2X...);
// with a gate y, dout *= leaky'(y)
__global__ void k_up2_bwd(const bf16 *din, int ictot, int ic0, bf16 *dout, int octot, int oc0,
                          int c, int batch, int X, int Y, int Z, const bf16 *gy, int gctot,
                          int gc0, float slope) {
  const int c8 = c / 8;
  const unsigned n = (unsigned)batch * X * Y * Z * c8;
  const int X2 = 2 * X, Y2 = 2 * Y;
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    unsigned g = i / c8;
    const int k = (int)(i - g * c8) * 8;
    const int x = (int)(g % X);
    g /= X;
    const int y = (int)(g % Y);
    g /= Y;
    const int z = (int)(g % Z);
    const unsigned s = g / Z;
    Bf8 acc{};
    for (int d = 0; d < 8; ++d) {
      const size_t q = (((size_t)s * 2 * Z + 2 * z + (d >> 2)) * Y2 + 2 * y + ((d >> 1) & 1)) *
                           X2 + 2 * x + (d & 1);
      const Bf8 t = load8(din + q * ictot + ic0 + k);
#pragma unroll
      for (int e = 0; e < 8; ++e) acc.v[e] += t.v[e];
    }
    const size_t o = (((size_t)s * Z + z) * Y + y) * X + x;
    if (gy) {
#pragma unroll
      for (int e = 0; e < 8; ++e) acc.v[e] = __bfloat162float(__float2bfloat16_rn(acc.v[e]));
      gate8(acc, gy + o * gctot + gc0 + k, slope);
    }
    store8(dout + o * octot + oc0 + k, acc);
  }
}

// 1x1 output head (c -> 1, FP32 weights) fused with the MSE loss and its
// gradient.  pred = w . h + b; with a target: loss += (pred - t)^2,
// dpred = 2 (pred - t) / nvox, dh = dpred * w (BF16) * leaky'(h) (h is the
// activation output of the last convolution), dw += dpred * h, db += dpred.
// One thread per voxel; h rows are 16-channel multiples (hctot <= 16 here).
__global__ void k_head(const bf16 *h, int hctot, int c, const float *w, const float *b,
                       long long nvox, float *pred, const float *target, bf16 *dh,
                       float *dw, float *db, float *loss, float over_weight, float slope) {
  __shared__ float red[256];
  __shared__ float redw[16][33];
  float l = 0.f, gb = 0.f;
  float gw[16] = {};
  float wk[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) wk[k] = k < c ? w[k] : 0.f;
  const float b0 = b[0];
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nvox;
       v += (long long)gridDim.x * blockDim.x) {
    const Bf8 h0 = load8(h + v * hctot), h1 = load8(h + v * hctot + 8);
    float hv[16];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      hv[k] = h0.v[k];
      hv[k + 8] = h1.v[k];
    }
    float p = b0;
#pragma unroll
    for (int k = 0; k < 16; ++k)
      if (k < c) p = fmaf(wk[k], hv[k], p);
    if (pred) pred[v] = p;
    if (target) {
      const float diff = p - target[v];
      // squared errors of predictions above the target (too neutral) weigh
      // over_weight: those fronts recover one cell per plain iteration
      const float wl = diff > 0.f ? over_weight : 1.f;
      l += wl * diff * diff;
      const float g = 2.f * wl * diff / (float)nvox;
      gb += g;
      Bf8 d0, d1;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        // BF16 gradient, then the activation derivative (two roundings, as a
        // stored gradient followed by the activation backward)
        float a0 = k < c ? __bfloat162float(__float2bfloat16_rn(g * wk[k])) : 0.f;
        float a1 = k + 8 < c ? __bfloat162float(__float2bfloat16_rn(g * wk[k + 8])) : 0.f;
        if (!(hv[k] > 0.f)) a0 *= slope;
        if (!(hv[k + 8] > 0.f)) a1 *= slope;
        d0.v[k] = a0;
        d1.v[k] = a1;
      }
      store8(dh + v * hctot, d0);
      store8(dh + v * hctot + 8, d1);
#pragma unroll
      for (int k = 0; k < 16; ++k)
        if (k < c) gw[k] = fmaf(g, hv[k], gw[k]);
    }
  }
  if (!target) return;
  // block reductions: loss, db, dw
  red[threadIdx.x] = l;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss, red[0]);
  __syncthreads();
  red[threadIdx.x] = gb;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(db, red[0]);
  for (int k = 0; k < c; ++k) {
    float s = gw[k];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) redw[k][threadIdx.x >> 5] = s;
  }
  __syncthreads();
  if (threadIdx.x < c) {
    float s = 0.f;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += redw[threadIdx.x][i];
    atomicAdd(&dw[threadIdx.x], s);
  }
}

// Pack FP32 master weights W[co][tap][ci] into the K-step operand layout of
// k_conv3_tc: [tap][chunk][row][16] with 16-byte halves swapped in rows 4-7 of
// every 8 (the 32-byte swizzle).  Forward: rows = output channels, K =
// storage input channels.  Input gradient (flip = 1): rows = storage input
// channels, K = output channels, taps mirrored (tap -> 26 - tap).
struct PackArgs {
  const float *w;       // [cout][27][cin_real]
  bf16 *out;
  int cout, cin_real;
  int rows, kchan;      // packed rows and K channels (multiples of 16)
  const int *ci_of_storage;  // storage input channel -> real ci or -1 (length cin storage)
  int flip;
  int xf;               // x-folded layout of k_conv3_xf: [dz][dy][chunk][dx][row][16]
};

// k_conv3_xf serves convolutions whose three x taps fit one MMA's N (<= 256)
__host__ __device__ inline bool conv_xf(int npad) { return 3 * npad <= 256; }

// element i of a packed operand
__device__ __forceinline__ void pack_element(const PackArgs &a, long long i) {
  const int nchunk = a.kchan / 16;
  {
    long long g = i;
    const int e = (int)(g % 16);
    g /= 16;
    const int r = (int)(g % a.rows);
    g /= a.rows;
    const int ch = (int)(g % nchunk);
    const int tap = (int)(g / nchunk);
    const int kc = ch * 16 + e;  // K channel
    float v = 0.f;
    if (!a.flip) {
      const int co = r, ci = a.ci_of_storage[kc];
      if (co < a.cout && ci >= 0) v = a.w[((size_t)co * 27 + tap) * a.cin_real + ci];
    } else {
      const int co = kc, ci = a.ci_of_storage[r];
      if (co < a.cout && ci >= 0) v = a.w[((size_t)co * 27 + (26 - tap)) * a.cin_real + ci];
    }
    if (a.xf) {
      // K step (dz, dy, chunk) holds the rows of its three x taps: dx-major
      const size_t step = (size_t)(tap / 3) * nchunk + ch;
      const int rr = (tap % 3) * a.rows + r;
      const int half = (e >> 3) ^ ((rr >> 2) & 1);
      a.out[(step * 3 * a.rows + rr) * 16 + half * 8 + (e & 7)] = __float2bfloat16_rn(v);
    } else {
      const size_t step = (size_t)tap * nchunk + ch;
      const int half = (e >> 3) ^ ((r >> 2) & 1);
      a.out[(step * a.rows + r) * 16 + half * 8 + (e & 7)] = __float2bfloat16_rn(v);
    }
  }
}

__global__ void k_pack(PackArgs a) {
  const long long n = 27LL * (a.kchan / 16) * a.rows * 16;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    pack_element(a, i);
}

// every layer's packing in one launch: job k covers elements [begin, begin +
// count) of the whole; a job with a bias destination pads the FP32 bias to
// npad (zero beyond cout), the others pack one operand
struct PackJob {
  PackArgs a;
  long long begin, count;
  const float *bias;  // null: a weight job
  float *bias_pad;
};
__global__ void k_pack_all(const PackJob *jobs, int njobs, long long total) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    int k = 0;
    while (k + 1 < njobs && jobs[k + 1].begin <= i) ++k;
    const PackJob &jb = jobs[k];
    const long long r = i - jb.begin;
    if (jb.bias) jb.bias_pad[r] = r < jb.a.cout ? jb.bias[r] : 0.f;
    else pack_element(jb.a, r);
  }
}

// Adam on FP32 master parameters
__global__ void k_adam(float *p, const float *g, float *m, float *v, long long n, float lr,
                       float b1, float b2, float eps, float c1, float c2) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// input features -> the 16-channel BF16 input tensor (channels 3..15 zero)
__global__ void k_input(const float *f, bf16 *x, unsigned nvox) {
  // one voxel (16 storage channels, 32 bytes) per thread
  for (unsigned v = blockIdx.x * blockDim.x + threadIdx.x; v < nvox; v += gridDim.x * blockDim.x) {
    __align__(16) bf16 o[16];
#pragma unroll
    for (int k = 0; k < 16; ++k)
      o[k] = __float2bfloat16_rn(k < kFeatures ? f[(size_t)v * kFeatures + k] : 0.f);
    uint4 *d = reinterpret_cast<uint4 *>(x + (size_t)v * 16);
    d[0] = reinterpret_cast<const uint4 *>(o)[0];
    d[1] = reinterpret_cast<const uint4 *>(o)[1];
  }
}

// Features of one grid (cube order, Z = ix slowest), each (raw - mean) / scale:
//  0: log10 n_H
//  1: log10 sum_i L_i / (4 pi r_i^2), r clamped to half a cell
//  2: log10 sum_i L_i / (4 pi alpha R_i), R_i = integral of n_H^2 r^2 dr along
//     the ray from source i to the cell centre (the Stromgren condition: a
//     source ionizes a ray up to where its recombinations use up L_i / 4 pi).
//     The integral is a midpoint sum over ceil(r / (cell / 2)) steps with n_H
//     of the cell that holds each sample point, in FP32 cell units with n_H in
//     units of its grid mean, so the march costs a few FP32 operations per
//     step.  Explicitly rounded operations (no contraction) make the sample
//     cells reproducible by the same float32 sum on the host.
struct FeatureArgs {
  const double *nH;
  const float *nrel;    // n_H / n_ref (FP32), cube order
  float *out;
  int dims[3];          // X (iz), Y (iy), Z (ix)
  int n3[3];            // cells along ix, iy, iz
  double origin[3];     // box corner along ix, iy, iz
  double cell[3];       // cell size along ix, iy, iz
  const double *src;    // [nsrc][4]: position (x, y, z), L
  int nsrc;
  double alpha, nref;
  float norm[2 * kFeatures];  // (mean, scale) per channel
  // 0: all three channels; 1: raw log10 of channel 2 only (out holds one
  // float per cell); 2: channels 0-1 here, channel 2 interpolated
  // (trilinear, in log10) from `ratio`, a raw mode-1 field on the grid
  // coarser by `rf` per axis (rm cells along ix, iy, iz)
  int mode;
  const float *ratio;
  int rm[3];
  int rf;
};

// channel 2 of a fine cell from the coarse raw field: coarse cell centres
// sit at fine coordinate (c + 0.5) rf - 0.5; outside them the edge value holds
__device__ float ratio_from_coarse(const FeatureArgs &a, const int i3[3]) {
  int lo[3], hi[3];
  float t[3];
  for (int k = 0; k < 3; ++k) {
    float u = ((float)i3[k] + 0.5f) / (float)a.rf - 0.5f;
    u = fminf(fmaxf(u, 0.f), (float)(a.rm[k] - 1));
    lo[k] = min((int)u, a.rm[k] - 1);
    hi[k] = min(lo[k] + 1, a.rm[k] - 1);
    t[k] = u - (float)lo[k];
  }
  float acc = 0.f;
  for (int c = 0; c < 8; ++c) {
    const int j0 = (c & 4) ? hi[0] : lo[0], j1 = (c & 2) ? hi[1] : lo[1],
              j2 = (c & 1) ? hi[2] : lo[2];
    const float w = ((c & 4) ? t[0] : 1.f - t[0]) * ((c & 2) ? t[1] : 1.f - t[1]) *
                    ((c & 1) ? t[2] : 1.f - t[2]);
    acc += w * a.ratio[((long long)j0 * a.rm[1] + j1) * a.rm[2] + j2];
  }
  return acc;
}

__global__ void k_nrel(const double *nH, float *nrel, long long n, double inv_nref) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    nrel[i] = (float)__dmul_rn(nH[i], inv_nref);
}

__global__ void k_features(FeatureArgs a) {
  const long long nvox = (long long)a.dims[0] * a.dims[1] * a.dims[2];
  const double hmin = fmin(a.cell[0], fmin(a.cell[1], a.cell[2]));
  const double rmin = 0.5 * hmin;
  // march in units of cells along each axis; step length in units of hmin
  const float hstep = 0.5f;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nvox;
       v += (long long)gridDim.x * blockDim.x) {
    const int i3[3] = {(int)(v / ((long long)a.dims[0] * a.dims[1])),
                       (int)((v / a.dims[0]) % a.dims[1]), (int)(v % a.dims[0])};
    double flux = 0., strom = 0.;
    for (int s = 0; s < a.nsrc; ++s) {
      const double *S = a.src + 4 * s;
      double dm[3], sc[3];
      float dc[3];
      for (int k = 0; k < 3; ++k) {
        const double p = __dadd_rn(a.origin[k], __dmul_rn((double)i3[k] + 0.5, a.cell[k]));
        dm[k] = __dsub_rn(p, S[k]);
        sc[k] = __ddiv_rn(__dsub_rn(S[k], a.origin[k]), a.cell[k]);  // source in cell units
        dc[k] = (float)__ddiv_rn(dm[k], a.cell[k]);                  // ray in cell units
      }
      const double r = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dm[0], dm[0]),
                                                      __dmul_rn(dm[1], dm[1])),
                                            __dmul_rn(dm[2], dm[2])));
      const double rc = fmax(r, rmin);
      flux += S[3] / (4. * 3.141592653589793 * rc * rc);
      if (a.mode == 2) continue;  // channel 2 comes from the coarse field
      const float rh = (float)__ddiv_rn(r, hmin);  // length in units of hmin
      const int nstep = max(1, (int)ceilf(__fdiv_rn(rh, hstep)));
      const float inv = __frcp_rn((float)nstep);
      const float sf[3] = {(float)sc[0], (float)sc[1], (float)sc[2]};
      float col = 0.f;
      for (int k = 0; k < nstep; ++k) {
        const float t = __fmul_rn(__fadd_rn((float)k, 0.5f), inv);
        int c3[3];
        for (int m = 0; m < 3; ++m) {
          const int ci = (int)floorf(__fadd_rn(sf[m], __fmul_rn(t, dc[m])));
          c3[m] = min(max(ci, 0), a.n3[m] - 1);
        }
        const float n = a.nrel[((long long)c3[0] * a.n3[1] + c3[1]) * a.n3[2] + c3[2]];
        const float rr = __fmul_rn(t, rh);
        col = __fadd_rn(col, __fmul_rn(__fmul_rn(n, n), __fmul_rn(rr, rr)));
      }
      // R = sum n^2 r^2 dr in SI: (n_ref^2) (hmin^3) col * (rh / nstep)
      const double R = (double)col * ((double)rh * (double)inv) * a.nref * a.nref * hmin * hmin *
                       hmin;
      strom += S[3] / (4. * 3.141592653589793 * a.alpha * fmax(R, 1e-300));
    }
    const double lratio = log10(fmin(fmax(strom, 1e-30), 1e30));
    if (a.mode == 1) {
      a.out[v] = (float)lratio;
      continue;
    }
    float *o = a.out + kFeatures * v;
    o[0] = (float)((log10(a.nH[v]) - a.norm[0]) / a.norm[1]);
    o[1] = (float)((log10(fmax(flux, 1e-300)) - a.norm[2]) / a.norm[3]);
    const float l2 = a.mode == 2 ? ratio_from_coarse(a, i3) : (float)lratio;
    o[2] = (l2 - a.norm[4]) / a.norm[5];
  }
}

// block mean of an FP64 cube (dims of the source, cube order) by `f` per axis
__global__ void k_block_mean(const double *src, double *dst, int n0, int n1, int n2, int f) {
  const int m0 = n0 / f, m1 = n1 / f, m2 = n2 / f;
  const long long n = (long long)m0 * m1 * m2;
  const double inv = 1. / ((double)f * f * f);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int c2 = (int)(i % m2), c1 = (int)((i / m2) % m1), c0 = (int)(i / ((long long)m1 * m2));
    double s = 0.;
    for (int a = 0; a < f; ++a)
      for (int b = 0; b < f; ++b)
        for (int d = 0; d < f; ++d)
          s += src[((long long)(c0 * f + a) * n1 + (c1 * f + b)) * n2 + (c2 * f + d)];
    dst[i] = s * inv;
  }
}

// nearest-neighbour upsampling of an FP32 cube by `f` per axis
__global__ void k_upsample_nearest(const float *src, float *dst, int n0, int n1, int n2, int f) {
  const int M0 = n0 * f, M1 = n1 * f, M2 = n2 * f;
  const long long n = (long long)M0 * M1 * M2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int c2 = (int)(i % M2), c1 = (int)((i / M2) % M1), c0 = (int)(i / ((long long)M1 * M2));
    dst[i] = src[((long long)(c0 / f) * n1 + c1 / f) * n2 + c2 / f];
  }
}

// x_H = 10^clamp(pred, lo, 0) as FP64 (the engine's field)
__global__ void k_to_xH(const float *pred, double *xH, long long n, float lo) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    xH[i] = exp10((double)fminf(fmaxf(pred[i], lo), 0.f));
}

// ---------------------------------------------------------------------------
// host side: the network
// ---------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int get_encoder(EncodeTiledFn *fn) {
  static std::mutex mu;
  static EncodeTiledFn cached = nullptr;
  std::lock_guard<std::mutex> lock(mu);
  if (!cached) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    UN_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || !p)
      return fail(CMI_ERR_NOT_SUPPORTED, "cuTensorMapEncodeTiled is not available");
    cached = reinterpret_cast<EncodeTiledFn>(p);
  }
  *fn = cached;
  return CMI_OK;
}

inline int pad16(int c) { return (c + 15) / 16 * 16; }

// a channel slice of an activation tensor
struct Slice {
  bf16 *base = nullptr;
  int ctot = 0, c0 = 0, c = 0;  // storage channels of the tensor, first channel, count (x16)
};

struct Layer {
  int cout = 0, cin_real = 0, npad = 0, kin = 0;  // kin: storage input channels
  std::vector<int> ci_of_storage;                 // kin entries
  size_t w_off = 0, b_off = 0;                    // into the FP32 parameter arrays
  bf16 *wf = nullptr, *wd = nullptr;              // packed forward / input-gradient weights
  int *d_map = nullptr;
  float *bias_pad = nullptr;                      // [npad] BF16-layer bias (FP32)
};

struct Level {
  int X = 0, Y = 0, Z = 0;
};

}  // namespace cmiu

using namespace cmiu;

struct cmi_unet {
  int device = 0;
  int ch[3] = {12, 24, 48};
  float slope = 0.1f;
  cudaStream_t stream = nullptr;
  std::vector<Layer> L;  // 10 convolutions
  size_t nparams = 0;
  size_t head_w = 0, head_b = 0;
  float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  long long adam_t = 0;
  uint32_t *d_err = nullptr;
  float *d_loss = nullptr;
  float *wg_part = nullptr;    // the weight gradient's per-CTA sums (64 MB, allocated once)
  size_t wg_part_floats = 0;
  // activation buffers for the current (batch, dims)
  int batch = 0, dims[3] = {0, 0, 0};
  std::vector<void *> bufs;
  // tensors
  bf16 *X0 = nullptr, *E1A = nullptr, *CAT1 = nullptr, *P1 = nullptr, *E2A = nullptr,
       *CAT2 = nullptr, *P2 = nullptr, *BA = nullptr, *BB = nullptr, *D2A = nullptr,
       *D2B = nullptr, *D1A = nullptr, *D1B = nullptr;
  bf16 *gE1A = nullptr, *gCAT1 = nullptr, *gP1 = nullptr, *gE2A = nullptr, *gCAT2 = nullptr,
       *gP2 = nullptr, *gBA = nullptr, *gBB = nullptr, *gD2A = nullptr, *gD2B = nullptr,
       *gD1A = nullptr, *gD1B = nullptr;
  float *pred = nullptr, *feat = nullptr;
  double *d_src = nullptr;  // sources of the features kernel
  size_t src_cap = 0;
  float *d_nrel = nullptr;  // n_H / n_ref for the features kernel
  size_t nrel_cap = 0;
  double *d_ncoarse = nullptr;  // block-mean n_H of the coarse ratio pass
  size_t ncoarse_cap = 0;
  float *d_ratio = nullptr;     // raw coarse channel 2
  size_t ratio_cap = 0;
  float over_weight = 1.f;      // loss weight of predictions above the target
  bool packed = false;
  // CUDA graphs of the launch sequences whose arguments do not change between
  // calls: the forward layers and the backward layers (for the current
  // activation buffers), the weight packing (for the life of the network)
  cudaGraphExec_t gx_fwd = nullptr, gx_bwd = nullptr, gx_pack = nullptr;
  void *d_jobs = nullptr;  // the packing jobs of every layer (k_pack_all)
  int njobs = 0;
  long long jobs_total = 0;
};

namespace cmiu {

int dev_zero_alloc(void **p, size_t bytes) {
  UN_CUDA(cudaMalloc(p, bytes));
  UN_CUDA(cudaMemset(*p, 0, bytes));
  return CMI_OK;
}

void drop_graph(cudaGraphExec_t *g) {
  if (*g) cudaGraphExecDestroy(*g);
  *g = nullptr;
}

// the graphs that name the activation buffers go with them
void free_bufs(cmi_unet *u) {
  drop_graph(&u->gx_fwd);
  drop_graph(&u->gx_bwd);
  for (void *b : u->bufs) cudaFree(b);
  u->bufs.clear();
  u->batch = 0;
}

// body() (a sequence of launches on u->stream) is captured into *exec on the
// first call and replayed from then on: the per-launch host work (tensor maps,
// attributes, occupancy) is done once
template <class F>
int graph_run(cmi_unet *u, cudaGraphExec_t *exec, F &&body) {
  if (!*exec) {
    UN_CUDA(cudaStreamBeginCapture(u->stream, cudaStreamCaptureModeRelaxed));
    const int rc = body();
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(u->stream, &g);
    if (rc != CMI_OK) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (ce != cudaSuccess)
      return fail(CMI_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
    const cudaError_t ie = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
      *exec = nullptr;
      return fail(CMI_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ie));
    }
  }
  UN_CUDA(cudaGraphLaunch(*exec, u->stream));
  return CMI_OK;
}

int alloc_t(cmi_unet *u, bf16 **t, long long nvox, int ctot) {
  void *p = nullptr;
  UN_TRY(dev_zero_alloc(&p, sizeof(bf16) * (size_t)nvox * ctot));
  u->bufs.push_back(p);
  *t = static_cast<bf16 *>(p);
  return CMI_OK;
}

// storage channels of the tensors
struct Chans {
  int c1, c2, c3, s1, s2, s3, cat1, cat2;
};
Chans chans(const cmi_unet *u) {
  Chans c{};
  c.c1 = u->ch[0];
  c.c2 = u->ch[1];
  c.c3 = u->ch[2];
  c.s1 = pad16(c.c1);
  c.s2 = pad16(c.c2);
  c.s3 = pad16(c.c3);
  c.cat1 = c.s2 + c.s1;  // [up from level 2 | skip of level 1]
  c.cat2 = c.s3 + c.s2;  // [up from level 3 | skip of level 2]
  return c;
}

// the weight gradient's per-CTA scratch: allocated once, before any graph that
// names it is recorded (every launch configuration of this network fits)
int ensure_wg_part(cmi_unet *u) {
  if (u->wg_part) return CMI_OK;
  const size_t n = (size_t)16 << 20;
  UN_CUDA(cudaMalloc(&u->wg_part, n * sizeof(float)));
  u->wg_part_floats = n;
  return CMI_OK;
}

int ensure_buffers(cmi_unet *u, int batch, const int dims[3]) {
  UN_TRY(ensure_wg_part(u));
  if (u->batch == batch && u->dims[0] == dims[0] && u->dims[1] == dims[1] &&
      u->dims[2] == dims[2])
    return CMI_OK;
  free_bufs(u);
  const Chans c = chans(u);
  const long long v1 = (long long)batch * dims[0] * dims[1] * dims[2];
  const long long v2 = v1 / 8, v3 = v1 / 64;
  UN_TRY(alloc_t(u, &u->X0, v1, 16));
  UN_TRY(alloc_t(u, &u->E1A, v1, c.s1));
  UN_TRY(alloc_t(u, &u->CAT1, v1, c.cat1));
  UN_TRY(alloc_t(u, &u->P1, v2, c.s1));
  UN_TRY(alloc_t(u, &u->E2A, v2, c.s2));
  UN_TRY(alloc_t(u, &u->CAT2, v2, c.cat2));
  UN_TRY(alloc_t(u, &u->P2, v3, c.s2));
  UN_TRY(alloc_t(u, &u->BA, v3, c.s3));
  UN_TRY(alloc_t(u, &u->BB, v3, c.s3));
  UN_TRY(alloc_t(u, &u->D2A, v2, c.s2));
  UN_TRY(alloc_t(u, &u->D2B, v2, c.s2));
  UN_TRY(alloc_t(u, &u->D1A, v1, c.s1));
  UN_TRY(alloc_t(u, &u->D1B, v1, c.s1));
  UN_TRY(alloc_t(u, &u->gE1A, v1, c.s1));
  UN_TRY(alloc_t(u, &u->gCAT1, v1, c.cat1));
  UN_TRY(alloc_t(u, &u->gP1, v2, c.s1));
  UN_TRY(alloc_t(u, &u->gE2A, v2, c.s2));
  UN_TRY(alloc_t(u, &u->gCAT2, v2, c.cat2));
  UN_TRY(alloc_t(u, &u->gP2, v3, c.s2));
  UN_TRY(alloc_t(u, &u->gBA, v3, c.s3));
  UN_TRY(alloc_t(u, &u->gBB, v3, c.s3));
  UN_TRY(alloc_t(u, &u->gD2A, v2, c.s2));
  UN_TRY(alloc_t(u, &u->gD2B, v2, c.s2));
  UN_TRY(alloc_t(u, &u->gD1A, v1, c.s1));
  UN_TRY(alloc_t(u, &u->gD1B, v1, c.s1));
  void *p = nullptr;
  UN_TRY(dev_zero_alloc(&p, sizeof(float) * (size_t)v1));
  u->bufs.push_back(p);
  u->pred = static_cast<float *>(p);
  UN_TRY(dev_zero_alloc(&p, sizeof(float) * kFeatures * (size_t)v1));
  u->bufs.push_back(p);
  u->feat = static_cast<float *>(p);
  u->batch = batch;
  for (int a = 0; a < 3; ++a) u->dims[a] = dims[a];
  return CMI_OK;
}

int grid_for(long long n, int threads = 256) {
  return (int)std::min<long long>((n + threads - 1) / threads, 148LL * 16);
}

// tensor map of a slice: dims (channels, X, Y, Z, batch); boxes of box_c
// channels (16: 32-byte voxel rows with the 32-byte swizzle; 8: unswizzled
// 16-byte rows) x box_x/y/z voxels
int make_map_box(CUtensorMap *map, const Slice &s, int batch, const int dims[3], int box_c,
                 int box_x, int box_y, int box_z) {
  EncodeTiledFn enc;
  UN_TRY(get_encoder(&enc));
  const cuuint64_t gdim[5] = {(cuuint64_t)s.c, (cuuint64_t)dims[0], (cuuint64_t)dims[1],
                              (cuuint64_t)dims[2], (cuuint64_t)batch};
  const cuuint64_t row = (cuuint64_t)s.ctot * sizeof(bf16);
  const cuuint64_t gstride[4] = {row, row * dims[0], row * dims[0] * dims[1],
                                 row * dims[0] * dims[1] * dims[2]};
  const cuuint32_t box[5] = {(cuuint32_t)box_c, (cuuint32_t)box_x, (cuuint32_t)box_y,
                             (cuuint32_t)box_z, 1};
  const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, (void *)(s.base + s.c0), gdim,
                         gstride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         box_c == 16 ? CU_TENSOR_MAP_SWIZZLE_32B : CU_TENSOR_MAP_SWIZZLE_NONE,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(CMI_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return CMI_OK;
}

// the tile shape of a grid: 8 x 16 x 1 when Y is a multiple of 16, else 8 x 8 x 2
int tile_y(const int dims[3]) {
  if (dims[0] % 8 == 0 && dims[1] % 16 == 0) return 16;
  if (dims[0] % 8 == 0 && dims[1] % 8 == 0 && dims[2] % 2 == 0) return 8;
  return 0;
}

// one y-copy of the input halo of a tile (box 10 x rows x slices voxels)
template <int TY, int KZ = 1>
int make_halo_map(CUtensorMap *map, const Slice &s, int batch, const int dims[3]) {
  using T = ConvTile<TY, KZ>;
  return make_map_box(map, s, batch, dims, 16, T::kHX, T::kCopyRows, T::kHZ);
}

// dynamic shared memory a CTA of kernel f may take (the opt-in limit less the
// kernel's static shared memory)
template <typename F>
int smem_optin(cmi_unet *u, F f, int *bytes) {
  int dev = 0;
  UN_CUDA(cudaGetDevice(&dev));
  UN_CUDA(cudaDeviceGetAttribute(bytes, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa{};
  UN_CUDA(cudaFuncGetAttributes(&fa, f));
  *bytes -= (int)fa.sharedSizeBytes;
  return CMI_OK;
}

// shared memory of a convolution CTA: halo buffers, weight stages, bias, barriers
struct ConvPlan {
  int nbuf = 0, wstages = 0;
  size_t smem = 0;
};
template <int TY, int KZ>
ConvPlan conv_plan(int nchunk, int npad, int optin) {
  using T = ConvTile<TY, KZ>;
  const size_t tbytes = (size_t)nchunk * npad * 32;
  auto smem_for = [&](int nbuf, int stages) {
    return 1024 + (size_t)stages * tbytes + (size_t)nbuf * nchunk * T::kChunkBytes +
           (size_t)npad * 4 + (2 * kMaxWStages + 9) * 8 + 16;
  };
  auto stages_for = [&](int nbuf) {
    const size_t fixed = smem_for(nbuf, 0);
    return fixed >= (size_t)optin ? 0 : (int)std::min<size_t>(27, (optin - fixed) / tbytes);
  };
  // weights resident (27 stages) when they fit beside two halo buffers, else a
  // ring of as many tap stages as fit (at least 4), else one halo buffer
  ConvPlan p;
  p.nbuf = stages_for(2) >= 4 ? 2 : 1;
  p.wstages = stages_for(p.nbuf);
  p.smem = smem_for(p.nbuf, p.wstages);
  return p;
}

template <int TY, int KZ>
int conv_launch(cmi_unet *u, const Slice &in, const bf16 *wpack, const float *bias,
                const Slice &out, int act, int batch, const int dims[3], int optin,
                const Slice *gate) {
  using T = ConvTile<TY, KZ>;
  CUtensorMap map;
  UN_TRY((make_halo_map<TY, KZ>(&map, in, batch, dims)));
  ConvArgs a{};
  a.wpack = wpack;
  a.bias = bias;
  a.out = out.base;
  a.out_ctot = out.ctot;
  a.out_c0 = out.c0;
  a.npad = out.c;
  a.nchunk = in.c / 16;
  for (int k = 0; k < 3; ++k) a.dims[k] = dims[k];
  a.batch = batch;
  a.act = act;
  a.slope = u->slope;
  if (gate) {
    a.gate = gate->base;
    a.gate_ctot = gate->ctot;
    a.gate_c0 = gate->c0;
  }
  a.err = u->d_err;
  const ConvPlan p = conv_plan<TY, KZ>(a.nchunk, a.npad, optin);
  if (p.wstages < 2)
    return fail(CMI_ERR_NOT_SUPPORTED, "convolution: weights of one tap (%d B) do not fit",
                a.nchunk * a.npad * 32);
  a.nbuf = p.nbuf;
  a.wstages = p.wstages;
  auto kern = k_conv3_tc<TY, KZ>;
  // the kernel's limit is the device's whole opt-in size, the same for every
  // launch: a launch captured in a graph must stay valid whatever limit a
  // later launch of the same kernel would otherwise have set
  UN_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
  int per_sm = 0;
  UN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kConvThreads, p.smem));
  // TMEM: two accumulator sets of a CTA, at most 512 columns per SM
  const int acols = a.npad <= 32 ? 32 : a.npad <= 64 ? 64 : a.npad <= 128 ? 128 : 256;
  per_sm = std::max(1, std::min(per_sm, 512 / (2 * KZ * acols)));
  int sms = 0, dev = 0;
  UN_CUDA(cudaGetDevice(&dev));
  UN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int tiles = T::num_tiles(batch, dims);
  const int grid = std::max(1, std::min(tiles, per_sm * sms));
  kern<<<grid, kConvThreads, p.smem, u->stream>>>(map, a);
  UN_CUDA(cudaGetLastError());
  return CMI_OK;
}

// the deepest tile (KZ z slices) whose two accumulator sets fit the tensor
// memory, whose weights stay resident beside two halo buffers and that still
// gives every SM a tile
template <int KZ>
bool conv_deep_ok(const Slice &in, const Slice &out, int batch, const int dims[3], int optin,
                  int sms) {
  using T = ConvTile<16, KZ>;
  const int acols = out.c <= 32 ? 32 : out.c <= 64 ? 64 : out.c <= 128 ? 128 : 256;
  if (dims[2] % KZ || 2 * KZ * acols > 512) return false;
  const ConvPlan p = conv_plan<16, KZ>(in.c / 16, out.c, optin);
  return p.wstages == 27 && p.nbuf == 2 && T::num_tiles(batch, dims) >= sms;
}

// shared memory of an x-folded convolution CTA: the weights resident (9 tap
// rows) beside two input buffers when they fit, else a ring of stages of kq K
// steps (the largest divisor of nchunk that leaves at least 4 stages, or at
// least 2 with one input buffer)
struct XfPlan {
  int nbuf = 0, wstages = 0, kq = 0;
  size_t smem = 0;
};
template <int KZ>
XfPlan xf_plan(int nchunk, int npad, int optin) {
  using T = XTile<KZ>;
  const size_t bbytes = (size_t)3 * npad * 32;
  auto smem_for = [&](int nbuf, int stages, int kq) {
    return 1024 + (size_t)stages * kq * bbytes + (size_t)nbuf * nchunk * T::kChunkBytes +
           (size_t)npad * 4 + (2 * kMaxWStages + 2 * kMaxInBufs + 5) * 8 + 16;
  };
  XfPlan p;
  if (smem_for(2, 9, nchunk) <= (size_t)optin) {
    // resident weights and as many input buffers as fit
    p.nbuf = 2;
    while (p.nbuf < kMaxInBufs && smem_for(p.nbuf + 1, 9, nchunk) <= (size_t)optin) ++p.nbuf;
    p.wstages = 9;
    p.kq = nchunk;
  } else {
    for (int nbuf = 2; nbuf >= 1 && !p.kq; --nbuf) {
      const int need = nbuf == 2 ? 4 : 2;
      for (int kq = nchunk; kq >= 1; --kq) {
        if (nchunk % kq) continue;
        const size_t fixed = smem_for(nbuf, 0, kq);
        if (fixed >= (size_t)optin) break;
        const int stages = (int)std::min<size_t>(std::min(kMaxWStages, 9 * nchunk / kq),
                                                 (optin - fixed) / (kq * bbytes));
        if (stages >= need) {
          p.nbuf = nbuf;
          p.wstages = stages;
          p.kq = kq;
          break;
        }
      }
    }
    if (!p.kq) return p;
  }
  p.smem = smem_for(p.nbuf, p.wstages, p.kq);
  return p;
}

template <int KZ>
int xf_launch(cmi_unet *u, const Slice &in, const bf16 *wpack, const float *bias,
              const Slice &out, int act, int batch, const int dims[3], int optin,
              const Slice *gate, const XfPlan &p) {
  using T = XTile<KZ>;
  CUtensorMap map;
  UN_TRY(make_map_box(&map, in, batch, dims, 16, T::kUX, T::kHY, T::kHZ));
  ConvArgs a{};
  a.wpack = wpack;
  a.bias = bias;
  a.out = out.base;
  a.out_ctot = out.ctot;
  a.out_c0 = out.c0;
  a.npad = out.c;
  a.nchunk = in.c / 16;
  for (int k = 0; k < 3; ++k) a.dims[k] = dims[k];
  a.batch = batch;
  a.act = act;
  a.slope = u->slope;
  if (gate) {
    a.gate = gate->base;
    a.gate_ctot = gate->ctot;
    a.gate_c0 = gate->c0;
  }
  a.err = u->d_err;
  a.nbuf = p.nbuf;
  a.wstages = p.wstages;
  a.kq = p.kq;
  // resident weights or a stage per tap row: the MMA sequence unrolled for the
  // common chunk counts
  auto kern = k_conv3_xf<KZ, 0>;
  if (p.kq == a.nchunk) {
    if (a.nchunk == 1) kern = k_conv3_xf<KZ, 1>;
    if (a.nchunk == 2) kern = k_conv3_xf<KZ, 2>;
    if (a.nchunk == 3) kern = k_conv3_xf<KZ, 3>;
    if (a.nchunk == 5) kern = k_conv3_xf<KZ, 5>;
  }
  // the kernel's limit is the device's whole opt-in size, the same for every
  // launch: a launch captured in a graph must stay valid whatever limit a
  // later launch of the same kernel would otherwise have set
  UN_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
  int per_sm = 0;
  UN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kXfThreads, p.smem));
  const int nrow = 3 * a.npad;
  const int acols = nrow <= 64 ? 64 : nrow <= 128 ? 128 : 256;
  per_sm = std::max(1, std::min(per_sm, 512 / (2 * KZ * acols)));
  int sms = 0, dev = 0;
  UN_CUDA(cudaGetDevice(&dev));
  UN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int tiles = T::num_tiles(batch, dims);
  const int grid = std::max(1, std::min(tiles, per_sm * sms));
  kern<<<grid, kXfThreads, p.smem, u->stream>>>(map, a);
  UN_CUDA(cudaGetLastError());
  return CMI_OK;
}

// x-folded convolution (weights packed with conv_xf): the deepest tile whose
// accumulators fit the tensor memory, whose weights stay resident beside two
// input buffers and that still gives every SM a tile; else one z slice
int conv_xf_tc(cmi_unet *u, const Slice &in, const bf16 *wpack, const float *bias,
               const Slice &out, int act, int batch, const int dims[3], const Slice *gate,
               int sms) {
  int optin = 0;
  UN_TRY(smem_optin(u, k_conv3_xf<1, 0>, &optin));
  const int nchunk = in.c / 16, npad = out.c;
  const int acols = 3 * npad <= 64 ? 64 : 3 * npad <= 128 ? 128 : 256;
  auto deep = [&](int kz, const XfPlan &p, int tiles) {
    return dims[2] % kz == 0 && 2 * kz * acols <= 512 && p.kq == nchunk && p.wstages == 9 &&
           p.nbuf >= 2 && tiles >= sms;
  };
  const XfPlan p4 = xf_plan<4>(nchunk, npad, optin);
  if (deep(4, p4, XTile<4>::num_tiles(batch, dims)))
    return xf_launch<4>(u, in, wpack, bias, out, act, batch, dims, optin, gate, p4);
  const XfPlan p2 = xf_plan<2>(nchunk, npad, optin);
  if (deep(2, p2, XTile<2>::num_tiles(batch, dims)))
    return xf_launch<2>(u, in, wpack, bias, out, act, batch, dims, optin, gate, p2);
  const XfPlan p1 = xf_plan<1>(nchunk, npad, optin);
  if (!p1.kq)
    return fail(CMI_ERR_NOT_SUPPORTED,
                "convolution: %d input channels do not fit the shared memory", in.c);
  return xf_launch<1>(u, in, wpack, bias, out, act, batch, dims, optin, gate, p1);
}

// y = act(conv(x) + b) into out slice; wpack rows = out.c; with a gate (an
// activation output of out's shape), y *= leaky'(gate)
int conv_tc(cmi_unet *u, const Slice &in, const bf16 *wpack, const float *bias, const Slice &out,
            int act, int batch, const int dims[3], const Slice *gate = nullptr) {
  const int ty = tile_y(dims);
  if (!ty)
    return fail(CMI_ERR_INVALID_ARGUMENT,
                "grid %dx%dx%d: X and Y must be multiples of 8, and Y of 16 or Z of 2",
                dims[0], dims[1], dims[2]);
  if (in.c % 16 || out.c % 16 || out.c > 256 || out.c < 16)
    return fail(CMI_ERR_INVALID_ARGUMENT, "channel counts must be multiples of 16 (<= 256)");
  int optin = 0, sms = 0, dev = 0;
  // the kernels' static shared memory is the same for every instance
  UN_TRY(smem_optin(u, k_conv3_tc<16, 1>, &optin));
  UN_CUDA(cudaGetDevice(&dev));
  UN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  if (gate && (gate->c != out.c || gate->c0 % 16 || gate->ctot % 16))
    return fail(CMI_ERR_INVALID_ARGUMENT, "gate slice does not match the output");
  if (conv_xf(out.c)) return conv_xf_tc(u, in, wpack, bias, out, act, batch, dims, gate, sms);
  if (ty == 8) return conv_launch<8, 1>(u, in, wpack, bias, out, act, batch, dims, optin, gate);
  if (conv_deep_ok<4>(in, out, batch, dims, optin, sms))
    return conv_launch<16, 4>(u, in, wpack, bias, out, act, batch, dims, optin, gate);
  if (conv_deep_ok<2>(in, out, batch, dims, optin, sms))
    return conv_launch<16, 2>(u, in, wpack, bias, out, act, batch, dims, optin, gate);
  return conv_launch<16, 1>(u, in, wpack, bias, out, act, batch, dims, optin, gate);
}

template <int TY>
int wgrad_t(cmi_unet *u, const Slice &x, const Slice &dy, float *dw, float *db,
            const int *ci_map, int cin_real, int cout_real, int batch, const int dims[3]) {
  using T = ConvTile<TY>;
  CUtensorMap xm, dym;
  UN_TRY(make_halo_map<TY>(&xm, x, batch, dims));
  using D = DyTile<TY>;
  UN_TRY(make_map_box(&dym, dy, batch, dims, 16, T::kTX, D::kRows, D::kTZ));
  WgradTcArgs a{};
  a.cout = dy.c;
  a.nchunk = x.c / 16;
  for (int k = 0; k < 3; ++k) a.dims[k] = dims[k];
  a.batch = batch;
  // units spread evenly over the fewest groups that fit the tensor memory
  const int units = 3 * (a.cout / 16) * a.nchunk;
  const int groups = (units + kWgradUnitsPerCta - 1) / kWgradUnitsPerCta;
  a.units_per_cta = (units + groups - 1) / groups;
  uint32_t cols = 32;
  while (cols < (uint32_t)(a.units_per_cta * kUnitCols)) cols <<= 1;
  a.tmem_cols = cols;
  a.dw = dw;
  a.db = db;
  a.ci_map = ci_map;
  a.cin_real = cin_real;
  a.cout_real = cout_real;
  a.err = u->d_err;
  int optin = 0;
  UN_TRY(smem_optin(u, k_conv3_wgrad_tc<TY>, &optin));
  // buffers [dy chunks][input halo]; the barriers sit past the buffers and past
  // the furthest byte the last dy chunk's A operands reach
  const size_t buf = (size_t)(a.cout / 16) * D::kChunkBytes + (size_t)a.nchunk * T::kChunkBytes;
  auto bars_at = [&](int nbuf) {
    const size_t reach_end =
        (size_t)(nbuf - 1) * buf + (size_t)(a.cout / 16 - 1) * D::kChunkBytes + D::kReach;
    return (std::max(nbuf * buf, reach_end) + 127) / 128 * 128;
  };
  auto smem_for = [&](int nbuf) { return 1024 + bars_at(nbuf) + 128; };
  // as many tile buffers (up to kWgMaxBufs) as leave room for the CTAs per SM
  // that the tensor memory allows
  const int tmem_ctas = std::max(1, (int)(512 / a.tmem_cols));
  const size_t cap = std::min<size_t>((size_t)optin, 233472 / tmem_ctas - 2048);
  a.nbuf = smem_for(2) <= (size_t)optin ? 2 : 1;  // fewer CTAs per SM before one buffer
  for (int nb = kWgMaxBufs; nb > 2; --nb)
    if (smem_for(nb) <= cap) {
      a.nbuf = nb;
      break;
    }
  a.bar_off = (int)bars_at(a.nbuf);
  const size_t smem = smem_for(a.nbuf);
  if (smem > (size_t)optin)
    return fail(CMI_ERR_NOT_SUPPORTED, "weight gradient needs %zu B of shared memory", smem);
  // the whole opt-in size, the same for every launch (see xf_launch)
  UN_CUDA(cudaFuncSetAttribute(k_conv3_wgrad_tc<TY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               optin));
  int per_sm = 0;
  UN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_conv3_wgrad_tc<TY>,
                                                        kWgradThreads, smem));
  // TMEM: at most 512 columns per SM
  per_sm = std::max(1, std::min(per_sm, (int)(512 / a.tmem_cols)));
  int sms = 0, dev = 0;
  UN_CUDA(cudaGetDevice(&dev));
  UN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int tiles = batch * (dims[0] / T::kTX) * (dims[1] / T::kTY) * (dims[2] / T::kTZ);
  const int ctas = std::max(1, std::min(tiles, per_sm * sms / groups));
  // the CTAs' sums go through the network's scratch and one reduction pass when
  // they fit (without it every CTA adds its sums to the same dw entries with
  // FP32 atomics, which costs more than the scratch round trip)
  const size_t part_floats = (size_t)groups * ctas * a.units_per_cta * 3 * 768;
  if (u->wg_part && part_floats <= u->wg_part_floats) a.part = u->wg_part;
  k_conv3_wgrad_tc<TY><<<dim3(ctas, groups), kWgradThreads, smem, u->stream>>>(xm, dym, a);
  UN_CUDA(cudaGetLastError());
  if (a.part) {
    const long long outs = (long long)units * 3 * 768;
    k_wgrad_reduce<<<(int)std::min<long long>((outs + 31) / 32, 8192), 32 * kReduceSlices, 0,
                     u->stream>>>(a.part, ctas, units, a);
    UN_CUDA(cudaGetLastError());
  }
  return CMI_OK;
}

// dW (and, with db, the bias gradient) of a convolution from its input x and
// output gradient dy, accumulated
int wgrad(cmi_unet *u, const Slice &x, const Slice &dy, float *dw, float *db, const int *ci_map,
          int cin_real, int cout_real, int batch, const int dims[3]) {
  const int ty = tile_y(dims);
  if (!ty)
    return fail(CMI_ERR_INVALID_ARGUMENT,
                "grid %dx%dx%d: X and Y must be multiples of 8, and Y of 16 or Z of 2",
                dims[0], dims[1], dims[2]);
  if (x.c % 16 || dy.c % 16 || x.c < 16 || x.c > 256 || dy.c < 16 || dy.c > 128)
    return fail(CMI_ERR_NOT_SUPPORTED,
                "weight gradient: input channels must be 16..256, output channels 16..128, "
                "multiples of 16");
  return ty == 16 ? wgrad_t<16>(u, x, dy, dw, db, ci_map, cin_real, cout_real, batch, dims)
                  : wgrad_t<8>(u, x, dy, dw, db, ci_map, cin_real, cout_real, batch, dims);
}

// the packing jobs of every layer: forward operand, input-gradient operand
// (flipped, transposed), bias padded to npad; uploaded once
int make_pack_jobs(cmi_unet *u) {
  std::vector<PackJob> jobs;
  long long at = 0;
  for (Layer &l : u->L) {
    PackJob j{};
    j.a.w = u->p + l.w_off;
    j.a.cout = l.cout;
    j.a.cin_real = l.cin_real;
    j.a.ci_of_storage = l.d_map;
    j.a.out = l.wf;
    j.a.rows = l.npad;
    j.a.kchan = l.kin;
    j.a.flip = 0;
    j.a.xf = conv_xf(j.a.rows);
    j.begin = at;
    j.count = 27LL * l.kin * l.npad;
    at += j.count;
    jobs.push_back(j);
    j.a.out = l.wd;
    j.a.rows = l.kin;
    j.a.kchan = l.npad;
    j.a.flip = 1;
    j.a.xf = conv_xf(j.a.rows);
    j.begin = at;
    at += j.count;
    jobs.push_back(j);
    PackJob b{};
    b.a.cout = l.cout;
    b.bias = u->p + l.b_off;
    b.bias_pad = l.bias_pad;
    b.begin = at;
    b.count = l.npad;
    at += b.count;
    jobs.push_back(b);
  }
  UN_CUDA(cudaMalloc(&u->d_jobs, sizeof(PackJob) * jobs.size()));
  UN_CUDA(cudaMemcpy(u->d_jobs, jobs.data(), sizeof(PackJob) * jobs.size(),
                     cudaMemcpyHostToDevice));
  u->njobs = (int)jobs.size();
  u->jobs_total = at;
  return CMI_OK;
}

// packs every layer's weights from the FP32 master parameters (one launch)
int pack_launches(cmi_unet *u) {
  k_pack_all<<<grid_for(u->jobs_total), 256, 0, u->stream>>>(
      static_cast<const PackJob *>(u->d_jobs), u->njobs, u->jobs_total);
  UN_CUDA(cudaGetLastError());
  return CMI_OK;
}
int pack_all(cmi_unet *u) {
  UN_TRY(graph_run(u, &u->gx_pack, [&] { return pack_launches(u); }));
  u->packed = true;
  return CMI_OK;
}

int check_dims(const int dims[3]) {
  for (int a = 0; a < 3; ++a)
    if (dims[a] <= 0 || dims[a] % 32)
      return fail(CMI_ERR_INVALID_ARGUMENT,
                  "grid sides must be positive multiples of 32 (three levels of 8x4x4 tiles)");
  return CMI_OK;
}

// the elementwise kernels index 16-byte groups with 32-bit arithmetic
int check_size(int batch, const int dims[3]) {
  if ((long long)batch * dims[0] * dims[1] * dims[2] * 16 > (1LL << 31))
    return fail(CMI_ERR_NOT_SUPPORTED, "batch x cells must be at most 2^27 (134217728)");
  return CMI_OK;
}

// forward pass from u->X0; writes u->pred
int forward_layers(cmi_unet *u, int batch, const int d1[3]) {
  const Chans c = chans(u);
  const int d2[3] = {d1[0] / 2, d1[1] / 2, d1[2] / 2};
  const int d3[3] = {d1[0] / 4, d1[1] / 4, d1[2] / 4};
  const long long v1 = (long long)batch * d1[0] * d1[1] * d1[2];
  auto S = [](bf16 *b, int ctot, int c0, int cc) { return Slice{b, ctot, c0, cc}; };
  std::vector<Layer> &L = u->L;
  // level 1
  UN_TRY(conv_tc(u, S(u->X0, 16, 0, 16), L[0].wf, L[0].bias_pad, S(u->E1A, c.s1, 0, c.s1), 1,
                 batch, d1));
  UN_TRY(conv_tc(u, S(u->E1A, c.s1, 0, c.s1), L[1].wf, L[1].bias_pad,
                 S(u->CAT1, c.cat1, c.s2, c.s1), 1, batch, d1));
  k_pool2<<<grid_for(v1 / 8 * c.s1 / 8), 256, 0, u->stream>>>(u->CAT1, c.cat1, c.s2, u->P1, c.s1, 0,
                                                           c.s1, batch, d1[0], d1[1], d1[2]);
  // level 2
  UN_TRY(conv_tc(u, S(u->P1, c.s1, 0, c.s1), L[2].wf, L[2].bias_pad, S(u->E2A, c.s2, 0, c.s2), 1,
                 batch, d2));
  UN_TRY(conv_tc(u, S(u->E2A, c.s2, 0, c.s2), L[3].wf, L[3].bias_pad,
                 S(u->CAT2, c.cat2, c.s3, c.s2), 1, batch, d2));
  k_pool2<<<grid_for(v1 / 64 * c.s2 / 8), 256, 0, u->stream>>>(u->CAT2, c.cat2, c.s3, u->P2, c.s2, 0,
                                                            c.s2, batch, d2[0], d2[1], d2[2]);
  // level 3
  UN_TRY(conv_tc(u, S(u->P2, c.s2, 0, c.s2), L[4].wf, L[4].bias_pad, S(u->BA, c.s3, 0, c.s3), 1,
                 batch, d3));
  UN_TRY(conv_tc(u, S(u->BA, c.s3, 0, c.s3), L[5].wf, L[5].bias_pad, S(u->BB, c.s3, 0, c.s3), 1,
                 batch, d3));
  // up to level 2
  k_up2<<<grid_for(v1 / 8 * c.s3 / 8), 256, 0, u->stream>>>(u->BB, c.s3, 0, u->CAT2, c.cat2, 0, c.s3,
                                                         batch, d3[0], d3[1], d3[2]);
  UN_TRY(conv_tc(u, S(u->CAT2, c.cat2, 0, c.cat2), L[6].wf, L[6].bias_pad,
                 S(u->D2A, c.s2, 0, c.s2), 1, batch, d2));
  UN_TRY(conv_tc(u, S(u->D2A, c.s2, 0, c.s2), L[7].wf, L[7].bias_pad, S(u->D2B, c.s2, 0, c.s2), 1,
                 batch, d2));
  // up to level 1
  k_up2<<<grid_for(v1 * c.s2 / 8), 256, 0, u->stream>>>(u->D2B, c.s2, 0, u->CAT1, c.cat1, 0, c.s2,
                                                     batch, d2[0], d2[1], d2[2]);
  UN_TRY(conv_tc(u, S(u->CAT1, c.cat1, 0, c.cat1), L[8].wf, L[8].bias_pad,
                 S(u->D1A, c.s1, 0, c.s1), 1, batch, d1));
  UN_TRY(conv_tc(u, S(u->D1A, c.s1, 0, c.s1), L[9].wf, L[9].bias_pad, S(u->D1B, c.s1, 0, c.s1), 1,
                 batch, d1));
  UN_CUDA(cudaGetLastError());
  return CMI_OK;
}

// loss + backward from u->D1B etc. (forward must have run); gradients into u->g
// the loss and the head's gradients from the target; dy of the last convolution
int backward_head(cmi_unet *u, const float *target, int batch, const int d1[3]) {
  const Chans c = chans(u);
  const long long v1 = (long long)batch * d1[0] * d1[1] * d1[2];
  UN_CUDA(cudaMemsetAsync(u->g, 0, sizeof(float) * u->nparams, u->stream));
  UN_CUDA(cudaMemsetAsync(u->d_loss, 0, sizeof(float), u->stream));
  // the head writes dy of the last convolution, times its activation derivative
  k_head<<<grid_for(v1), 256, 0, u->stream>>>(u->D1B, c.s1, c.c1, u->p + u->head_w,
                                               u->p + u->head_b, v1, u->pred, target, u->gD1B,
                                               u->g + u->head_w, u->g + u->head_b, u->d_loss,
                                               u->over_weight, u->slope);
  UN_CUDA(cudaGetLastError());
  return CMI_OK;
}

// the convolution layers backwards from dy of the last one: gradients into u->g
int backward_layers(cmi_unet *u, int batch, const int d1[3]) {
  const Chans c = chans(u);
  const int d2[3] = {d1[0] / 2, d1[1] / 2, d1[2] / 2};
  const int d3[3] = {d1[0] / 4, d1[1] / 4, d1[2] / 4};
  const long long v1 = (long long)batch * d1[0] * d1[1] * d1[2];
  const long long v2 = v1 / 8, v3 = v1 / 64;
  auto S = [](bf16 *b, int ctot, int c0, int cc) { return Slice{b, ctot, c0, cc}; };
  std::vector<Layer> &L = u->L;
  const float sl = u->slope;
  // one convolution layer backwards from dy (already times the derivative of
  // its activation): weight and bias gradients, then the input gradient dx,
  // with a gate the activation output that dx is the gradient of
  auto layer_bwd = [&](int li, const Slice &x, const Slice &dy, const Slice *dx,
                       const Slice *gate, int b, const int *dims) -> int {
    UN_TRY(wgrad(u, x, dy, u->g + L[li].w_off, u->g + L[li].b_off, L[li].d_map,
                 L[li].cin_real, L[li].cout, b, dims));
    if (dx) UN_TRY(conv_tc(u, dy, L[li].wd, nullptr, *dx, 0, b, dims, gate));
    return CMI_OK;
  };
  // level 1 decoder
  {
    const Slice dx = S(u->gD1A, c.s1, 0, c.s1), gate = S(u->D1A, c.s1, 0, c.s1);
    UN_TRY(layer_bwd(9, S(u->D1A, c.s1, 0, c.s1), S(u->gD1B, c.s1, 0, c.s1), &dx, &gate, batch,
                     d1));
  }
  {
    const Slice dx = S(u->gCAT1, c.cat1, 0, c.cat1);
    UN_TRY(layer_bwd(8, S(u->CAT1, c.cat1, 0, c.cat1), S(u->gD1A, c.s1, 0, c.s1), &dx, nullptr,
                     batch, d1));
  }
  // up1 backward: gD2B = sum of children of gCAT1[0:s2], times leaky'(D2B)
  k_up2_bwd<<<grid_for(v2 * c.s2 / 8), 256, 0, u->stream>>>(
      u->gCAT1, c.cat1, 0, u->gD2B, c.s2, 0, c.s2, batch, d2[0], d2[1], d2[2], u->D2B, c.s2, 0,
      sl);
  {
    const Slice dx = S(u->gD2A, c.s2, 0, c.s2), gate = S(u->D2A, c.s2, 0, c.s2);
    UN_TRY(layer_bwd(7, S(u->D2A, c.s2, 0, c.s2), S(u->gD2B, c.s2, 0, c.s2), &dx, &gate, batch,
                     d2));
  }
  {
    const Slice dx = S(u->gCAT2, c.cat2, 0, c.cat2);
    UN_TRY(layer_bwd(6, S(u->CAT2, c.cat2, 0, c.cat2), S(u->gD2A, c.s2, 0, c.s2), &dx, nullptr,
                     batch, d2));
  }
  // up2 backward: gBB = sum of children of gCAT2[0:s3], times leaky'(BB)
  k_up2_bwd<<<grid_for(v3 * c.s3 / 8), 256, 0, u->stream>>>(
      u->gCAT2, c.cat2, 0, u->gBB, c.s3, 0, c.s3, batch, d3[0], d3[1], d3[2], u->BB, c.s3, 0, sl);
  {
    const Slice dx = S(u->gBA, c.s3, 0, c.s3), gate = S(u->BA, c.s3, 0, c.s3);
    UN_TRY(layer_bwd(5, S(u->BA, c.s3, 0, c.s3), S(u->gBB, c.s3, 0, c.s3), &dx, &gate, batch,
                     d3));
  }
  {
    const Slice dx = S(u->gP2, c.s2, 0, c.s2);
    UN_TRY(layer_bwd(4, S(u->P2, c.s2, 0, c.s2), S(u->gBA, c.s3, 0, c.s3), &dx, nullptr, batch,
                     d3));
  }
  // pool2 backward, added to the skip gradient gCAT2[s3 : s3 + s2], times the
  // derivative of that activation (CAT2[s3:])
  k_pool2_bwd_add<<<grid_for(v2 * c.s2 / 8), 256, 0, u->stream>>>(
      u->gP2, c.s2, 0, u->gCAT2, c.cat2, c.s3, c.s2, batch, d2[0], d2[1], d2[2], u->CAT2, c.cat2,
      c.s3, sl);
  {
    const Slice dx = S(u->gE2A, c.s2, 0, c.s2), gate = S(u->E2A, c.s2, 0, c.s2);
    UN_TRY(layer_bwd(3, S(u->E2A, c.s2, 0, c.s2), S(u->gCAT2, c.cat2, c.s3, c.s2), &dx, &gate,
                     batch, d2));
  }
  {
    const Slice dx = S(u->gP1, c.s1, 0, c.s1);
    UN_TRY(layer_bwd(2, S(u->P1, c.s1, 0, c.s1), S(u->gE2A, c.s2, 0, c.s2), &dx, nullptr, batch,
                     d2));
  }
  k_pool2_bwd_add<<<grid_for(v1 * c.s1 / 8), 256, 0, u->stream>>>(
      u->gP1, c.s1, 0, u->gCAT1, c.cat1, c.s2, c.s1, batch, d1[0], d1[1], d1[2], u->CAT1, c.cat1,
      c.s2, sl);
  {
    const Slice dx = S(u->gE1A, c.s1, 0, c.s1), gate = S(u->E1A, c.s1, 0, c.s1);
    UN_TRY(layer_bwd(1, S(u->E1A, c.s1, 0, c.s1), S(u->gCAT1, c.cat1, c.s2, c.s1), &dx, &gate,
                     batch, d1));
  }
  UN_TRY(layer_bwd(0, S(u->X0, 16, 0, 16), S(u->gE1A, c.s1, 0, c.s1), nullptr, nullptr, batch,
                   d1));
  UN_CUDA(cudaGetLastError());
  return CMI_OK;
}

int check_err(cmi_unet *u) {
  uint32_t e = 0;
  UN_CUDA(cudaMemcpyAsync(&e, u->d_err, sizeof(e), cudaMemcpyDeviceToHost, u->stream));
  UN_CUDA(cudaStreamSynchronize(u->stream));
  if (e) {
    UN_CUDA(cudaMemsetAsync(u->d_err, 0, sizeof(uint32_t), u->stream));
    return fail(CMI_ERR_DEVICE_TIMEOUT, "tensor-core convolution wait timed out (flags 0x%x)", e);
  }
  return CMI_OK;
}

int load_input(cmi_unet *u, const float *in, int batch, const int dims[3]) {
  UN_TRY(check_dims(dims));
  if (batch <= 0) return fail(CMI_ERR_INVALID_ARGUMENT, "batch must be > 0");
  UN_TRY(check_size(batch, dims));
  UN_CUDA(cudaSetDevice(u->device));
  UN_TRY(ensure_buffers(u, batch, dims));
  if (!u->packed) UN_TRY(pack_all(u));
  const long long v1 = (long long)batch * dims[0] * dims[1] * dims[2];
  k_input<<<grid_for(v1), 256, 0, u->stream>>>(in, u->X0, (unsigned)v1);
  UN_CUDA(cudaGetLastError());
  return CMI_OK;
}

// the layers of a pass, replayed from their graphs (the buffers are those of
// (batch, dims), which load_input has made current)
int forward(cmi_unet *u, int batch, const int d[3]) {
  return graph_run(u, &u->gx_fwd, [&] { return forward_layers(u, batch, d); });
}
int backward(cmi_unet *u, const float *target, int batch, const int d[3]) {
  UN_TRY(backward_head(u, target, batch, d));
  return graph_run(u, &u->gx_bwd, [&] { return backward_layers(u, batch, d); });
}

}  // namespace cmiu

// ===========================================================================
// extern "C"
// ===========================================================================
extern "C" {

void cmi_unet_default_config(cmi_unet_config *c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->channels[0] = 12;
  c->channels[1] = 24;
  c->channels[2] = 48;
  c->leaky_slope = 0.1f;
  c->device = 0;
}

const char *cmi_unet_last_error_string(void) { return g_err; }

int cmi_unet_create(const cmi_unet_config *cfg, cmi_unet **out) {
  if (!cfg || !out) return fail(CMI_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  for (int k = 0; k < 3; ++k)
    if (cfg->channels[k] < 1 || cfg->channels[k] > 64)
      return fail(CMI_ERR_INVALID_ARGUMENT, "channels must be in [1, 64]");
  if (cfg->channels[0] > 16)
    return fail(CMI_ERR_INVALID_ARGUMENT, "level-1 channels must be <= 16 (the output head)");
  if (!(cfg->leaky_slope >= 0.f && cfg->leaky_slope < 1.f))
    return fail(CMI_ERR_INVALID_ARGUMENT, "leaky_slope must be in [0, 1)");
  int ndev = 0;
  UN_CUDA(cudaGetDeviceCount(&ndev));
  if (cfg->device < 0 || cfg->device >= ndev)
    return fail(CMI_ERR_INVALID_ARGUMENT, "device %d out of range", cfg->device);
  UN_CUDA(cudaSetDevice(cfg->device));
  cudaDeviceProp prop{};
  UN_CUDA(cudaGetDeviceProperties(&prop, cfg->device));
  if (prop.major != 10)
    return fail(CMI_ERR_NOT_SUPPORTED, "tcgen05 kernels need compute capability 10.x (got %d.%d)",
                prop.major, prop.minor);
  cmi_unet *u = new (std::nothrow) cmi_unet();
  if (!u) return fail(CMI_ERR_OUT_OF_MEMORY, "host allocation");
  u->device = cfg->device;
  for (int k = 0; k < 3; ++k) u->ch[k] = cfg->channels[k];
  u->slope = cfg->leaky_slope;
  auto bail = [&](int rc) {
    cmi_unet_destroy(u);
    return rc;
  };
  if (cudaStreamCreateWithFlags(&u->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(CMI_ERR_CUDA, "stream creation failed"));
  const Chans c = chans(u);
  // layer table: (cout, input segments (real, storage width))
  struct Spec {
    int cout;
    int seg_real[2], seg_store[2];
  };
  const Spec specs[10] = {
      {c.c1, {kFeatures, 0}, {16, 0}},  {c.c1, {c.c1, 0}, {c.s1, 0}},
      {c.c2, {c.c1, 0}, {c.s1, 0}},     {c.c2, {c.c2, 0}, {c.s2, 0}},
      {c.c3, {c.c2, 0}, {c.s2, 0}},     {c.c3, {c.c3, 0}, {c.s3, 0}},
      {c.c2, {c.c3, c.c2}, {c.s3, c.s2}}, {c.c2, {c.c2, 0}, {c.s2, 0}},
      {c.c1, {c.c2, c.c1}, {c.s2, c.s1}}, {c.c1, {c.c1, 0}, {c.s1, 0}},
  };
  size_t off = 0;
  u->L.resize(10);
  for (int i = 0; i < 10; ++i) {
    Layer &l = u->L[i];
    l.cout = specs[i].cout;
    l.npad = pad16(l.cout);
    l.cin_real = specs[i].seg_real[0] + specs[i].seg_real[1];
    l.kin = specs[i].seg_store[0] + specs[i].seg_store[1];
    l.ci_of_storage.assign(l.kin, -1);
    int real = 0, store = 0;
    for (int sgm = 0; sgm < 2; ++sgm) {
      for (int k = 0; k < specs[i].seg_real[sgm]; ++k) l.ci_of_storage[store + k] = real + k;
      real += specs[i].seg_real[sgm];
      store += specs[i].seg_store[sgm];
    }
    l.w_off = off;
    off += (size_t)l.cout * 27 * l.cin_real;
    l.b_off = off;
    off += l.cout;
  }
  u->head_w = off;
  off += c.c1;
  u->head_b = off;
  off += 1;
  u->nparams = off;
  int rc = CMI_OK;
  void *p = nullptr;
  if ((rc = dev_zero_alloc(&p, sizeof(float) * off))) return bail(rc);
  u->p = static_cast<float *>(p);
  if ((rc = dev_zero_alloc(&p, sizeof(float) * off))) return bail(rc);
  u->g = static_cast<float *>(p);
  if ((rc = dev_zero_alloc(&p, sizeof(float) * off))) return bail(rc);
  u->m = static_cast<float *>(p);
  if ((rc = dev_zero_alloc(&p, sizeof(float) * off))) return bail(rc);
  u->v = static_cast<float *>(p);
  if ((rc = dev_zero_alloc(&p, sizeof(uint32_t)))) return bail(rc);
  u->d_err = static_cast<uint32_t *>(p);
  if ((rc = dev_zero_alloc(&p, sizeof(float)))) return bail(rc);
  u->d_loss = static_cast<float *>(p);
  for (Layer &l : u->L) {
    const size_t nw = (size_t)27 * l.kin * l.npad;
    if ((rc = dev_zero_alloc(&p, sizeof(bf16) * nw))) return bail(rc);
    l.wf = static_cast<bf16 *>(p);
    if ((rc = dev_zero_alloc(&p, sizeof(bf16) * nw))) return bail(rc);
    l.wd = static_cast<bf16 *>(p);
    if ((rc = dev_zero_alloc(&p, sizeof(int) * l.kin))) return bail(rc);
    l.d_map = static_cast<int *>(p);
    if (cudaMemcpy(l.d_map, l.ci_of_storage.data(), sizeof(int) * l.kin,
                   cudaMemcpyHostToDevice) != cudaSuccess)
      return bail(fail(CMI_ERR_CUDA, "upload channel map"));
    if ((rc = dev_zero_alloc(&p, sizeof(float) * l.npad))) return bail(rc);
    l.bias_pad = static_cast<float *>(p);
  }
  if ((rc = make_pack_jobs(u))) return bail(rc);
  *out = u;
  return CMI_OK;
}

int cmi_unet_destroy(cmi_unet *u) {
  if (!u) return CMI_OK;
  cudaSetDevice(u->device);
  if (u->stream) cudaStreamSynchronize(u->stream);
  free_bufs(u);
  drop_graph(&u->gx_pack);
  cudaFree(u->d_jobs);
  for (Layer &l : u->L) {
    cudaFree(l.wf);
    cudaFree(l.wd);
    cudaFree(l.d_map);
    cudaFree(l.bias_pad);
  }
  cudaFree(u->p);
  cudaFree(u->g);
  cudaFree(u->m);
  cudaFree(u->v);
  cudaFree(u->d_err);
  cudaFree(u->d_loss);
  cudaFree(u->wg_part);
  cudaFree(u->d_src);
  cudaFree(u->d_nrel);
  cudaFree(u->d_ncoarse);
  cudaFree(u->d_ratio);
  if (u->stream) cudaStreamDestroy(u->stream);
  delete u;
  return CMI_OK;
}

int cmi_unet_num_params(cmi_unet *u, int64_t *n) {
  if (!u || !n) return fail(CMI_ERR_INVALID_ARGUMENT, "null argument");
  *n = (int64_t)u->nparams;
  return CMI_OK;
}

int cmi_unet_get_params(cmi_unet *u, float *host) {
  if (!u || !host) return fail(CMI_ERR_INVALID_ARGUMENT, "null argument");
  UN_CUDA(cudaSetDevice(u->device));
  UN_CUDA(cudaMemcpyAsync(host, u->p, sizeof(float) * u->nparams, cudaMemcpyDeviceToHost,
                          u->stream));
  UN_CUDA(cudaStreamSynchronize(u->stream));
  return CMI_OK;
}

int cmi_unet_set_params(cmi_unet *u, const float *host) {
  if (!u || !host) return fail(CMI_ERR_INVALID_ARGUMENT, "null argument");
  UN_CUDA(cudaSetDevice(u->device));
  UN_CUDA(cudaMemcpyAsync(u->p, host, sizeof(float) * u->nparams, cudaMemcpyHostToDevice,
                          u->stream));
  UN_CUDA(cudaMemsetAsync(u->m, 0, sizeof(float) * u->nparams, u->stream));
  UN_CUDA(cudaMemsetAsync(u->v, 0, sizeof(float) * u->nparams, u->stream));
  u->adam_t = 0;
  UN_TRY(pack_all(u));
  UN_CUDA(cudaStreamSynchronize(u->stream));
  return CMI_OK;
}

int cmi_unet_forward(cmi_unet *u, const float *features, float *pred, int32_t batch,
                     const int32_t dims[3]) {
  if (!u || !features || !pred || !dims) return fail(CMI_ERR_INVALID_ARGUMENT, "null argument");
  const int d[3] = {dims[0], dims[1], dims[2]};
  UN_TRY(load_input(u, features, batch, d));
  UN_TRY(forward(u, batch, d));
  const long long v1 = (long long)batch * d[0] * d[1] * d[2];
  const Chans c = chans(u);
  k_head<<<grid_for(v1), 256, 0, u->stream>>>(u->D1B, c.s1, c.c1, u->p + u->head_w,
                                               u->p + u->head_b, v1, pred, nullptr, nullptr,
                                               nullptr, nullptr, nullptr, 1.f, u->slope);
  UN_CUDA(cudaGetLastError());
  return check_err(u);
}

int cmi_unet_gradients(cmi_unet *u, const float *features, const float *target, int32_t batch,
                       const int32_t dims[3], float *loss, float *grads_host) {
  if (!u || !features || !target || !dims) return fail(CMI_ERR_INVALID_ARGUMENT, "null argument");
  const int d[3] = {dims[0], dims[1], dims[2]};
  UN_TRY(load_input(u, features, batch, d));
  UN_TRY(forward(u, batch, d));
  UN_TRY(backward(u, target, batch, d));
  UN_TRY(check_err(u));
  const long long v1 = (long long)batch * d[0] * d[1] * d[2];
  if (loss) {
    float s = 0.f;
    UN_CUDA(cudaMemcpy(&s, u->d_loss, sizeof(float), cudaMemcpyDeviceToHost));
    *loss = s / (float)v1;
  }
  if (grads_host)
    UN_CUDA(cudaMemcpy(grads_host, u->g, sizeof(float) * u->nparams, cudaMemcpyDeviceToHost));
  return CMI_OK;
}

int cmi_unet_train_step(cmi_unet *u, const float *features, const float *target, int32_t batch,
                        const int32_t dims[3], float lr, float *loss) {
  if (!u || !features || !target || !dims) return fail(CMI_ERR_INVALID_ARGUMENT, "null argument");
  if (!(lr > 0.f) || !std::isfinite(lr)) return fail(CMI_ERR_INVALID_ARGUMENT, "lr must be > 0");
  const int d[3] = {dims[0], dims[1], dims[2]};
  UN_TRY(load_input(u, features, batch, d));
  UN_TRY(forward(u, batch, d));
  UN_TRY(backward(u, target, batch, d));
  u->adam_t += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, (float)u->adam_t), c2 = 1.f - std::pow(b2, (float)u->adam_t);
  k_adam<<<grid_for((long long)u->nparams), 256, 0, u->stream>>>(
      u->p, u->g, u->m, u->v, (long long)u->nparams, lr, b1, b2, 1e-8f, c1, c2);
  UN_TRY(pack_all(u));
  UN_TRY(check_err(u));
  if (loss) {
    float s = 0.f;
    UN_CUDA(cudaMemcpy(&s, u->d_loss, sizeof(float), cudaMemcpyDeviceToHost));
    *loss = s / (float)((long long)batch * d[0] * d[1] * d[2]);
  }
  return CMI_OK;
}

}  // extern "C"

namespace cmiu {

// grow-only device scratch
template <class T>
int ensure(T **p, size_t *cap, size_t n) {
  if (n <= *cap) return CMI_OK;
  cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  UN_CUDA(cudaMalloc(p, sizeof(T) * n));
  *cap = n;
  return CMI_OK;
}

// geometry of a (dims, box) grid in the kernel's axis conventions
void grid_args(FeatureArgs &a, const int32_t dims[3], const double box[6]) {
  a.dims[0] = dims[2];  // X = iz (fastest)
  a.dims[1] = dims[1];
  a.dims[2] = dims[0];  // Z = ix
  for (int k = 0; k < 3; ++k) {
    a.n3[k] = dims[k];
    a.origin[k] = box[k];
    a.cell[k] = box[3 + k] / dims[k];
  }
}

int features_impl(cmi_unet *u, const double *nH_cube, const int32_t dims[3], const double box[6],
                  const double *sources, int32_t num_sources, double recombination_rate,
                  const float norm[6], int32_t ratio_factor, float *features) {
  if (!u || !nH_cube || !dims || !box || !norm || !features || (num_sources > 0 && !sources))
    return fail(CMI_ERR_INVALID_ARGUMENT, "null argument");
  if (num_sources < 0 || num_sources > 4096)
    return fail(CMI_ERR_INVALID_ARGUMENT, "0..4096 sources");
  if (!(recombination_rate > 0.) || !std::isfinite(recombination_rate))
    return fail(CMI_ERR_INVALID_ARGUMENT, "recombination rate must be > 0");
  if (ratio_factor < 1 || ratio_factor > 64)
    return fail(CMI_ERR_INVALID_ARGUMENT, "ratio factor must be in 1..64");
  for (int k = 0; k < 3; ++k) {
    if (dims[k] <= 0 || !(box[3 + k] > 0.))
      return fail(CMI_ERR_INVALID_ARGUMENT, "grid sides and box sizes must be > 0");
    if (dims[k] % ratio_factor)
      return fail(CMI_ERR_INVALID_ARGUMENT, "grid sides must be multiples of the ratio factor");
  }
  UN_CUDA(cudaSetDevice(u->device));
  FeatureArgs a{};
  a.nH = nH_cube;
  a.alpha = recombination_rate;
  a.nref = 1e8;  // n_H unit of the ray sums (FP32 range)
  UN_TRY(ensure(&u->d_src, &u->src_cap, (size_t)4 * std::max(num_sources, 1)));
  if (num_sources > 0)
    UN_CUDA(cudaMemcpyAsync(u->d_src, sources, sizeof(double) * 4 * num_sources,
                            cudaMemcpyHostToDevice, u->stream));
  a.src = u->d_src;
  a.nsrc = num_sources;
  for (int k = 0; k < 2 * kFeatures; ++k) a.norm[k] = norm[k];
  const long long nv = (long long)dims[0] * dims[1] * dims[2];
  if (ratio_factor == 1) {
    UN_TRY(ensure(&u->d_nrel, &u->nrel_cap, (size_t)nv));
    grid_args(a, dims, box);
    a.nrel = u->d_nrel;
    a.out = features;
    k_nrel<<<grid_for(nv), 256, 0, u->stream>>>(nH_cube, u->d_nrel, nv, 1. / a.nref);
    k_features<<<grid_for(nv), 256, 0, u->stream>>>(a);
  } else {
    // channel 2 on the grid coarser by ratio_factor (block-mean n_H), then
    // interpolated: the march costs ratio_factor^4 times less
    const int f = ratio_factor;
    const int32_t cd[3] = {dims[0] / f, dims[1] / f, dims[2] / f};
    const long long nc = (long long)cd[0] * cd[1] * cd[2];
    UN_TRY(ensure(&u->d_ncoarse, &u->ncoarse_cap, (size_t)nc));
    UN_TRY(ensure(&u->d_nrel, &u->nrel_cap, (size_t)nc));
    UN_TRY(ensure(&u->d_ratio, &u->ratio_cap, (size_t)nc));
    k_block_mean<<<grid_for(nc), 256, 0, u->stream>>>(nH_cube, u->d_ncoarse, dims[0], dims[1],
                                                      dims[2], f);
    k_nrel<<<grid_for(nc), 256, 0, u->stream>>>(u->d_ncoarse, u->d_nrel, nc, 1. / a.nref);
    FeatureArgs c = a;
    grid_args(c, cd, box);
    c.nH = u->d_ncoarse;
    c.nrel = u->d_nrel;
    c.out = u->d_ratio;
    c.mode = 1;
    k_features<<<grid_for(nc), 256, 0, u->stream>>>(c);
    grid_args(a, dims, box);
    a.out = features;
    a.mode = 2;
    a.ratio = u->d_ratio;
    a.rf = f;
    for (int k = 0; k < 3; ++k) a.rm[k] = cd[k];
    k_features<<<grid_for(nv), 256, 0, u->stream>>>(a);
  }
  UN_CUDA(cudaGetLastError());
  UN_CUDA(cudaStreamSynchronize(u->stream));
  return CMI_OK;
}

}  // namespace cmiu

extern "C" {

int cmi_unet_features(cmi_unet *u, const double *nH_cube, const int32_t dims[3],
                      const double box[6], const double *sources, int32_t num_sources,
                      double recombination_rate, const float norm[6], float *features) {
  return cmiu::features_impl(u, nH_cube, dims, box, sources, num_sources, recombination_rate,
                             norm, 1, features);
}

int cmi_unet_features_coarse_ratio(cmi_unet *u, const double *nH_cube, const int32_t dims[3],
                                   const double box[6], const double *sources,
                                   int32_t num_sources, double recombination_rate,
                                   const float norm[6], int32_t ratio_factor, float *features) {
  return cmiu::features_impl(u, nH_cube, dims, box, sources, num_sources, recombination_rate,
                             norm, ratio_factor, features);
}

int cmi_unet_set_loss_weight(cmi_unet *u, float over_weight) {
  if (!u) return fail(CMI_ERR_INVALID_ARGUMENT, "null network");
  if (!(over_weight > 0.f) || !std::isfinite(over_weight))
    return fail(CMI_ERR_INVALID_ARGUMENT, "loss weight must be finite and > 0");
  u->over_weight = over_weight;
  return CMI_OK;
}

int cmi_unet_to_neutral_fraction(cmi_unet *u, const float *pred, double *xH, int64_t n,
                                 float log10_min) {
  if (!u || !pred || !xH || n < 0) return fail(CMI_ERR_INVALID_ARGUMENT, "bad argument");
  UN_CUDA(cudaSetDevice(u->device));
  k_to_xH<<<grid_for(n), 256, 0, u->stream>>>(pred, xH, n, log10_min);
  UN_CUDA(cudaStreamSynchronize(u->stream));
  return CMI_OK;
}

int cmi_unet_block_mean(cmi_unet *u, const double *src, const int32_t dims[3], int32_t factor,
                        double *dst) {
  if (!u || !src || !dst || !dims || factor < 1)
    return fail(CMI_ERR_INVALID_ARGUMENT, "bad argument");
  for (int a = 0; a < 3; ++a)
    if (dims[a] <= 0 || dims[a] % factor)
      return fail(CMI_ERR_INVALID_ARGUMENT, "grid sides must be positive multiples of factor");
  UN_CUDA(cudaSetDevice(u->device));
  const long long n = (long long)(dims[0] / factor) * (dims[1] / factor) * (dims[2] / factor);
  k_block_mean<<<grid_for(n), 256, 0, u->stream>>>(src, dst, dims[0], dims[1], dims[2], factor);
  UN_CUDA(cudaGetLastError());
  UN_CUDA(cudaStreamSynchronize(u->stream));
  return CMI_OK;
}

int cmi_unet_upsample_nearest(cmi_unet *u, const float *src, const int32_t dims[3],
                              int32_t factor, float *dst) {
  if (!u || !src || !dst || !dims || factor < 1 || dims[0] <= 0 || dims[1] <= 0 || dims[2] <= 0)
    return fail(CMI_ERR_INVALID_ARGUMENT, "bad argument");
  UN_CUDA(cudaSetDevice(u->device));
  const long long n = (long long)dims[0] * dims[1] * dims[2] * factor * factor * factor;
  k_upsample_nearest<<<grid_for(n), 256, 0, u->stream>>>(src, dst, dims[0], dims[1], dims[2],
                                                        factor);
  UN_CUDA(cudaGetLastError());
  UN_CUDA(cudaStreamSynchronize(u->stream));
  return CMI_OK;
}

int cmi_unet_conv3(cmi_unet *u, const void *in, int32_t in_channels, const void *weights_packed,
                   const float *bias, void *out, int32_t out_channels, int32_t activation,
                   int32_t batch, const int32_t dims[3]) {
  if (!u || !in || !weights_packed || !out || !dims)
    return fail(CMI_ERR_INVALID_ARGUMENT, "null argument");
  UN_CUDA(cudaSetDevice(u->device));
  const int d[3] = {dims[0], dims[1], dims[2]};
  const Slice si{(bf16 *)in, in_channels, 0, in_channels};
  const Slice so{(bf16 *)out, out_channels, 0, out_channels};
  UN_TRY(conv_tc(u, si, (const bf16 *)weights_packed, bias, so, activation, batch, d));
  return check_err(u);
}

int cmi_unet_pack_weights(cmi_unet *u, const float *w, int32_t cout, int32_t cin,
                          int32_t flip, void *packed) {
  if (!u || !w || !packed || cout <= 0 || cin <= 0 || cout % 16 || cin % 16)
    return fail(CMI_ERR_INVALID_ARGUMENT, "bad argument (channel counts multiples of 16)");
  UN_CUDA(cudaSetDevice(u->device));
  int *map = nullptr;
  std::vector<int> id(cin);
  for (int k = 0; k < cin; ++k) id[k] = k;
  UN_CUDA(cudaMalloc(&map, sizeof(int) * cin));
  UN_CUDA(cudaMemcpy(map, id.data(), sizeof(int) * cin, cudaMemcpyHostToDevice));
  PackArgs a{};
  a.w = w;
  a.out = (bf16 *)packed;
  a.cout = cout;
  a.cin_real = cin;
  a.ci_of_storage = map;
  a.flip = flip;
  a.rows = flip ? cin : cout;
  a.kchan = flip ? cout : cin;
  a.xf = conv_xf(a.rows);
  k_pack<<<grid_for(27LL * cin * cout), 256, 0, u->stream>>>(a);
  const cudaError_t e = cudaStreamSynchronize(u->stream);
  cudaFree(map);
  if (e != cudaSuccess) return fail(CMI_ERR_CUDA, "pack: %s", cudaGetErrorString(e));
  return CMI_OK;
}

int cmi_unet_conv3_wgrad(cmi_unet *u, const void *x, int32_t cin, const void *dy, int32_t cout,
                         int32_t batch, const int32_t dims[3], float *dw) {
  if (!u || !x || !dy || !dw || !dims) return fail(CMI_ERR_INVALID_ARGUMENT, "null argument");
  if (cin % 16 || cout % 16) return fail(CMI_ERR_INVALID_ARGUMENT, "channels multiples of 16");
  UN_CUDA(cudaSetDevice(u->device));
  const int d[3] = {dims[0], dims[1], dims[2]};
  int *map = nullptr;
  std::vector<int> id(cin);
  for (int k = 0; k < cin; ++k) id[k] = k;
  UN_CUDA(cudaMalloc(&map, sizeof(int) * cin));
  UN_CUDA(cudaMemcpy(map, id.data(), sizeof(int) * cin, cudaMemcpyHostToDevice));
  UN_CUDA(cudaMemsetAsync(dw, 0, sizeof(float) * 27 * cin * cout, u->stream));
  UN_TRY(ensure_wg_part(u));
  const int rc = wgrad(u, Slice{(bf16 *)x, cin, 0, cin}, Slice{(bf16 *)dy, cout, 0, cout}, dw,
                       nullptr, map, cin, cout, batch, d);
  const cudaError_t e = cudaStreamSynchronize(u->stream);
  cudaFree(map);
  if (rc != CMI_OK) return rc;
  if (e != cudaSuccess) return fail(CMI_ERR_CUDA, "wgrad: %s", cudaGetErrorString(e));
  return CMI_OK;
}

}  // extern "C"
