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
//    5th-generation tensor cores.  A CTA owns 128 voxels (an 8x16x1 box of
//    one sample) = the 128 TMEM lanes of an M=128 tcgen05.mma; N = output
//    channels; one K step = one kernel tap x 16 input channels.  The CTA
//    loads its input box with a one-voxel halo once, by TMA (out-of-range
//    voxels read as zero: the padding), each 16-channel chunk as two 8-channel
//    halves, unswizzled, and each half as three copies of 10 x 8 x 4 voxels
//    shifted by -1, 0, +1 in y, so that within a copy the 8-voxel rows of both
//    z slices lie one 160-byte stride apart.  The A operand of a tap is the
//    copy of its y offset addressed at its x and z offsets (K-major, 16-byte
//    rows, 8-row groups 160 bytes apart, the two channel halves one
//    half-region apart).  A bulk
//    copy brings each step's weights (32-byte swizzled K-major) into a 4-stage
//    ring.  One thread issues the MMAs; tcgen05.commit frees a stage when its
//    MMA has read it.  The epilogue reads the accumulator with tcgen05.ld,
//    adds bias, applies leaky ReLU and stores BF16.
//    The input gradient of a convolution is the same kernel run on dy with
//    the weights flipped in space and transposed in channels.
//  * k_conv3_wgrad_tc: weight gradient dW[co][tap][ci] = sum_v dy[v][co] *
//    x[v + tap][ci], a reduction over all voxels, on the tensor cores: per tap
//    a GEMM with M = 128 output-channel rows (rows past the real count read
//    zeros), N = input channels and K = voxels, both operands MN-major
//    (channels contiguous).  A CTA owns a group of taps, one TMEM accumulator
//    each, and a range of 8x8x2 voxel tiles; per tile it loads dy and the
//    input with its halo by TMA (the input box of the forward kernel), and
//    every tap's B operand is that halo at the tap's offset.  At the end the
//    accumulators are read with tcgen05.ld and added to dW with FP32 atomics.
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

constexpr int kConvThreads = 128;
constexpr int kStages = 4;
constexpr int kTileX = 8, kTileY = 8, kTileZ = 2;  // 128 voxels, row r = x + 8 y + 64 z
// the input box with its one-voxel halo, per 8-channel half: three copies
// (y offsets -1, 0, +1) of 10 x 8 x 4 voxels of 16 bytes
constexpr int kHaloX = kTileX + 2, kHaloZ = kTileZ + 2;
constexpr int kCopyBytes = kHaloX * kTileY * kHaloZ * 16;  // 5120 B (a multiple of 128)
constexpr int kHalfBytes = 3 * kCopyBytes;
static_assert(kCopyBytes % 128 == 0, "TMA destinations are 128-byte aligned");
constexpr unsigned long long kWaitNs = 2000000000ull;
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
__device__ __forceinline__ unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
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
// bounded wait: false (and the error flag) after kWaitNs
__device__ __forceinline__ bool mbar_wait(uint64_t *b, uint32_t parity, uint32_t *err) {
  if (mbar_try(b, parity)) return true;
  const unsigned long long t0 = now_ns();
  while (!mbar_try(b, parity)) {
    if (now_ns() - t0 > kWaitNs) {
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
// shared-memory matrix descriptor without swizzle: 8 x 16-byte core matrices;
// lbo: from one core matrix to the next along K (K-major) or along M/N
// (MN-major), sbo: along the other dimension
__device__ __forceinline__ uint64_t plain_desc(const void *p, uint32_t lbo, uint32_t sbo) {
  const uint64_t a = (smem_u32(p) & 0x3FFFFu) >> 4;
  return a | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) | (1ull << 46);
}
// instruction descriptor: BF16 x BF16 -> F32, A and B K-major, M = 128
__host__ __device__ constexpr uint32_t idesc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(128 >> 4) << 24);
}

// ---------------------------------------------------------------------------
// 3x3x3 convolution on tensor cores
// ---------------------------------------------------------------------------
struct ConvArgs {
  const bf16 *wpack;     // [steps][npad][16], 32-byte swizzled rows
  const float *bias;     // [npad] (may be null)
  bf16 *out;             // output tensor base
  int out_ctot, out_c0;  // its channel count and this convolution's first channel
  int npad;              // output channels (multiple of 16, <= 256)
  int nchunk;            // 16-channel chunks of the input
  int dims[3];           // X, Y, Z
  int act;               // 1: leaky ReLU
  float slope;
  uint32_t *err;
};

__global__ void __launch_bounds__(kConvThreads) k_conv3_tc(const __grid_constant__ CUtensorMap in,
                                                           ConvArgs a) {
  extern __shared__ __align__(1024) unsigned char sm_raw[];
  // 1024-aligned base for the swizzled weight operands
  unsigned char *sm = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(sm_raw) + 1023) & ~(uintptr_t)1023);
  const int bbytes = a.npad * 32;
  unsigned char *sB = sm;                              // [kStages][npad * 32]
  unsigned char *sH = sB + kStages * bbytes;           // halo [nchunk][2][kHalfBytes]
  uint64_t *full = reinterpret_cast<uint64_t *>(sH + (size_t)a.nchunk * 2 * kHalfBytes);
  uint64_t *empty = full + kStages;
  uint64_t *done = empty + kStages;
  uint64_t *halo = done + 1;
  uint32_t *tslot = reinterpret_cast<uint32_t *>(halo + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tx = a.dims[0] / kTileX, ty = a.dims[1] / kTileY, tz = a.dims[2] / kTileZ;
  int t = blockIdx.x;
  const int bx = t % tx;
  t /= tx;
  const int by = t % ty;
  t /= ty;
  const int bz = t % tz;
  const int n = t / tz;
  const int x0 = bx * kTileX, y0 = by * kTileY, z0 = bz * kTileZ;
  const int nsteps = 27 * a.nchunk;
  const uint32_t ncols = a.npad <= 32 ? 32u : a.npad <= 64 ? 64u : a.npad <= 128 ? 128u : 256u;

  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    mbar_init(halo, 1);
    fence_mbar_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tslot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;

  bool ok = true;
  if (tid == 0) {
    const uint32_t idesc = idesc_bf16(a.npad);
    // the input box with its halo, once: chunk c, half h, y offset d at
    // sH + (2c + h) * kHalfBytes + d * kCopyBytes
    mbar_expect_tx(halo, (uint32_t)(a.nchunk * 2 * kHalfBytes));
    for (int c = 0; c < a.nchunk; ++c)
      for (int h = 0; h < 2; ++h)
        for (int d = 0; d < 3; ++d)
          tma_load_5d(sH + (size_t)(2 * c + h) * kHalfBytes + d * kCopyBytes, &in,
                      c * 16 + h * 8, x0 - 1, y0 - 1 + d, z0 - 1, n, halo);
    auto load = [&](int k) {
      const int s = k % kStages;
      mbar_expect_tx(&full[s], (uint32_t)bbytes);
      bulk_load(sB + s * bbytes, a.wpack + (size_t)k * a.npad * 16, (uint32_t)bbytes, &full[s]);
    };
    for (int k = 0; k < kStages && k < nsteps; ++k) load(k);
    ok = mbar_wait(halo, 0u, a.err);
    for (int k = 0; k < nsteps && ok; ++k) {
      const int s = k % kStages;
      const uint32_t ph = (uint32_t)(k / kStages) & 1u;
      ok = mbar_wait(&full[s], ph, a.err);
      if (!ok) break;
      tc_fence_after();
      // tap (dz, dy, dx) reads the input at (x + dx, y + dy, z + dz): copy dy + 1
      // of the halo, shifted by (dx + 1, dz + 1) voxels
      const int tap = k / a.nchunk, c = k - tap * a.nchunk;
      const int hz = tap / 9, hy = (tap / 3) % 3, hx = tap % 3;
      const unsigned char *a0 = sH + (size_t)(2 * c) * kHalfBytes + hy * kCopyBytes +
                                (hz * kTileY * kHaloX + hx) * 16;
      const uint64_t ad = plain_desc(a0, (uint32_t)kHalfBytes, (uint32_t)(kHaloX * 16));
      const uint64_t bd = sw32_desc(sB + s * bbytes);
      const uint32_t acc = k > 0 ? 1u : 0u;
      asm volatile(
          "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
          " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(tmem),
          "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
          : "memory");
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
              smem_u32(&empty[s]))
          : "memory");
      // refill the stage of the previous MMA (MMA k stays queued meanwhile)
      const int kp = k - 1;
      if (kp >= 0 && kp + kStages < nsteps) {
        const int sp = kp % kStages;
        ok = mbar_wait(&empty[sp], (uint32_t)(kp / kStages) & 1u, a.err);
        if (ok) load(kp + kStages);
      }
    }
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            smem_u32(done))
        : "memory");
  }
  __syncwarp();
  // every thread: the accumulator is complete
  const bool done_ok = __all_sync(0xffffffffu, mbar_wait(done, 0u, a.err));
  tc_fence_after();
  if (done_ok) {
    // row r = voxel (x0 + r % 8, y0 + (r / 8) % 8, z0 + r / 64); warp w owns lanes 32w..
    const int r = warp * 32 + lane;
    const int vx = x0 + (r & 7), vy = y0 + ((r >> 3) & 7), vz = z0 + (r >> 6);
    const size_t vox = (((size_t)n * a.dims[2] + vz) * a.dims[1] + vy) * a.dims[0] + vx;
    bf16 *dst = a.out + vox * a.out_ctot + a.out_c0;
    for (int j = 0; j < a.npad; j += 16) {
      uint32_t v[16];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)j;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,"
          "%13,%14,%15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
            "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
            "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      __align__(16) bf16 o[16];
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        float f = __uint_as_float(v[e]);
        if (a.bias) f += a.bias[j + e];
        if (a.act) f = f > 0.f ? f : f * a.slope;
        o[e] = __float2bfloat16_rn(f);
      }
      uint4 *d4 = reinterpret_cast<uint4 *>(dst + j);
      d4[0] = reinterpret_cast<const uint4 *>(o)[0];
      d4[1] = reinterpret_cast<const uint4 *>(o)[1];
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(ncols)
                 : "memory");
  }
}

// ---------------------------------------------------------------------------
// weight gradient on the tensor cores
// ---------------------------------------------------------------------------
struct WgradTcArgs {
  int cout;                  // dy channels (storage, multiple of 16, <= 128)
  int nchunk;                // 16-channel chunks of the input (N = 16 nchunk <= 256)
  int dims[3];
  int batch;
  int tap0, taps;            // taps of this launch's CTAs: blockIdx.y selects a group
  int taps_per_cta;
  uint32_t tmem_cols;        // power of two >= taps_per_cta * N (<= 256: two CTAs per SM)
  int tiles_per_cta;         // voxel tiles of one CTA (blockIdx.x)
  float *dw;                 // [cout_real][27][cin_real] (FP32, accumulated)
  const int *ci_map;         // storage input channel -> real input channel or -1
  int cin_real, cout_real;
  uint32_t *err;
};
constexpr int kDyGroupBytes = kTileX * kTileY * kTileZ * 16;  // 8 output channels: 2 KB
constexpr int kDyBytes = 16 * kDyGroupBytes;          // the 128 A rows (16 groups of 8)

__global__ void __launch_bounds__(kConvThreads) k_conv3_wgrad_tc(
    const __grid_constant__ CUtensorMap xmap, const __grid_constant__ CUtensorMap dymap,
    WgradTcArgs a) {
  extern __shared__ __align__(1024) unsigned char sm_raw[];
  unsigned char *sm = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(sm_raw) + 1023) & ~(uintptr_t)1023);
  unsigned char *sA = sm;                 // dy: [16 groups of 8 channels][16 y][8 x][8]
  unsigned char *sH = sA + kDyBytes;      // input halo: [2 nchunk][3 copies][4][8][10][8]
  uint64_t *loaded = reinterpret_cast<uint64_t *>(sH + (size_t)a.nchunk * 2 * kHalfBytes);
  uint64_t *mma_done = loaded + 1;
  uint32_t *tslot = reinterpret_cast<uint32_t *>(mma_done + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int N = a.nchunk * 16;
  const int t0 = a.tap0 + blockIdx.y * a.taps_per_cta;
  const int ntap = min(a.taps_per_cta, a.tap0 + a.taps - t0);
  const int tx = a.dims[0] / kTileX, ty = a.dims[1] / kTileY, tz = a.dims[2] / kTileZ;
  const int tiles = a.batch * tx * ty * tz;
  const int tile0 = blockIdx.x * a.tiles_per_cta, tile1 = min(tiles, tile0 + a.tiles_per_cta);

  // rows of A past the real output channels read zeros
  for (int i = tid; i < (kDyBytes - (a.cout / 8) * kDyGroupBytes) / 16; i += kConvThreads)
    reinterpret_cast<uint4 *>(sA + (a.cout / 8) * kDyGroupBytes)[i] = make_uint4(0, 0, 0, 0);
  if (tid == 0) {
    mbar_init(loaded, 1);
    mbar_init(mma_done, 1);
    fence_mbar_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tslot)),
                 "r"(a.tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  // the zeros above are generic-proxy writes that the MMAs read through the async proxy
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;

  bool ok = true;
  if (tid == 0 && ntap > 0) {
    // BF16 x BF16 -> F32, A and B MN-major, M = 128, N
    const uint32_t idesc = idesc_bf16(N) | (1u << 15) | (1u << 16);
    const uint32_t bytes = (uint32_t)((a.cout / 8) * kDyGroupBytes + a.nchunk * 2 * kHalfBytes);
    bool first = true;
    uint32_t phase = 0;
    for (int t = tile0; t < tile1 && ok; ++t) {
      int r = t;
      const int bx = r % tx;
      r /= tx;
      const int by = r % ty;
      r /= ty;
      const int bz = r % tz;
      const int n = r / tz;
      const int x0 = bx * kTileX, y0 = by * kTileY, z0 = bz * kTileZ;
      if (!first) {  // the previous tile's MMAs have read the buffers
        ok = mbar_wait(mma_done, phase ^ 1u, a.err);
        if (!ok) break;
      }
      mbar_expect_tx(loaded, bytes);
      for (int g = 0; g < a.cout / 8; ++g)
        tma_load_5d(sA + g * kDyGroupBytes, &dymap, g * 8, x0, y0, z0, n, loaded);
      for (int c = 0; c < a.nchunk; ++c)
        for (int h = 0; h < 2; ++h)
          for (int d = 0; d < 3; ++d)
            tma_load_5d(sH + (size_t)(2 * c + h) * kHalfBytes + d * kCopyBytes, &xmap,
                        c * 16 + h * 8, x0 - 1, y0 - 1 + d, z0 - 1, n, loaded);
      ok = mbar_wait(loaded, phase, a.err);
      if (!ok) break;
      tc_fence_after();
      for (int j = 0; j < ntap; ++j) {
        const int tap = t0 + j;
        const int hz = tap / 9, hy = (tap / 3) % 3, hx = tap % 3;
        const unsigned char *b0 = sH + hy * kCopyBytes + (hz * kTileY * kHaloX + hx) * 16;
        // K step k: tile rows q = 2k, 2k + 1 of 8 voxels (q = y + 8 z)
        for (int k = 0; k < kTileY * kTileZ / 2; ++k) {
          // A: core matrices of 8 voxels x 8 channels; LBO along K (next row),
          // SBO along M (next 8 output channels)
          const uint64_t ad = plain_desc(sA + k * 2 * kTileX * 16, kTileX * 16, kDyGroupBytes);
          // B: rows 2k, 2k + 1 of the tap's halo copy at its x and z offsets;
          // SBO along N (next 8 input channels: the next half region)
          const uint64_t bd =
              plain_desc(b0 + k * 2 * kHaloX * 16, kHaloX * 16, (uint32_t)kHalfBytes);
          const uint32_t acc = (first && k == 0) ? 0u : 1u;
          asm volatile(
              "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
              " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(
                  tmem + (uint32_t)(j * N)),
              "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
              : "memory");
        }
      }
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
              smem_u32(mma_done))
          : "memory");
      first = false;
      phase ^= 1u;
    }
    if (!first && ok) ok = mbar_wait(mma_done, phase ^ 1u, a.err);
    if (first) ok = false;  // no tile: nothing accumulated
  }
  __syncwarp();
  // thread 0 knows whether the accumulators are complete; share it
  __shared__ int s_have;
  if (tid == 0) s_have = ok ? 1 : 0;
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (s_have && warp * 32 < a.cout_real) {
    // lane = output channel (TMEM lane), columns = input channels
    const int co = warp * 32 + lane;
    for (int j = 0; j < ntap; ++j) {
      const int tap = t0 + j;
      for (int c = 0; c < N; c += 16) {
        uint32_t v[16];
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(j * N + c);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,"
            "%13,%14,%15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
              "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
              "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (co < a.cout_real) {
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            const int ci = a.ci_map[c + e];
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
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(a.tmem_cols)
                 : "memory");
  }
}

// bias gradient: db[c] = sum over voxels of dy[v][c]
__global__ void k_bias_grad(const bf16 *dy, int ctot, int c0, int cout, long long nvox,
                            float *db) {
  __shared__ float red[256];
  const int c = blockIdx.y;
  float s = 0.f;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nvox;
       v += (long long)gridDim.x * blockDim.x)
    s += __bfloat162float(dy[v * ctot + c0 + c]);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0 && c < cout) atomicAdd(&db[c], red[0]);
}

// ---------------------------------------------------------------------------
// elementwise and resampling kernels (channel slices of channels-last tensors)
// ---------------------------------------------------------------------------
// dy *= leaky'(y) (y is the activation output: same sign as its input)
__global__ void k_act_bwd(bf16 *dy, int dctot, int dc0, const bf16 *y, int yctot, int yc0,
                          int c, long long nvox, float slope) {
  const long long n = nvox * c;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long v = i / c;
    const int k = (int)(i - v * c);
    const float yy = __bfloat162float(y[v * yctot + yc0 + k]);
    bf16 &d = dy[v * dctot + dc0 + k];
    if (!(yy > 0.f)) d = __float2bfloat16_rn(__bfloat162float(d) * slope);
  }
}

// 2x2x2 average pooling: out (X/2, Y/2, Z/2) from in (X, Y, Z)
__global__ void k_pool2(const bf16 *in, int ictot, int ic0, bf16 *out, int octot, int oc0, int c,
                        int batch, int X, int Y, int Z) {
  const int Xo = X / 2, Yo = Y / 2, Zo = Z / 2;
  const long long n = (long long)batch * Xo * Yo * Zo * c;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    long long g = i / c;
    const int k = (int)(i - g * c);
    const int x = (int)(g % Xo);
    g /= Xo;
    const int y = (int)(g % Yo);
    g /= Yo;
    const int z = (int)(g % Zo);
    const long long s = g / Zo;
    float acc = 0.f;
    for (int d = 0; d < 8; ++d) {
      const size_t q = (((size_t)s * Z + 2 * z + (d >> 2)) * Y + 2 * y + ((d >> 1) & 1)) * X +
                       2 * x + (d & 1);
      acc += __bfloat162float(in[q * ictot + ic0 + k]);
    }
    const size_t o = (((size_t)s * Zo + z) * Yo + y) * Xo + x;
    out[o * octot + oc0 + k] = __float2bfloat16_rn(acc * 0.125f);
  }
}

// gradient of pooling, added to din: din[child] += dout[parent] / 8
__global__ void k_pool2_bwd_add(const bf16 *dout, int octot, int oc0, bf16 *din, int ictot,
                                int ic0, int c, int batch, int X, int Y, int Z) {
  const long long n = (long long)batch * X * Y * Z * c;
  const int Xo = X / 2, Yo = Y / 2, Zo = Z / 2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    long long g = i / c;
    const int k = (int)(i - g * c);
    const int x = (int)(g % X);
    g /= X;
    const int y = (int)(g % Y);
    g /= Y;
    const int z = (int)(g % Z);
    const long long s = g / Z;
    const size_t o = (((size_t)s * Zo + z / 2) * Yo + y / 2) * Xo + x / 2;
    const size_t q = (((size_t)s * Z + z) * Y + y) * X + x;
    bf16 &d = din[q * ictot + ic0 + k];
    d = __float2bfloat16_rn(__bfloat162float(d) +
                            0.125f * __bfloat162float(dout[o * octot + oc0 + k]));
  }
}

// nearest-neighbour upsampling by 2: out (2X, 2Y, 2Z)
__global__ void k_up2(const bf16 *in, int ictot, int ic0, bf16 *out, int octot, int oc0, int c,
                      int batch, int X, int Y, int Z) {
  const int X2 = 2 * X, Y2 = 2 * Y, Z2 = 2 * Z;
  const long long n = (long long)batch * X2 * Y2 * Z2 * c;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    long long g = i / c;
    const int k = (int)(i - g * c);
    const int x = (int)(g % X2);
    g /= X2;
    const int y = (int)(g % Y2);
    g /= Y2;
    const int z = (int)(g % Z2);
    const long long s = g / Z2;
    const size_t q = (((size_t)s * Z + z / 2) * Y + y / 2) * X + x / 2;
    const size_t o = (((size_t)s * Z2 + z) * Y2 + y) * X2 + x;
    out[o * octot + oc0 + k] = in[q * ictot + ic0 + k];
  }
}

// gradient of upsampling: dout (X, Y, Z) = sum of the 8 children in din (2X...)
__global__ void k_up2_bwd(const bf16 *din, int ictot, int ic0, bf16 *dout, int octot, int oc0,
                          int c, int batch, int X, int Y, int Z) {
  const long long n = (long long)batch * X * Y * Z * c;
  const int X2 = 2 * X, Y2 = 2 * Y;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    long long g = i / c;
    const int k = (int)(i - g * c);
    const int x = (int)(g % X);
    g /= X;
    const int y = (int)(g % Y);
    g /= Y;
    const int z = (int)(g % Z);
    const long long s = g / Z;
    float acc = 0.f;
    for (int d = 0; d < 8; ++d) {
      const size_t q = (((size_t)s * 2 * Z + 2 * z + (d >> 2)) * Y2 + 2 * y + ((d >> 1) & 1)) *
                           X2 + 2 * x + (d & 1);
      acc += __bfloat162float(din[q * ictot + ic0 + k]);
    }
    const size_t o = (((size_t)s * Z + z) * Y + y) * X + x;
    dout[o * octot + oc0 + k] = __float2bfloat16_rn(acc);
  }
}

// 1x1 output head (c -> 1, FP32 weights) fused with the MSE loss and its
// gradient.  pred = w . h + b; with a target: loss += (pred - t)^2,
// dpred = 2 (pred - t) / nvox, dh = dpred * w (BF16), dw += dpred * h,
// db += dpred.
__global__ void k_head(const bf16 *h, int hctot, int c, const float *w, const float *b,
                       long long nvox, float *pred, const float *target, bf16 *dh,
                       float *dw, float *db, float *loss, float over_weight) {
  __shared__ float red[256];
  __shared__ float redw[16][33];
  float l = 0.f, gb = 0.f;
  float gw[16] = {};
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nvox;
       v += (long long)gridDim.x * blockDim.x) {
    float hv[16];
    float p = b[0];
    for (int k = 0; k < c; ++k) {
      hv[k] = __bfloat162float(h[v * hctot + k]);
      p = fmaf(w[k], hv[k], p);
    }
    if (pred) pred[v] = p;
    if (target) {
      const float diff = p - target[v];
      // squared errors of predictions above the target (too neutral) weigh
      // over_weight: those fronts recover one cell per plain iteration
      const float wl = diff > 0.f ? over_weight : 1.f;
      l += wl * diff * diff;
      const float g = 2.f * wl * diff / (float)nvox;
      gb += g;
      for (int k = 0; k < hctot; ++k)
        dh[v * hctot + k] = __float2bfloat16_rn(k < c ? g * w[k] : 0.f);
      for (int k = 0; k < c; ++k) gw[k] = fmaf(g, hv[k], gw[k]);
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
};

__global__ void k_pack(PackArgs a) {
  const int nchunk = a.kchan / 16;
  const long long n = 27LL * nchunk * a.rows * 16;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
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
    const size_t step = (size_t)tap * nchunk + ch;
    const int half = (e >> 3) ^ ((r >> 2) & 1);
    a.out[(step * a.rows + r) * 16 + half * 8 + (e & 7)] = __float2bfloat16_rn(v);
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
__global__ void k_input(const float *f, bf16 *x, long long nvox) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nvox * 16;
       i += (long long)gridDim.x * blockDim.x) {
    const long long v = i / 16;
    const int k = (int)(i % 16);
    x[i] = __float2bfloat16_rn(k < kFeatures ? f[v * kFeatures + k] : 0.f);
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
};

namespace cmiu {

int dev_zero_alloc(void **p, size_t bytes) {
  UN_CUDA(cudaMalloc(p, bytes));
  UN_CUDA(cudaMemset(*p, 0, bytes));
  return CMI_OK;
}

void free_bufs(cmi_unet *u) {
  for (void *b : u->bufs) cudaFree(b);
  u->bufs.clear();
  u->batch = 0;
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

int ensure_buffers(cmi_unet *u, int batch, const int dims[3]) {
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

// tensor map of an input slice: dims (channels, X, Y, Z, batch), box (8, 10, 8, 4, 1):
// one 8-channel half of one y-shifted copy of a convolution tile's input with its
// x and z halo, unswizzled
int make_map(CUtensorMap *map, const Slice &s, int batch, const int dims[3]) {
  EncodeTiledFn enc;
  UN_TRY(get_encoder(&enc));
  const cuuint64_t gdim[5] = {(cuuint64_t)s.c, (cuuint64_t)dims[0], (cuuint64_t)dims[1],
                              (cuuint64_t)dims[2], (cuuint64_t)batch};
  const cuuint64_t row = (cuuint64_t)s.ctot * sizeof(bf16);
  const cuuint64_t gstride[4] = {row, row * dims[0], row * dims[0] * dims[1],
                                 row * dims[0] * dims[1] * dims[2]};
  const cuuint32_t box[5] = {8, kHaloX, kTileY, kHaloZ, 1};
  const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, (void *)(s.base + s.c0), gdim,
                         gstride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(CMI_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return CMI_OK;
}

size_t conv_smem(int npad, int nchunk) {
  return 1024 + (size_t)kStages * npad * 32 + (size_t)nchunk * 2 * kHalfBytes +
         (2 * kStages + 2) * 8 + 16;
}

// y = act(conv(x) + b) into out slice; wpack rows = out.c
int conv_tc(cmi_unet *u, const Slice &in, const bf16 *wpack, const float *bias, const Slice &out,
            int act, int batch, const int dims[3]) {
  if (dims[0] % kTileX || dims[1] % kTileY || dims[2] % kTileZ)
    return fail(CMI_ERR_INVALID_ARGUMENT, "grid %dx%dx%d is not a multiple of the 8x8x2 tile",
                dims[0], dims[1], dims[2]);
  if (in.c % 16 || out.c % 16 || out.c > 256 || out.c < 16)
    return fail(CMI_ERR_INVALID_ARGUMENT, "channel counts must be multiples of 16 (<= 256)");
  CUtensorMap map;
  UN_TRY(make_map(&map, in, batch, dims));
  ConvArgs a{};
  a.wpack = wpack;
  a.bias = bias;
  a.out = out.base;
  a.out_ctot = out.ctot;
  a.out_c0 = out.c0;
  a.npad = out.c;
  a.nchunk = in.c / 16;
  for (int k = 0; k < 3; ++k) a.dims[k] = dims[k];
  a.act = act;
  a.slope = u->slope;
  a.err = u->d_err;
  const size_t smem = conv_smem(out.c, a.nchunk);
  UN_CUDA(cudaFuncSetAttribute(k_conv3_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem));
  const int tiles = batch * (dims[0] / kTileX) * (dims[1] / kTileY) * (dims[2] / kTileZ);
  k_conv3_tc<<<tiles, kConvThreads, smem, u->stream>>>(map, a);
  UN_CUDA(cudaGetLastError());
  return CMI_OK;
}

// tensor map of a tile's dy: dims (channels, X, Y, Z, batch), box (8, 8, 8, 2, 1)
int make_dy_map(CUtensorMap *map, const Slice &s, int batch, const int dims[3]) {
  EncodeTiledFn enc;
  UN_TRY(get_encoder(&enc));
  const cuuint64_t gdim[5] = {(cuuint64_t)s.c, (cuuint64_t)dims[0], (cuuint64_t)dims[1],
                              (cuuint64_t)dims[2], (cuuint64_t)batch};
  const cuuint64_t row = (cuuint64_t)s.ctot * sizeof(bf16);
  const cuuint64_t gstride[4] = {row, row * dims[0], row * dims[0] * dims[1],
                                 row * dims[0] * dims[1] * dims[2]};
  const cuuint32_t box[5] = {8, kTileX, kTileY, kTileZ, 1};
  const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, (void *)(s.base + s.c0), gdim,
                         gstride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(CMI_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return CMI_OK;
}

int wgrad(cmi_unet *u, const Slice &x, const Slice &dy, float *dw, const int *ci_map,
          int cin_real, int cout_real, int batch, const int dims[3]) {
  if (dims[0] % kTileX || dims[1] % kTileY || dims[2] % kTileZ)
    return fail(CMI_ERR_INVALID_ARGUMENT, "grid %dx%dx%d is not a multiple of the 8x8x2 tile",
                dims[0], dims[1], dims[2]);
  if (x.c % 16 || dy.c % 16 || x.c < 16 || x.c > 256 || dy.c < 16 || dy.c > 128)
    return fail(CMI_ERR_NOT_SUPPORTED,
                "weight gradient: input channels must be 16..256, output channels 16..128, "
                "multiples of 16");
  CUtensorMap xm, dym;
  UN_TRY(make_map(&xm, x, batch, dims));
  UN_TRY(make_dy_map(&dym, dy, batch, dims));
  WgradTcArgs a{};
  a.cout = dy.c;
  a.nchunk = x.c / 16;
  for (int k = 0; k < 3; ++k) a.dims[k] = dims[k];
  a.batch = batch;
  a.tap0 = 0;
  a.taps = 27;
  const int N = x.c;
  a.taps_per_cta = std::min(27, 256 / N);
  uint32_t cols = 32;
  while (cols < (uint32_t)(a.taps_per_cta * N)) cols <<= 1;
  a.tmem_cols = cols;
  const int groups = (27 + a.taps_per_cta - 1) / a.taps_per_cta;
  const int tiles = batch * (dims[0] / kTileX) * (dims[1] / kTileY) * (dims[2] / kTileZ);
  // about two CTAs per SM over all tap groups
  const int want = std::max(1, 2 * 148 / groups);
  a.tiles_per_cta = (tiles + want - 1) / want;
  const int ctas = (tiles + a.tiles_per_cta - 1) / a.tiles_per_cta;
  a.dw = dw;
  a.ci_map = ci_map;
  a.cin_real = cin_real;
  a.cout_real = cout_real;
  a.err = u->d_err;
  const size_t smem = 1024 + (size_t)kDyBytes + (size_t)a.nchunk * 2 * kHalfBytes + 64;
  UN_CUDA(cudaFuncSetAttribute(k_conv3_wgrad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem));
  k_conv3_wgrad_tc<<<dim3(ctas, groups), kConvThreads, smem, u->stream>>>(xm, dym, a);
  UN_CUDA(cudaGetLastError());
  return CMI_OK;
}

// packs every layer's weights from the FP32 master parameters
int pack_all(cmi_unet *u) {
  for (Layer &l : u->L) {
    PackArgs a{};
    a.w = u->p + l.w_off;
    a.cout = l.cout;
    a.cin_real = l.cin_real;
    a.ci_of_storage = l.d_map;
    a.out = l.wf;
    a.rows = l.npad;
    a.kchan = l.kin;
    a.flip = 0;
    k_pack<<<grid_for(27LL * l.kin * l.npad), 256, 0, u->stream>>>(a);
    a.out = l.wd;
    a.rows = l.kin;
    a.kchan = l.npad;
    a.flip = 1;
    k_pack<<<grid_for(27LL * l.kin * l.npad), 256, 0, u->stream>>>(a);
    // bias padded to npad (zero beyond cout)
    UN_CUDA(cudaMemsetAsync(l.bias_pad, 0, sizeof(float) * l.npad, u->stream));
    UN_CUDA(cudaMemcpyAsync(l.bias_pad, u->p + l.b_off, sizeof(float) * l.cout,
                            cudaMemcpyDeviceToDevice, u->stream));
  }
  UN_CUDA(cudaGetLastError());
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

// forward pass from u->X0; writes u->pred
int forward(cmi_unet *u, int batch, const int d1[3]) {
  if (!u->packed) UN_TRY(pack_all(u));
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
  k_pool2<<<grid_for(v1 / 8 * c.s1), 256, 0, u->stream>>>(u->CAT1, c.cat1, c.s2, u->P1, c.s1, 0,
                                                           c.s1, batch, d1[0], d1[1], d1[2]);
  // level 2
  UN_TRY(conv_tc(u, S(u->P1, c.s1, 0, c.s1), L[2].wf, L[2].bias_pad, S(u->E2A, c.s2, 0, c.s2), 1,
                 batch, d2));
  UN_TRY(conv_tc(u, S(u->E2A, c.s2, 0, c.s2), L[3].wf, L[3].bias_pad,
                 S(u->CAT2, c.cat2, c.s3, c.s2), 1, batch, d2));
  k_pool2<<<grid_for(v1 / 64 * c.s2), 256, 0, u->stream>>>(u->CAT2, c.cat2, c.s3, u->P2, c.s2, 0,
                                                            c.s2, batch, d2[0], d2[1], d2[2]);
  // level 3
  UN_TRY(conv_tc(u, S(u->P2, c.s2, 0, c.s2), L[4].wf, L[4].bias_pad, S(u->BA, c.s3, 0, c.s3), 1,
                 batch, d3));
  UN_TRY(conv_tc(u, S(u->BA, c.s3, 0, c.s3), L[5].wf, L[5].bias_pad, S(u->BB, c.s3, 0, c.s3), 1,
                 batch, d3));
  // up to level 2
  k_up2<<<grid_for(v1 / 8 * c.s3), 256, 0, u->stream>>>(u->BB, c.s3, 0, u->CAT2, c.cat2, 0, c.s3,
                                                         batch, d3[0], d3[1], d3[2]);
  UN_TRY(conv_tc(u, S(u->CAT2, c.cat2, 0, c.cat2), L[6].wf, L[6].bias_pad,
                 S(u->D2A, c.s2, 0, c.s2), 1, batch, d2));
  UN_TRY(conv_tc(u, S(u->D2A, c.s2, 0, c.s2), L[7].wf, L[7].bias_pad, S(u->D2B, c.s2, 0, c.s2), 1,
                 batch, d2));
  // up to level 1
  k_up2<<<grid_for(v1 * c.s2), 256, 0, u->stream>>>(u->D2B, c.s2, 0, u->CAT1, c.cat1, 0, c.s2,
                                                     batch, d2[0], d2[1], d2[2]);
  UN_TRY(conv_tc(u, S(u->CAT1, c.cat1, 0, c.cat1), L[8].wf, L[8].bias_pad,
                 S(u->D1A, c.s1, 0, c.s1), 1, batch, d1));
  UN_TRY(conv_tc(u, S(u->D1A, c.s1, 0, c.s1), L[9].wf, L[9].bias_pad, S(u->D1B, c.s1, 0, c.s1), 1,
                 batch, d1));
  UN_CUDA(cudaGetLastError());
  return CMI_OK;
}

// loss + backward from u->D1B etc. (forward must have run); gradients into u->g
int backward(cmi_unet *u, const float *target, int batch, const int d1[3]) {
  const Chans c = chans(u);
  const int d2[3] = {d1[0] / 2, d1[1] / 2, d1[2] / 2};
  const int d3[3] = {d1[0] / 4, d1[1] / 4, d1[2] / 4};
  const long long v1 = (long long)batch * d1[0] * d1[1] * d1[2];
  const long long v2 = v1 / 8, v3 = v1 / 64;
  auto S = [](bf16 *b, int ctot, int c0, int cc) { return Slice{b, ctot, c0, cc}; };
  std::vector<Layer> &L = u->L;
  UN_CUDA(cudaMemsetAsync(u->g, 0, sizeof(float) * u->nparams, u->stream));
  UN_CUDA(cudaMemsetAsync(u->d_loss, 0, sizeof(float), u->stream));
  k_head<<<grid_for(v1), 256, 0, u->stream>>>(u->D1B, c.s1, c.c1, u->p + u->head_w,
                                               u->p + u->head_b, v1, u->pred, target, u->gD1B,
                                               u->g + u->head_w, u->g + u->head_b, u->d_loss,
                                               u->over_weight);
  const float sl = u->slope;
  // one convolution layer backwards: dy (in place) *= act'(y); wgrad; input gradient
  auto layer_bwd = [&](int li, const Slice &x, const Slice &y, const Slice &dy, const Slice *dx,
                       int b, const int *dims, long long nv) -> int {
    k_act_bwd<<<grid_for(nv * dy.c), 256, 0, u->stream>>>(dy.base, dy.ctot, dy.c0, y.base, y.ctot,
                                                         y.c0, dy.c, nv, sl);
    UN_TRY(wgrad(u, x, dy, u->g + L[li].w_off, L[li].d_map, L[li].cin_real, L[li].cout, b,
                 dims));
    k_bias_grad<<<dim3(64, dy.c), 256, 0, u->stream>>>(dy.base, dy.ctot, dy.c0, L[li].cout, nv,
                                                       u->g + L[li].b_off);
    if (dx) UN_TRY(conv_tc(u, dy, L[li].wd, nullptr, *dx, 0, b, dims));
    return CMI_OK;
  };
  // level 1 decoder
  {
    const Slice dx = S(u->gD1A, c.s1, 0, c.s1);
    UN_TRY(layer_bwd(9, S(u->D1A, c.s1, 0, c.s1), S(u->D1B, c.s1, 0, c.s1),
                     S(u->gD1B, c.s1, 0, c.s1), &dx, batch, d1, v1));
  }
  {
    const Slice dx = S(u->gCAT1, c.cat1, 0, c.cat1);
    UN_TRY(layer_bwd(8, S(u->CAT1, c.cat1, 0, c.cat1), S(u->D1A, c.s1, 0, c.s1),
                     S(u->gD1A, c.s1, 0, c.s1), &dx, batch, d1, v1));
  }
  // up1 backward: gD2B = sum of children of gCAT1[0:s2]
  k_up2_bwd<<<grid_for(v2 * c.s2), 256, 0, u->stream>>>(u->gCAT1, c.cat1, 0, u->gD2B, c.s2, 0,
                                                         c.s2, batch, d2[0], d2[1], d2[2]);
  {
    const Slice dx = S(u->gD2A, c.s2, 0, c.s2);
    UN_TRY(layer_bwd(7, S(u->D2A, c.s2, 0, c.s2), S(u->D2B, c.s2, 0, c.s2),
                     S(u->gD2B, c.s2, 0, c.s2), &dx, batch, d2, v2));
  }
  {
    const Slice dx = S(u->gCAT2, c.cat2, 0, c.cat2);
    UN_TRY(layer_bwd(6, S(u->CAT2, c.cat2, 0, c.cat2), S(u->D2A, c.s2, 0, c.s2),
                     S(u->gD2A, c.s2, 0, c.s2), &dx, batch, d2, v2));
  }
  // up2 backward: gBB = sum of children of gCAT2[0:s3]
  k_up2_bwd<<<grid_for(v3 * c.s3), 256, 0, u->stream>>>(u->gCAT2, c.cat2, 0, u->gBB, c.s3, 0,
                                                         c.s3, batch, d3[0], d3[1], d3[2]);
  {
    const Slice dx = S(u->gBA, c.s3, 0, c.s3);
    UN_TRY(layer_bwd(5, S(u->BA, c.s3, 0, c.s3), S(u->BB, c.s3, 0, c.s3),
                     S(u->gBB, c.s3, 0, c.s3), &dx, batch, d3, v3));
  }
  {
    const Slice dx = S(u->gP2, c.s2, 0, c.s2);
    UN_TRY(layer_bwd(4, S(u->P2, c.s2, 0, c.s2), S(u->BA, c.s3, 0, c.s3),
                     S(u->gBA, c.s3, 0, c.s3), &dx, batch, d3, v3));
  }
  // pool2 backward, added to the skip gradient gCAT2[s3 : s3 + s2]
  k_pool2_bwd_add<<<grid_for(v2 * c.s2), 256, 0, u->stream>>>(
      u->gP2, c.s2, 0, u->gCAT2, c.cat2, c.s3, c.s2, batch, d2[0], d2[1], d2[2]);
  {
    const Slice dx = S(u->gE2A, c.s2, 0, c.s2);
    UN_TRY(layer_bwd(3, S(u->E2A, c.s2, 0, c.s2), S(u->CAT2, c.cat2, c.s3, c.s2),
                     S(u->gCAT2, c.cat2, c.s3, c.s2), &dx, batch, d2, v2));
  }
  {
    const Slice dx = S(u->gP1, c.s1, 0, c.s1);
    UN_TRY(layer_bwd(2, S(u->P1, c.s1, 0, c.s1), S(u->E2A, c.s2, 0, c.s2),
                     S(u->gE2A, c.s2, 0, c.s2), &dx, batch, d2, v2));
  }
  k_pool2_bwd_add<<<grid_for(v1 * c.s1), 256, 0, u->stream>>>(
      u->gP1, c.s1, 0, u->gCAT1, c.cat1, c.s2, c.s1, batch, d1[0], d1[1], d1[2]);
  {
    const Slice dx = S(u->gE1A, c.s1, 0, c.s1);
    UN_TRY(layer_bwd(1, S(u->E1A, c.s1, 0, c.s1), S(u->CAT1, c.cat1, c.s2, c.s1),
                     S(u->gCAT1, c.cat1, c.s2, c.s1), &dx, batch, d1, v1));
  }
  UN_TRY(layer_bwd(0, S(u->X0, 16, 0, 16), S(u->E1A, c.s1, 0, c.s1), S(u->gE1A, c.s1, 0, c.s1),
                   nullptr, batch, d1, v1));
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
  UN_CUDA(cudaSetDevice(u->device));
  UN_TRY(ensure_buffers(u, batch, dims));
  const long long v1 = (long long)batch * dims[0] * dims[1] * dims[2];
  k_input<<<grid_for(v1 * 16), 256, 0, u->stream>>>(in, u->X0, v1);
  UN_CUDA(cudaGetLastError());
  return CMI_OK;
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
  *out = u;
  return CMI_OK;
}

int cmi_unet_destroy(cmi_unet *u) {
  if (!u) return CMI_OK;
  cudaSetDevice(u->device);
  if (u->stream) cudaStreamSynchronize(u->stream);
  free_bufs(u);
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
                                               nullptr, nullptr, nullptr, 1.f);
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
  const int rc = wgrad(u, Slice{(bf16 *)x, cin, 0, cin}, Slice{(bf16 *)dy, cout, 0, cout}, dw, map,
                       cin, cout, batch, d);
  const cudaError_t e = cudaStreamSynchronize(u->stream);
  cudaFree(map);
  if (rc != CMI_OK) return rc;
  if (e != cudaSuccess) return fail(CMI_ERR_CUDA, "wgrad: %s", cudaGetErrorString(e));
  return CMI_OK;
}

}  // extern "C"
