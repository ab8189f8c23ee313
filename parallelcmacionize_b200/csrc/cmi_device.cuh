// Device-side data layout and helpers of the B200 transport engine.
//
// Internal header of cmi_engine.cu (single translation unit): structures in
// HBM, TravelDirection tables, the counter-based and the reference random
// generators.
#pragma once

#include <cfloat>
#include <cstdint>
#include <cuda_runtime.h>

#include "cmacionize/ranlxd.h"

namespace cmi {

constexpr int kNumDirections = 27;
constexpr uint32_t kOutside = 0xffffffffu;
constexpr int kInside = 0;

// ---------------------------------------------------------------------------
// TravelDirections (TravelDirections.hpp:46-403) as axis-sign triples.
// Packed code of a direction: bits [2a, 2a+1] hold sign(axis a) + 1.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int dir_from_signs(int sx, int sy, int sz) {
  // INSIDE 0, CORNER 1-8, EDGE_X 9-12, EDGE_Y 13-16, EDGE_Z 17-20, FACE 21-26
  return (sx == 0 && sy == 0 && sz == 0) ? 0
         : (sx != 0 && sy != 0 && sz != 0)
             ? 1 + (sx < 0) * 4 + (sy < 0) * 2 + (sz < 0)
         : (sx == 0 && sy != 0 && sz != 0) ? 9 + (sy < 0) * 2 + (sz < 0)
         : (sy == 0 && sx != 0 && sz != 0) ? 13 + (sx < 0) * 2 + (sz < 0)
         : (sz == 0 && sx != 0 && sy != 0) ? 17 + (sx < 0) * 2 + (sy < 0)
         : (sx != 0)                       ? 21 + (sx < 0)
         : (sy != 0)                       ? 23 + (sy < 0)
                                           : 25 + (sz < 0);
}

struct DirectionTables {
  uint8_t sign_code[32];  // per direction
  uint8_t mirror[32];     // output_to_input_direction
  uint8_t mask_dir[64];   // 6-bit out-of-range mask -> direction (255: invalid)
};

inline DirectionTables make_direction_tables() {
  DirectionTables t{};
  for (int sx = -1; sx <= 1; ++sx)
    for (int sy = -1; sy <= 1; ++sy)
      for (int sz = -1; sz <= 1; ++sz) {
        const int d = dir_from_signs(sx, sy, sz);
        t.sign_code[d] = (uint8_t)((sx + 1) | ((sy + 1) << 2) | ((sz + 1) << 4));
        t.mirror[d] = (uint8_t)dir_from_signs(-sx, -sy, -sz);
      }
  for (int m = 0; m < 64; ++m) {
    int s[3];
    bool ok = true;
    for (int a = 0; a < 3; ++a) {
      const int hi = (m >> (5 - 2 * a)) & 1, lo = (m >> (4 - 2 * a)) & 1;
      ok = ok && !(hi && lo);
      s[a] = hi ? 1 : (lo ? -1 : 0);
    }
    t.mask_dir[m] = ok ? (uint8_t)dir_from_signs(s[0], s[1], s[2]) : (uint8_t)255;
  }
  return t;
}

__device__ __forceinline__ int sign_of(uint8_t code, int axis) {
  return (int)((code >> (2 * axis)) & 3u) - 1;
}

// ---------------------------------------------------------------------------
// Structures resident in HBM.
// ---------------------------------------------------------------------------
struct alignas(16) DevSubgrid {
  double anchor[3];
  double cell_size[3];
  double inv_cell_size[3];
  float cell_size_f[3];
  int32_t ncell[3];
  int32_t ncells;         // nx * ny * nz
  int32_t padded_cells;   // ncells rounded up to a multiple of 4 (16 B in FP32)
  int64_t field_offset;   // first cell in the flat field arrays (multiple of 4)
  uint32_t instance;
  uint32_t ngb[kNumDirections];
};

struct alignas(16) DevInstance {
  double jfac;            // L_tot / N / V_cell (DensitySubGrid.hpp:1633)
  double alpha;
  double sigma;
  double total_luminosity;
  uint64_t num_photon;
  uint32_t first_subgrid, num_subgrids;
  uint32_t first_source, num_sources;
  int64_t num_cells;
  uint32_t frozen;        // 1: converged, emits nothing and keeps x_H (run until converged)
  float reemission;       // probability that an absorbed packet is re-emitted
};

struct alignas(16) DevSource {
  double position[3];
  double luminosity;
  float pos_cell[3];      // position in cell units relative to its subgrid
  uint32_t subgrid;       // global subgrid index
  uint32_t instance;
  uint32_t local_index;   // index among the instance's sources
};

// Work unit of a wavefront round: packets [begin, begin+count) of the sorted
// arena, all waiting to enter `subgrid`.
struct alignas(16) Chunk {
  uint32_t subgrid;
  uint32_t count;
  uint32_t begin;
  uint32_t rem;  // chunks of this subgrid from this one to its last, inclusive
};

// Per-iteration counters of one instance (device side of cmi_stats).
struct alignas(16) DevStats {
  unsigned long long emitted, absorbed, escaped, crossings, transits;
  double dx_sum;
  uint32_t flags, rounds;
  unsigned long long reemitted;
};

// Control block of the wavefront.
struct alignas(16) RoundState {
  uint32_t chunk_next;     // chunks claimed in this round
  uint32_t num_chunks;     // chunks of this round
  uint32_t arena_count;    // packets appended by this round
  uint32_t total_in;       // packets in the sorted arena
  uint32_t emit_total;     // packets emitted this iteration
  uint32_t iteration;      // Philox stream of the current iteration
  uint64_t seed;
  uint32_t flags;          // CMI_FLAG_* of the whole context
  uint32_t rounds_active;
  uint32_t capacity;       // arena capacity (packets)
  uint32_t round_index;    // walks started this iteration (graph loop)
  uint32_t pad[2];
};

// FP64 packet: the reference Photon layout (80 B); `meta` (the reserved
// slot) carries the input TravelDirection.
struct alignas(16) Packet64 {
  double pos[3];
  double dir[3];
  double tau;
  double sigma;
  double weight;
  int32_t type;
  uint32_t meta;
};
static_assert(sizeof(Packet64) == 80, "Packet64 must match cmi_photon");

// FP32 packet (32 B, one sector): position in cell units relative to the
// subgrid it is about to enter, direction, remaining target optical depth.
struct alignas(16) Packet32 {
  float pos[3];
  float dir[3];
  float tau;
  uint32_t meta;  // low 5 bits: input TravelDirection
};
static_assert(sizeof(Packet32) == 32, "Packet32 is one 32-byte sector");

// Mixed-precision packet (64 B, two sectors): the reference's absolute FP64
// position and direction, the remaining target optical depth in FP32.
struct alignas(16) PacketM {
  double pos[3];
  double dir[3];
  float tau;
  uint32_t meta;  // low 5 bits: input TravelDirection
  uint32_t pad[2];
};
static_assert(sizeof(PacketM) == 64, "PacketM is two 32-byte sectors");

// The three packet records, as a template argument of the kernels that
// create or move packets.
enum PacketKind : int { kPk64 = 0, kPk32 = 1, kPkM = 2 };
template <int K> struct PacketOf { using type = Packet64; };
template <> struct PacketOf<kPk32> { using type = Packet32; };
template <> struct PacketOf<kPkM> { using type = PacketM; };

// FP32 target optical depth of a mixed-precision packet: round to nearest;
// a positive depth below the FP32 range becomes the smallest subnormal, not
// 0, so every packet the reference walks is walked.
__host__ __device__ __forceinline__ float tau32(double tau) {
  const float f = (float)tau;
  if (f == 0.f && tau > 0.) {
#ifdef __CUDA_ARCH__
    return __int_as_float(1);
#else
    return 1.40129846e-45f;
#endif
  }
  return f;
}

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as easy
// as 1, 2, 3", SC'11).
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ void mulhilo32(uint32_t a, uint32_t b, uint32_t &hi,
                                                   uint32_t &lo) {
#ifdef __CUDA_ARCH__
  lo = a * b;
  hi = __umulhi(a, b);
#else
  const uint64_t p = (uint64_t)a * b;
  lo = (uint32_t)p;
  hi = (uint32_t)(p >> 32);
#endif
}

__host__ __device__ __forceinline__ void philox4x32_10(const uint32_t in[4], uint32_t k0,
                                                       uint32_t k1, uint32_t out[4]) {
  uint32_t c0 = in[0], c1 = in[1], c2 = in[2], c3 = in[3];
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
  for (int r = 0; r < 10; ++r) {
    if (r > 0) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(0xD2511F53u, c0, hi0, lo0);
    mulhilo32(0xCD9E8D57u, c2, hi1, lo1);
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

constexpr uint32_t kPhiloxPacketTag = 0x434D4901u;
constexpr uint32_t kPhiloxSplitTag = 0x434D4902u;

// Isotropic direction and exponential optical depth of one packet
// (testDensitySubGrid_omp.cpp:529-545, 585-586, drawn from Philox).
__device__ __forceinline__ void philox_packet(uint64_t seed, uint32_t instance,
                                              uint32_t iteration, uint64_t packet,
                                              double dir[3], double &tau) {
  const uint32_t ctr[4] = {(uint32_t)packet, (uint32_t)(packet >> 32), iteration,
                           kPhiloxPacketTag};
  uint32_t w[4];
  philox4x32_10(ctr, (uint32_t)seed, (uint32_t)(seed >> 32) + instance, w);
  const double u0 = ((double)w[0] + 0.5) * (1.0 / 4294967296.0);
  const double u1 = ((double)w[1] + 0.5) * (1.0 / 4294967296.0);
  const uint64_t k53 = ((uint64_t)w[2] << 21) ^ (uint64_t)(w[3] >> 11);
  const double u2 = ((double)k53 + 0.5) * (1.0 / 9007199254740992.0);
  const double cost = 2. * u0 - 1.;
  const double phi = 2. * 3.14159265358979323846 * u1;
  const double s2 = 1. - cost * cost;
  const double sint = sqrt((s2 < 0.) ? 0. : s2);
  double sp, cp;
  sincos(phi, &sp, &cp);
  dir[0] = sint * cp;
  dir[1] = sint * sp;
  dir[2] = cost;
  tau = -log(u2);
}

// Reemission of an absorbed packet (do_reemission, testDensitySubGrid_omp.cpp:
// 675-702): with probability p a new isotropic direction and optical depth.
// The draws come from Philox with the instance's emission key and a counter
// made of the absorption position (h0..h2), the iteration, the number of
// earlier reemissions of the packet in this subgrid visit and a tag of their
// own, so they are independent of the emission streams and a packet absorbed
// twice at the same position (a move below the coordinate's resolution) still
// draws afresh.  They use only
// correctly rounded operations (no sin/cos/log), so the oracle's host copy of
// this function draws the same bits: the direction by Marsaglia's method (a
// point of the unit disc, rejection from the square; attempt k uses tag + k),
// the optical depth -ln u by the series ln m = 2 atanh((m - 1) / (m + 1))
// after an exact power-of-two range reduction.
constexpr uint32_t kPhiloxReemitTag = 0x434D4952u;
// reemissions of one packet in one subgrid visit before it counts as
// absorbed (probability p^1024): keeps every walk finite whatever the draws
constexpr uint32_t kMaxReemissions = 1024u;

__device__ __forceinline__ uint32_t reemit_hash(double x) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(x);
  return (uint32_t)b ^ (uint32_t)(b >> 32);
}

// -ln(u) for u in (0, 1): u = m 2^e with m in [sqrt(1/2), sqrt(2)), then
// ln m = 2 (s + s^3/3 + ... + s^31/31), s = (m - 1) / (m + 1), |s| < 0.1716
__device__ __forceinline__ double reemit_neg_log(double u) {
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

__device__ __forceinline__ bool reemit_draw(uint64_t seed, uint32_t instance, uint32_t iteration,
                                            uint32_t h0, uint32_t h1, uint32_t h2, uint32_t count,
                                            double p, double dir[3], double &tau) {
  const double inv32 = 1.0 / 4294967296.0;
  for (uint32_t k = 0; k < 16u; ++k) {
    const uint32_t ctr[4] = {h0, h1, h2 ^ iteration, kPhiloxReemitTag + (count << 4) + k};
    uint32_t w[4];
    philox4x32_10(ctr, (uint32_t)seed, (uint32_t)(seed >> 32) + instance, w);
    if (k == 0u && !(((double)w[0] + 0.5) * inv32 < p)) return false;
    const double x1 = 2. * (((double)w[1] + 0.5) * inv32) - 1.;
    const double x2 = 2. * (((double)w[2] + 0.5) * inv32) - 1.;
    const double s = x1 * x1 + x2 * x2;
    if (s < 1.) {
      const double f = 2. * sqrt(1. - s);
      dir[0] = x1 * f;
      dir[1] = x2 * f;
      dir[2] = 1. - 2. * s;
      tau = reemit_neg_log(((double)w[3] + 0.5) * inv32);
      return true;
    }
  }
  dir[0] = 0.;  // 16 rejections in a row: probability 0.21^16
  dir[1] = 0.;
  dir[2] = 1.;
  tau = 1.;
  return true;
}

// Out-of-line copy for the walk kernels (the draw is rare; inlined it would
// cost the walk loop registers): out = direction (3), optical depth.
__device__ __noinline__ bool reemit_draw_call(uint64_t seed, uint32_t instance,
                                              uint32_t iteration, uint32_t h0, uint32_t h1,
                                              uint32_t h2, uint32_t count, double p,
                                              double *out) {
  double d[3], tau;
  if (count >= kMaxReemissions ||
      !reemit_draw(seed, instance, iteration, h0, h1, h2, count, p, d, tau))
    return false;
  out[0] = d[0];
  out[1] = d[1];
  out[2] = d[2];
  out[3] = tau;
  return true;
}

// ranlxd, the reference's generator (shared with the host C++ surface)
using Ranlux = cmi_ranlxd::Ranlxd;

// ---------------------------------------------------------------------------
// Correctly rounded sin, cos and -log for the replay of the reference's
// emission streams (get_random_direction and fill_buffer,
// testDensitySubGrid_omp.cpp:529-597): the same uniform draws give the same
// directions and optical depths on every machine, independent of any math
// library's last-bit behaviour.
//
// Double-double arithmetic (Dekker 1971; Knuth's TwoSum): a value is hi + lo
// with |lo| <= ulp(hi) / 2; products are split exactly with a fused
// multiply-add.  sin / cos: Cody-Waite reduction of x in [0, 8) by pi/2 held
// in three parts (P1 has three trailing zero bits, so k * P1 is exact for
// k <= 4 and x - k * P1 is exact by Sterbenz's lemma), then the Taylor
// series of sin and cos to x^29 / 29! in Horner form on |r| <= pi/4.  -log u:
// u = m 2^e with m in [sqrt(1/2), sqrt(2)), ln m = 2 atanh(s), s = (m - 1) /
// (m + 1), series to s^45 / 45, plus e ln 2 (ln 2 as a double-double).  The
// evaluation error is about 1e-30 relative, so rounding hi + lo to a double
// gives the correctly rounded result except when the exact value lies within
// about 1e-14 ulp of a rounding midpoint.
// ---------------------------------------------------------------------------
struct DD {
  double hi, lo;
};
__device__ __forceinline__ DD dd_two_sum(double a, double b) {
  const double s = __dadd_rn(a, b);
  const double bb = __dsub_rn(s, a);
  return {s, __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb))};
}
__device__ __forceinline__ DD dd_fast_two_sum(double a, double b) {  // |a| >= |b|
  const double s = __dadd_rn(a, b);
  return {s, __dsub_rn(b, __dsub_rn(s, a))};
}
__device__ __forceinline__ DD dd_two_prod(double a, double b) {
  const double p = __dmul_rn(a, b);
  return {p, __fma_rn(a, b, -p)};
}
__device__ __forceinline__ DD dd_add(DD a, DD b) {
  DD s = dd_two_sum(a.hi, b.hi);
  const DD t = dd_two_sum(a.lo, b.lo);
  s.lo = __dadd_rn(s.lo, t.hi);
  s = dd_fast_two_sum(s.hi, s.lo);
  s.lo = __dadd_rn(s.lo, t.lo);
  return dd_fast_two_sum(s.hi, s.lo);
}
__device__ __forceinline__ DD dd_mul(DD a, DD b) {
  DD p = dd_two_prod(a.hi, b.hi);
  p.lo = __dadd_rn(p.lo, __dadd_rn(__dmul_rn(a.hi, b.lo), __dmul_rn(a.lo, b.hi)));
  return dd_fast_two_sum(p.hi, p.lo);
}
__device__ __forceinline__ DD dd_div_d(DD a, double b) {
  const double q1 = __ddiv_rn(a.hi, b);
  const DD p = dd_two_prod(q1, b);
  DD s = dd_two_sum(a.hi, -p.hi);
  s.lo = __dadd_rn(__dsub_rn(s.lo, p.lo), a.lo);
  return dd_fast_two_sum(q1, __ddiv_rn(__dadd_rn(s.hi, s.lo), b));
}
__device__ __forceinline__ DD dd_div(DD a, DD b) {
  const double q1 = __ddiv_rn(a.hi, b.hi);
  DD r = dd_add(a, dd_mul({-q1, 0.}, b));
  const double q2 = __ddiv_rn(r.hi, b.hi);
  r = dd_add(r, dd_mul({-q2, 0.}, b));
  const double q3 = __ddiv_rn(r.hi, b.hi);
  return dd_add(dd_fast_two_sum(q1, q2), {q3, 0.});
}

// sin and cos of x in [0, 8)
__device__ __noinline__ void cr_sincos(double x, double *sn, double *cs) {
  const double P1 = 0x1.921fb54442d18p+0, P2 = 0x1.1a62633145c07p-54,
               P3 = -0x1.f1976b7ed8fbcp-110;
  const double k = rint(__dmul_rn(x, __drcp_rn(P1)));
  DD r = {__dsub_rn(x, __dmul_rn(k, P1)), 0.};
  r = dd_add(r, dd_two_prod(-k, P2));
  r = dd_add(r, {__dmul_rn(-k, P3), 0.});
  const DD r2 = dd_mul(r, r);
  const DD one = {1., 0.};
  DD ts = one, tc = one;
  for (int n = 14; n >= 1; --n) {
    ts = dd_add(one, dd_div_d(dd_mul(r2, ts), -(double)((2 * n) * (2 * n + 1))));
    tc = dd_add(one, dd_div_d(dd_mul(r2, tc), -(double)((2 * n - 1) * (2 * n))));
  }
  const DD s = dd_mul(r, ts);
  const double sv = __dadd_rn(s.hi, s.lo), cv = __dadd_rn(tc.hi, tc.lo);
  const int q = ((int)k) & 3;
  *sn = (q == 0) ? sv : (q == 1) ? cv : (q == 2) ? -sv : -cv;
  *cs = (q == 0) ? cv : (q == 1) ? -sv : (q == 2) ? -cv : sv;
}

// -ln(u) for u in [0, 1) (+inf at 0)
__device__ __noinline__ double cr_neg_log(double u) {
  if (u == 0.) return __longlong_as_double(0x7ff0000000000000ll);
  int e;
  double m = frexp(u, &e);
  if (m < 0.70710678118654752440) {
    m = __dmul_rn(m, 2.);
    e -= 1;
  }
  const DD one = {1., 0.};
  const DD s = dd_div({__dsub_rn(m, 1.), 0.}, dd_two_sum(m, 1.));
  const DD s2 = dd_mul(s, s);
  DD t = {0., 0.};
  for (int k = 22; k >= 0; --k) t = dd_add(dd_div_d(one, (double)(2 * k + 1)), dd_mul(s2, t));
  const DD lm = dd_mul(dd_mul({2., 0.}, s), t);
  const double L2H = 0x1.62e42fefa39efp-1, L2L = 0x1.abc9e3b39803fp-56;
  const DD el = dd_add(dd_two_prod(L2H, (double)e), {__dmul_rn(L2L, (double)e), 0.});
  const DD l = dd_add(el, lm);
  return -__dadd_rn(l.hi, l.lo);
}

}  // namespace cmi
