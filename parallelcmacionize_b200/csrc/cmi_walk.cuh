// Cell walk of one packet through one subgrid: DensitySubGrid::interact
// (DensitySubGrid.hpp:1180-1323) split into entry + one-crossing steps, so a
// warp can advance 32 packets one crossing at a time.
//
// Three precisions:
//  * Walk64 -- the reference's FP64 arithmetic, operation for operation.  The
//    translation unit is compiled with --fmad=false, so no multiply-add is
//    contracted and every result rounds exactly as on the host.
//  * WalkM -- mixed: Walk64's geometry (positions, face distances, path
//    lengths) operation for operation, the cell opacity sigma n x, optical
//    depths and tallies in FP32.  Cell sequences and path lengths equal the
//    reference's; only the absorbing cell's length carries FP32 error.
//  * Walk32 -- FP32 in cell units: the position is kept relative to the
//    subgrid in units of cells, so cell faces are exact small integers; path
//    lengths stay in metres, l = (face - p) * (cell_size / d).
// Walk32 and WalkM path lengths go to shared-memory tallies (Tally32) merged
// into FP64 J.
#pragma once

#include "cmi_device.cuh"

namespace cmi {

enum WalkStatus : int { kRun = 0, kAbsorbed = 1, kExited = 2 };

// What a FP64 walk does in each cell (the dust path, testDensitySubGrid_omp_dust.cpp):
//  kInteract  DensitySubGrid::interact: path length into J, stop at the target depth
//  kPropagate DensitySubGrid::propagate (DensitySubGrid.hpp:1333-1472): the same walk
//             without the J tally
//  kDepth     DensitySubGrid::compute_optical_depth (DensitySubGrid.hpp:1482-1604): no
//             target, the optical depth of the whole crossing is added to the packet
enum WalkMode : int { kInteract = 0, kPropagate = 1, kDepth = 2 };

template <class T>
__device__ __forceinline__ T min_ref(T a, T b) {  // std::min semantics
  return (b < a) ? b : a;
}

// View of the staged subgrid in shared memory (FP32 mode).
struct View32 {
  const float *kappa;  // sigma * n * x per cell (1/m)
  int n[3];
  int nyz;
  float cs[3];         // cell size (m)
  float inv_cs[3];     // 1 / cell size, rounded from FP64
};

// Shared-memory path-length tallies of one staged subgrid.
//  kTally 0: FP32 atomics
//  kTally 1: FP32 atomics with the rounding error of each addition (TwoSum of
//            the atomic's own old value) accumulated in a second FP32 array
//  kTally 2: fixed point (units of lref / 2^22) in one 32-bit word per cell by
//            integer atomic add; a wrap of the word (rare: 1024 cell lengths)
//            adds its 2^32 units straight to the FP64 J array in HBM
//  kTally 3: 64-bit fixed point with 64-bit integer atomics
// The fixed-point forms round len * 2^22 / lref (< 2^23 since len <= sqrt(3)
// lref) half-to-even through the float adder: adding 2^23 leaves the
// rounded integer in the mantissa bits, so no conversion instruction is used.
template <int kTally>
struct Tally32 {
  float *f_hi, *f_lo;
  uint32_t *u_lo, *u_hi;
  unsigned long long *u64;
  double *carry_J;      // kTally 2: J of the staged subgrid (HBM)
  double carry_value;   // kTally 2: 2^32 units in J units
  float scale;  // 2^22 / lref

  static __device__ __forceinline__ uint32_t fixed(float len, float scale) {
    const float q = fmaxf(__fmul_rn(len, scale), 0.f);
    return __float_as_uint(__fadd_rn(q, 8388608.f)) - 0x4B000000u;
  }

  __device__ __forceinline__ void add(int cell, float len) const {
    if (kTally == 0) {
      atomicAdd(&f_hi[cell], len);
    } else if (kTally == 1) {
      const float old = atomicAdd(&f_hi[cell], len);
      const float nw = __fadd_rn(old, len);
      const float bv = __fsub_rn(nw, old);
      const float err = __fadd_rn(__fsub_rn(old, __fsub_rn(nw, bv)), __fsub_rn(len, bv));
      if (err != 0.f) atomicAdd(&f_lo[cell], err);
    } else if (kTally == 2) {
      const uint32_t v = fixed(len, scale);
      const uint32_t old = atomicAdd(&u_lo[cell], v);
      if (old + v < old) atomicAdd(&carry_J[cell], carry_value);
    } else {
      atomicAdd(&u64[cell], (unsigned long long)fixed(len, scale));
    }
  }

  // Sum of cell c in units of metres (lref / 2^22 for the fixed-point forms);
  // resets the cell.
  __device__ __forceinline__ double take(int c, double unit) const {
    double v;
    if (kTally == 0) {
      v = (double)f_hi[c];
      f_hi[c] = 0.f;
    } else if (kTally == 1) {
      v = (double)f_hi[c] + (double)f_lo[c];
      f_hi[c] = 0.f;
      f_lo[c] = 0.f;
    } else if (kTally == 2) {
      v = (double)u_lo[c] * unit;
      u_lo[c] = 0u;
    } else {
      v = (double)u64[c] * unit;
      u64[c] = 0ull;
    }
    return v;
  }

  __device__ __forceinline__ void zero(int c) const {
    if (kTally == 0) f_hi[c] = 0.f;
    else if (kTally == 1) { f_hi[c] = 0.f; f_lo[c] = 0.f; }
    else if (kTally == 2) u_lo[c] = 0u;
    else u64[c] = 0ull;
  }
};

// View of the staged subgrid in shared memory (FP64 mode).
struct View64 {
  const double *nH;
  const double *xH;
  double *J;
  int n[3];
  int nyz;
  double anchor[3];
  double cs[3];
  double inv_cs[3];
};

// ----------------------------------------------------------------------------
// FP32 cell-unit walk
// ----------------------------------------------------------------------------
struct Walk32 {
  // Per axis the packet looks only at the cell face ahead of it (direction
  // of travel): face = idx + 1 for d > 0, idx for d < 0, +inf for d == 0.
  // The path length to it is l = (face - p) * inv with inv = cs / d, the same
  // operands and roundings as (hi - p) * inv / (lo - p) * inv of the
  // reference loop, so the walk is unchanged; the per-axis branches, the
  // integer index and the cell-index recomputation of each step are gone.
  float p[3], d[3], face[3], inv[3], dcs[3];
  float fstep[3];  // +1 / -1: the face after the next one
  float fexit[3];  // the face whose crossing leaves the subgrid (n or 0)
  int cstep[3];    // cell-index change when the face is crossed
  float tau_done, tau_target;
  int cell;
  int steps;
  int exited;      // exit: bit a set when axis a left the subgrid

  // Entry: DensitySubGrid.hpp:1186-1219 (start index per get_start_index).
  // inv = cell_size * (1/d) and dcs = d * (1/cell_size): correctly rounded
  // reciprocals and products, no divisions.
  __device__ __forceinline__ int begin(const Packet32 &pk, const View32 &v,
                                      const uint8_t *sign_code) {
    const uint8_t code = sign_code[pk.meta & 31u];
    const int stride[3] = {v.nyz, v.n[2], 1};
    int idx[3];
    bool inside = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      p[a] = pk.pos[a];
      d[a] = pk.dir[a];
      dcs[a] = __fmul_rn(d[a], v.inv_cs[a]);
      const int s = sign_of(code, a);
      idx[a] = (s == 0) ? __float2int_rz(p[a]) : ((s < 0) ? 0 : v.n[a] - 1);
      inside = inside && idx[a] >= 0 && idx[a] < v.n[a];
      const bool up = d[a] > 0.f;
      const bool moving = up || d[a] < 0.f;
      inv[a] = moving ? __fmul_rn(v.cs[a], __frcp_rn(d[a])) : __int_as_float(0x7f800000);
      face[a] = moving ? (float)(up ? idx[a] + 1 : idx[a]) : __int_as_float(0x7f800000);
      fstep[a] = up ? 1.f : -1.f;
      fexit[a] = up ? (float)v.n[a] : 0.f;
      cstep[a] = up ? stride[a] : -stride[a];
    }
    cell = idx[0] * stride[0] + idx[1] * stride[1] + idx[2];
    tau_done = 0.f;
    tau_target = pk.tau;
    steps = 0;
    exited = 0;
    if (!(tau_done < tau_target)) return kAbsorbed;
    if (!inside) {
      // entered outside the index range (position on or beyond a face)
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        if (idx[a] < 0 || idx[a] >= v.n[a]) {
          exited |= 1 << a;
          // the side it left through, for exit_mask
          fstep[a] = idx[a] < 0 ? -1.f : 1.f;
        }
      }
      return kExited;
    }
    return kRun;
  }

  // One iteration of the loop at DensitySubGrid.hpp:1221-1305; the path
  // length lmin of the crossed cell `tally_cell` is returned for the tally.
  __device__ __forceinline__ int step(const View32 &v, int &tally_cell, float &lmin_out) {
    float l[3];
    const float k = v.kappa[cell];
#pragma unroll
    for (int a = 0; a < 3; ++a) l[a] = __fmul_rn(__fsub_rn(face[a], p[a]), inv[a]);
    float lmin = min_ref(l[0], min_ref(l[1], l[2]));
    const float tau = __fmul_rn(lmin, k);
    tau_done = __fadd_rn(tau_done, tau);
    tally_cell = cell;
    ++steps;
    if (tau_done >= tau_target) {
      const float corr = __fdiv_rn(__fsub_rn(tau_done, tau_target), tau);
      lmin = __fmul_rn(lmin, __fsub_rn(1.f, corr));
      lmin_out = lmin;
#pragma unroll
      for (int a = 0; a < 3; ++a)
        p[a] = (l[a] == lmin) ? face[a] : __fmaf_rn(lmin, dcs[a], p[a]);
      return kAbsorbed;
    }
    lmin_out = lmin;
    int out = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const bool cross = l[a] == lmin;
      p[a] = cross ? face[a] : __fmaf_rn(lmin, dcs[a], p[a]);
      if (cross) {
        out |= (face[a] == fexit[a]) ? (1 << a) : 0;
        face[a] = __fadd_rn(face[a], fstep[a]);
        cell += cstep[a];
      }
    }
    if (out) {
      exited = out;
      return kExited;
    }
    return kRun;
  }

  // Exit: 6-bit mask (DensitySubGrid.hpp:483-506).  With reanchor the
  // position moves into the neighbour's cell frame (exact: the exit
  // coordinate is 0 or n).
  __device__ __forceinline__ int exit_mask(const View32 &v, bool reanchor = true) {
    int mask = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (!((exited >> a) & 1)) continue;
      const bool high = fstep[a] > 0.f;
      mask |= high ? (1 << (5 - 2 * a)) : (1 << (4 - 2 * a));
      if (reanchor) {
        p[a] = high ? __fsub_rn(p[a], __int2float_rn(v.n[a]))
                    : __fadd_rn(p[a], __int2float_rn(v.n[a]));
      }
    }
    return mask;
  }

  __device__ __forceinline__ Packet32 packet(uint32_t meta) const {
    Packet32 pk;
    pk.pos[0] = p[0];
    pk.pos[1] = p[1];
    pk.pos[2] = p[2];
    pk.dir[0] = d[0];
    pk.dir[1] = d[1];
    pk.dir[2] = d[2];
    pk.tau = __fsub_rn(tau_target, tau_done);
    pk.meta = meta;
    return pk;
  }
  __device__ __forceinline__ Packet32 packet(const View32 &, uint32_t meta) const {
    return packet(meta);
  }

  // Reemission counter of an absorbed packet in subgrid `sub`: the cell-unit
  // position bits mixed with the subgrid index.
  __device__ __forceinline__ void reemit_counter(const View32 &, uint32_t sub,
                                                 uint32_t h[3]) const {
    h[0] = __float_as_uint(p[0]) ^ sub;
    h[1] = __float_as_uint(p[1]) ^ (sub * 0x9E3779B9u);
    h[2] = __float_as_uint(p[2]);
  }
  // The re-emitted packet: same position, drawn direction rd[0..2] and
  // optical depth rd[3].
  __device__ __forceinline__ Packet32 reemitted(const View32 &, const double rd[4]) const {
    Packet32 rp;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      rp.pos[a] = p[a];
      rp.dir[a] = (float)rd[a];
    }
    rp.tau = (float)rd[3];
    rp.meta = (uint32_t)kInside;
    return rp;
  }
};

// ----------------------------------------------------------------------------
// Mixed-precision walk: the reference's FP64 geometry, FP32 optical depths
// ----------------------------------------------------------------------------
// View of the staged subgrid: FP32 opacity kappa = sigma n x per cell, the
// subgrid's FP64 anchor, cell size and inverse cell size (shared memory, read
// where they are needed instead of being held in registers), and its cell
// faces: faces[face_off[a] + i] = i * cs[a], i = 0..n[a], the reference's
// idx * cs and (idx + 1.) * cs, computed once per subgrid.
struct ViewM {
  const float *kappa;
  const double *anchor, *cs, *inv_cs;
  const double *faces;
  int face_off[3];
  int n[3];
  int nyz;
};

// Fill the face table of a subgrid (threads t = 0, stride of the CTA).
__device__ __forceinline__ void fill_faces(double *faces, const int n[3], const double cs[3],
                                           int t, int stride) {
  const int o1 = n[0] + 1, o2 = o1 + n[1] + 1, total = o2 + n[2] + 1;
  for (int i = t; i < total; i += stride) {
    const int a = (i < o1) ? 0 : ((i < o2) ? 1 : 2);
    const int k = i - ((a == 0) ? 0 : ((a == 1) ? o1 : o2));
    faces[i] = __dmul_rn((double)k, cs[a]);
  }
}

// The geometry of interact (DensitySubGrid.hpp:1186-1305) in FP64, operation
// for operation: position relative to the anchor, face ahead (idx + 1) * cs
// or idx * cs, l = (face - pos) * (1 / d), crossed coordinates snapped to
// their face, pos + lmin * d for the others.  Every cell crossed and every
// path length up to the last one therefore equal the reference's bit for
// bit.  The optical depth of a crossing is (float)lmin * kappa, accumulated
// in FP32; in the absorbing cell the FP32 fraction (tau_target - tau_before) /
// tau (at most 1; tau_before the depth before the cell) scales the FP64
// length.  Path lengths reach the tallies as FP32.
struct WalkM {
  double pos[3], d[3];
  double inv[3];   // 1 / d, correctly rounded; +inf when d == 0
  double face[3];  // the face ahead; +inf when d == 0 (l = +inf)
  int idx[3];
  float tau_done, tau_target;
  int cell;
  int steps;

  // Entry: DensitySubGrid.hpp:1186-1219 and get_start_index (:428-469).
  __device__ __forceinline__ int begin(const PacketM &pk, const ViewM &v,
                                      const uint8_t *sign_code) {
    const uint8_t code = sign_code[pk.meta & 31u];
    bool inside = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      d[a] = pk.dir[a];
      pos[a] = __dsub_rn(pk.pos[a], v.anchor[a]);
      const int s = sign_of(code, a);
      idx[a] = (s == 0) ? __double2int_rz(__dmul_rn(pos[a], v.inv_cs[a]))
                        : ((s < 0) ? 0 : v.n[a] - 1);
      inside = inside && idx[a] >= 0 && idx[a] < v.n[a];
      const bool moving = d[a] > 0. || d[a] < 0.;
      inv[a] = moving ? __drcp_rn(d[a]) : __longlong_as_double(0x7ff0000000000000ll);
    }
    cell = idx[0] * v.nyz + idx[1] * v.n[2] + idx[2];
    tau_done = 0.f;
    tau_target = pk.tau;
    steps = 0;
    if (!(tau_done < tau_target)) return kAbsorbed;
    if (!inside) return kExited;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const bool up = d[a] > 0.;
      face[a] = (up || d[a] < 0.) ? v.faces[v.face_off[a] + idx[a] + (up ? 1 : 0)]
                                  : __longlong_as_double(0x7ff0000000000000ll);
    }
    return kRun;
  }

  // One iteration of the loop at DensitySubGrid.hpp:1221-1305; the FP32
  // path length of the crossed cell `tally_cell` is returned for the tally.
  __device__ __forceinline__ int step(const ViewM &v, int &tally_cell, float &lmin_out) {
    return step_k(v, v.kappa[cell], tally_cell, lmin_out, nullptr);
  }

  // The same with the cell's opacity k given; trace (may be null) receives
  // the FP64 length.
  __device__ __forceinline__ int step_k(const ViewM &v, float k, int &tally_cell,
                                        float &lmin_out, double *trace) {
    double l[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) l[a] = __dmul_rn(__dsub_rn(face[a], pos[a]), inv[a]);
    double lmin = min_ref(l[0], min_ref(l[1], l[2]));
    const float lf = __double2float_rn(lmin);
    const float tau = __fmul_rn(lf, k);
    const float tau_before = tau_done;
    tau_done = __fadd_rn(tau_done, tau);
    tally_cell = cell;
    ++steps;
    if (tau_done >= tau_target) {
      // the reference's 1 - (tau_done - tau_target) / tau as (tau_target -
      // tau_before) / tau: no cancellation when the packet stops early in the cell
      const float frac = fminf(__fdiv_rn(__fsub_rn(tau_target, tau_before), tau), 1.f);
      lmin = __dmul_rn(lmin, (double)frac);
      lmin_out = __double2float_rn(lmin);
      if (trace) *trace = lmin;
#pragma unroll
      for (int a = 0; a < 3; ++a)
        pos[a] = (l[a] == lmin) ? face[a] : __dadd_rn(pos[a], __dmul_rn(lmin, d[a]));
      return kAbsorbed;
    }
    lmin_out = lf;
    if (trace) *trace = lmin;
    const int stride[3] = {v.nyz, v.n[2], 1};
    int out = 0;
    // branch-free: the lanes of a warp cross different axes, so per-axis
    // branches would diverge; every axis reads its (clamped) next face and
    // keeps it only when it crossed into a cell of the subgrid
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const bool cross = l[a] == lmin;
      pos[a] = cross ? face[a] : __dadd_rn(pos[a], __dmul_rn(lmin, d[a]));
      const bool up = d[a] > 0.;
      const int di = cross ? (up ? 1 : -1) : 0;
      idx[a] += di;
      cell += di * stride[a];
      const bool inside = (unsigned)idx[a] < (unsigned)v.n[a];
      const double next = v.faces[v.face_off[a] + min(max(idx[a], 0), v.n[a] - 1) + (up ? 1 : 0)];
      face[a] = (cross && inside) ? next : face[a];
      out |= (cross && !inside) ? (1 << a) : 0;
    }
    return out ? kExited : kRun;
  }

  // Exit: 6-bit mask from the out-of-range indices (DensitySubGrid.hpp:483-506).
  __device__ __forceinline__ int exit_mask(const ViewM &v) const {
    int mask = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      mask |= ((idx[a] >= v.n[a]) ? (1 << (5 - 2 * a)) : 0) | ((idx[a] < 0) ? (1 << (4 - 2 * a)) : 0);
    }
    return mask;
  }

  // The packet as the reference leaves it (DensitySubGrid.hpp:1307-1309):
  // absolute position, remaining optical depth.
  __device__ __forceinline__ PacketM packet(const ViewM &v, uint32_t meta) const {
    PacketM pk;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      pk.pos[a] = __dadd_rn(pos[a], v.anchor[a]);
      pk.dir[a] = d[a];
    }
    pk.tau = __fsub_rn(tau_target, tau_done);
    pk.meta = meta;
    pk.pad[0] = pk.pad[1] = 0u;
    return pk;
  }

  // Reemission counter: the FP64 one of the reference walk (hash of each
  // absolute coordinate of the absorption point).
  __device__ __forceinline__ void reemit_counter(const ViewM &v, uint32_t,
                                                 uint32_t h[3]) const {
#pragma unroll
    for (int a = 0; a < 3; ++a) h[a] = reemit_hash(__dadd_rn(pos[a], v.anchor[a]));
  }
  __device__ __forceinline__ PacketM reemitted(const ViewM &v, const double rd[4]) const {
    PacketM rp;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      rp.pos[a] = __dadd_rn(pos[a], v.anchor[a]);
      rp.dir[a] = rd[a];
    }
    rp.tau = tau32(rd[3]);
    rp.meta = (uint32_t)kInside;
    rp.pad[0] = rp.pad[1] = 0u;
    return rp;
  }
};

// ----------------------------------------------------------------------------
// FP64 reference walk
// ----------------------------------------------------------------------------
struct Walk64 {
  double pos[3], d[3], inv[3];
  double tau_done, tau_target, sigma, weight;
  double didx[3];  // idx as double (exact): idx * cs and (idx + 1.) * cs without conversions
  int idx[3];
  int cell;
  int steps;
  int type;

  // DensitySubGrid.hpp:1186-1219 and get_start_index (:428-469).
  __device__ __forceinline__ int begin(const Packet64 &pk, const View64 &v,
                                      const uint8_t *sign_code) {
    const uint8_t code = sign_code[pk.meta & 31u];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      d[a] = pk.dir[a];
      inv[a] = 1. / d[a];
      pos[a] = pk.pos[a] - v.anchor[a];
      const int s = sign_of(code, a);
      idx[a] = (s == 0) ? __double2int_rz(pos[a] * v.inv_cs[a]) : ((s < 0) ? 0 : v.n[a] - 1);
      didx[a] = (double)idx[a];
    }
    cell = idx[0] * v.nyz + idx[1] * v.n[2] + idx[2];
    tau_done = 0.;
    tau_target = pk.tau;
    sigma = pk.sigma;
    weight = pk.weight;
    type = pk.type;
    steps = 0;
    if (!(tau_done < tau_target)) return kAbsorbed;
    return inside(v) ? kRun : kExited;
  }

  __device__ __forceinline__ bool inside(const View64 &v) const {
    return idx[0] < v.n[0] && idx[0] >= 0 && idx[1] < v.n[1] && idx[1] >= 0 &&
           idx[2] < v.n[2] && idx[2] >= 0;
  }

  // compute_optical_depth's entry (DensitySubGrid.hpp:1495-1519): no target,
  // so no absorption test; the packet's depth so far is kept in tau_target
  __device__ __forceinline__ int begin_depth(const Packet64 &pk, const View64 &v,
                                            const uint8_t *sign_code) {
    (void)begin(pk, v, sign_code);
    tau_target = pk.tau;
    tau_done = 0.;
    return inside(v) ? kRun : kExited;
  }

  // DensitySubGrid.hpp:1221-1305, one iteration (kMode: what the cell does).
  template <int kMode = kInteract>
  __device__ __forceinline__ int step(const View64 &v, double *trace_len = nullptr) {
    double lo[3], hi[3], l[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      lo[a] = didx[a] * v.cs[a];
      hi[a] = (didx[a] + 1.) * v.cs[a];
      l[a] = (d[a] > 0.)   ? (hi[a] - pos[a]) * inv[a]
             : (d[a] < 0.) ? (lo[a] - pos[a]) * inv[a]
                           : DBL_MAX;
    }
    double lmin = min_ref(l[0], min_ref(l[1], l[2]));
    double lminsigma = lmin * sigma;
    const double tau = lminsigma * v.nH[cell] * v.xH[cell];
    tau_done += tau;
    const bool absorbed = kMode != kDepth && tau_done >= tau_target;
    if (absorbed) {
      const double correction = (tau_done - tau_target) / tau;
      lmin *= (1. - correction);
      lminsigma = lmin * sigma;
    } else {
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        if (l[a] == lmin) {
          idx[a] += (d[a] > 0.) ? 1 : -1;
          didx[a] += (d[a] > 0.) ? 1. : -1.;
        }
      }
    }
    if (trace_len) *trace_len = lmin;
    if (kMode == kInteract) atomicAdd(&v.J[cell], lminsigma * weight);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      pos[a] = (l[a] == lmin) ? ((d[a] > 0.) ? hi[a] : lo[a]) : pos[a] + lmin * d[a];
    }
    ++steps;
    if (absorbed) return kAbsorbed;
    if (!inside(v)) return kExited;
    cell = idx[0] * v.nyz + idx[1] * v.n[2] + idx[2];
    return kRun;
  }

  __device__ __forceinline__ int exit_mask(const View64 &v) const {
    int mask = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const int low = idx[a] < 0;
      const int high = (idx[a] / v.n[a]) > 0;
      mask |= (high << (5 - 2 * a)) | (low << (4 - 2 * a));
    }
    return mask;
  }

  // The photon as the reference leaves it (DensitySubGrid.hpp:1307-1309).
  __device__ __forceinline__ Packet64 packet(const View64 &v, uint32_t meta) const {
    Packet64 pk;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      pk.pos[a] = pos[a] + v.anchor[a];
      pk.dir[a] = d[a];
    }
    pk.tau = tau_target - tau_done;
    pk.sigma = sigma;
    pk.weight = weight;
    pk.type = type;
    pk.meta = meta;
    return pk;
  }
};

// Packet record and subgrid view of each walk that runs in the wavefront.
template <class W> struct WalkTraits;
// kUnroll: crossings of a stretch unrolled in the walk loop (the mixed walk's
// FP64 step is long; on the 128^3 log-normal workload its walk took 3.45 /
// 3.26 / 3.49 ms per iteration unrolled 1 / 4 / 8 times).
template <> struct WalkTraits<Walk32> {
  using Packet = Packet32;
  using View = View32;
  static constexpr int kUnroll = 8;
};
template <> struct WalkTraits<WalkM> {
  using Packet = PacketM;
  using View = ViewM;
  static constexpr int kUnroll = 4;
};

}  // namespace cmi
