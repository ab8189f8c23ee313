/*
 * ranlxd generator (reference: RandomGenerator.hpp:36-232, itself a
 * restatement of GSL's ranlxd with luxury 397).  The sequence must match the
 * reference bit for bit, so the steps are the published algorithm's:
 * subtract-with-borrow on 12 doubles of 48 bits, leading single steps until
 * the lag index wraps, 12-step blocks with partner slot (i + 7) mod 12, then
 * trailing single steps.  Host and device (CUDA) code share this header.
 */
#ifndef CMACIONIZE_RANLXD_H
#define CMACIONIZE_RANLXD_H

#include <cstdint>

#ifdef __CUDACC__
#define CMI_HD __host__ __device__
#else
#define CMI_HD
#endif

namespace cmi_ranlxd {

struct Ranlxd {
  double x[12];
  double carry;
  uint32_t ir, jr, ir_old, pr;

  static constexpr double kOneBit = 1.0 / 281474976710656.0;  // 2^-48

  CMI_HD void step(uint32_t i, uint32_t j) {
    double y = x[j] - x[i];
    y = y - carry;
    if (y < 0) {
      carry = kOneBit;
      y += 1;
    } else {
      carry = 0;
    }
    x[i] = y;
  }

  // RandomGenerator.hpp:80-150
  CMI_HD void increment() {
    uint32_t i = ir, j = jr;
    int32_t k = 0;
    for (; i > 0; ++k) {
      step(i, j);
      i = (i + 1) % 12;
      j = (j + 1) % 12;
    }
    for (; k <= (int32_t)pr - 12; k += 12) {
      for (uint32_t q = 0; q < 12; ++q) step(q, (q + 7) % 12);
    }
    for (; k < (int32_t)pr; ++k) {
      step(i, j);
      i = (i + 1) % 12;
      j = (j + 1) % 12;
    }
    ir = i;
    ir_old = i;
    jr = j;
  }

  // RandomGenerator.hpp:158-197
  CMI_HD void seed(int32_t s) {
    if (s == 0) s = 1;
    int32_t bits[31];
    int32_t v = s & 0x7FFFFFFF;
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
      x[k] = kOneBit * acc;
    }
    carry = 0;
    ir = 11;
    jr = 7;
    ir_old = 0;
    pr = 397;
  }

  // RandomGenerator.hpp:214-222
  CMI_HD double uniform() {
    ir = (ir + 1) % 12;
    if (ir == ir_old) increment();
    return x[ir];
  }
};

}  // namespace cmi_ranlxd

#endif
