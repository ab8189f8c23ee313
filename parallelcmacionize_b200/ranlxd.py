"""ranlxd uniform doubles on the host: the stream of the reference's
RandomGenerator (RandomGenerator.hpp:36-232), which restates Luescher's ranlxd
(as in GSL) with luxury p = 397.

The state is 12 doubles holding 48-bit fractions and a borrow; every step is
one subtract-with-borrow (x[i] = x[j] - x[i] - carry, plus 1 on underflow),
exact in IEEE double, so Python floats give the reference's values bit for
bit.  Used for the set-up draws of the reference driver (random density
modes, random source positions), a few dozen numbers per run; the device
kernels use the same algorithm from include/cmacionize/ranlxd.h.
"""
from __future__ import annotations

_ONE_BIT = 2.0 ** -48


class Ranlxd:
    """RandomGenerator(seed).get_uniform_random_double() as ``uniform()``."""

    def __init__(self, seed: int):
        # RandomGenerator.hpp:158-197: a 31-bit shift register seeded with
        # the bits of the seed fills the 12 state words, 48 bits each
        s = int(seed)
        if s == 0:
            s = 1
        v = s & 0x7FFFFFFF
        bits = []
        for _ in range(31):
            bits.append(v % 2)
            v //= 2
        ib, jb = 0, 18
        self.x = [0.0] * 12
        for k in range(12):
            acc = 0.0
            for _ in range(48):
                y = float((bits[ib] + 1) % 2)
                acc += acc + y
                bits[ib] = (bits[ib] + bits[jb]) % 2
                ib = (ib + 1) % 31
                jb = (jb + 1) % 31
            self.x[k] = _ONE_BIT * acc
        self.carry = 0.0
        self.ir, self.jr, self.ir_old, self.pr = 11, 7, 0, 397

    def _step(self, i: int, j: int) -> None:
        y = self.x[j] - self.x[i]
        y = y - self.carry
        if y < 0:
            self.carry = _ONE_BIT
            y += 1
        else:
            self.carry = 0.0
        self.x[i] = y

    def _increment(self) -> None:
        # RandomGenerator.hpp:80-150: single steps until the lag index wraps,
        # blocks of 12 with partner (q + 7) mod 12, then the remaining steps
        i, j, k = self.ir, self.jr, 0
        while i > 0:
            self._step(i, j)
            i, j, k = (i + 1) % 12, (j + 1) % 12, k + 1
        while k <= self.pr - 12:
            for q in range(12):
                self._step(q, (q + 7) % 12)
            k += 12
        while k < self.pr:
            self._step(i, j)
            i, j, k = (i + 1) % 12, (j + 1) % 12, k + 1
        self.ir = self.ir_old = i
        self.jr = j

    def uniform(self) -> float:
        # RandomGenerator.hpp:214-222
        self.ir = (self.ir + 1) % 12
        if self.ir == self.ir_old:
            self._increment()
        return self.x[self.ir]
