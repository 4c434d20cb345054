"""Derivation and exhaustive check of the FMA-pipe reciprocal square root used by the kernels.

The device routine (``rsqrt_fma_x2`` in ``csrc/coul_device.cuh``) computes, lane by lane,

    y0 = bits_to_float(M - (float_to_bits(x) >> 1))
    y1 = y0 * fma(x, y0 * y0, -A1)          (= -y0 (A1 - x y0^2))
    y2 = y1 * fma(x, y1 * y1, -A2)          (= +|y1| (A2 - x y1^2): the two sign flips cancel)
    result: y2 ~= 1 / (S sqrt(x))

The first line is the integer "magic constant" estimate (Blinn 1997; Lomont, "Fast Inverse
Square-Root", 2003).  The steps have the Newton-Raphson form y (a - x y^2); the textbook iteration
is the special case y (3/2 - (x/2) y^2) with Lomont's constant 0x5f375a86.  Writing each step with
-a keeps the argument positive, so it is exactly the r^2 the MUFU path forms anyway, and no negated
or halved operand has to be prepared per pair.

Constants: following the analytic-constant approach of Moroz, Walczyk et al. ("Fast calculation of
inverse square root with the use of magic constant -- analytical approach", 2018), M and A1 are
chosen together to minimise the relative spread of y1 sqrt(x) about its mean lambda (``search``,
+-6.5e-4 against [-1.75e-3, 0] for the textbook first step); A2 = 3 lambda^2 centres the second
step on that scale (the maximum of g (A2 - g^2) sits at g = sqrt(A2 / 3)), and S, folded into the
charge by the kernels at no per-pair cost, removes the final scale and centres the residual
one-signed error.  Instruction count: 2 integer + 6 FP32, as for the textbook iteration.

Because the estimate depends only on the exponent parity and the mantissa, the relative error is
periodic over factors of 4: every FP32 value in [1, 4) covers all normal inputs.  ``error_profile``
emulates the FP32 operation sequence exactly (products of two FP32 values are exact in FP64; the
fused multiply-add is formed in FP64 and rounded once to FP32, which differs from a true FP32 fma
only on FP64 double-rounding ties).

    python -m ktt_b200.soft_rsqrt            # exhaustive bound of the shipped constants
    python -m ktt_b200.soft_rsqrt --search   # re-derive the constants (about a minute)
"""
from __future__ import annotations

import sys

import numpy as np

MAGIC = 0x5F1ED000
A1 = np.float32(2.3597500324)
A2 = np.float32(5.8324427605)
SCALE = np.float32(0.1844490021)

LOMONT = 0x5F375A86


def _binade_pair(step: int = 1) -> np.ndarray:
    lo = np.float32(1.0).view(np.uint32)
    hi = np.float32(4.0).view(np.uint32)
    return np.arange(lo, hi, step, dtype=np.uint32).view(np.float32)


def _magic(x: np.ndarray, m: int) -> np.ndarray:
    return (np.uint32(m) - (x.view(np.uint32) >> np.uint32(1))).astype(np.uint32).view(np.float32)


def _step(y: np.ndarray, arg64: np.ndarray, a) -> np.ndarray:
    t = (y * y).astype(np.float32)
    t = (arg64 * t.astype(np.float64) - float(a)).astype(np.float32)   # fma(arg, t, -a)
    return (y * t).astype(np.float32)


def rsqrt_fma(x, magic: int = MAGIC, a1=A1, a2=A2) -> np.ndarray:
    """FP32 emulation of the device routine for float32 x (unscaled result)."""
    x = np.asarray(x, dtype=np.float32)
    x64 = x.astype(np.float64)
    return _step(_step(_magic(x, magic), x64, a1), x64, a2)


def rsqrt_textbook(x) -> np.ndarray:
    """The textbook iteration, for comparison: Lomont's constant, two steps y (3/2 - (x/2) y^2)."""
    x = np.asarray(x, dtype=np.float32)
    h64 = (x * np.float32(0.5)).astype(np.float32).astype(np.float64)
    return _step(_step(_magic(x, LOMONT), h64, 1.5), h64, 1.5)


def error_profile(magic: int = MAGIC, a1=None, a2=None, scale=None, step: int = 1) -> tuple[float, float]:
    """(min, max) relative error of scale * rsqrt_fma(x) against 1/sqrt(x) over x in [1, 4)."""
    a1 = A1 if a1 is None else a1
    a2 = A2 if a2 is None else a2
    scale = SCALE if scale is None else scale
    x = _binade_pair(step)
    y = rsqrt_fma(x, magic, a1, a2).astype(np.float64) * float(scale)
    e = y * np.sqrt(x.astype(np.float64)) - 1.0
    return float(e.min()), float(e.max())


def _first_step_spread(magic: int, a1s: np.ndarray, x: np.ndarray) -> np.ndarray:
    g = _magic(x, magic).astype(np.float64) * np.sqrt(x.astype(np.float64))
    out = np.empty(a1s.size)
    for i, a1 in enumerate(a1s):
        r = g * (a1 - g * g)
        out[i] = (r.max() - r.min()) / (r.max() + r.min()) * 2.0 if r.min() > 0.3 else 9.0
    return out


def finish(m: int, a1) -> tuple[float, float]:
    """A2 and S for a given (M, A1)."""
    x = _binade_pair(53)
    y0 = _magic(x, m).astype(np.float64)
    r = y0 * (float(a1) - x.astype(np.float64) * y0 * y0) * np.sqrt(x.astype(np.float64))
    lam = 0.5 * (r.max() + r.min())
    a2 = np.float32(3.0 * lam * lam)
    xa = _binade_pair(1)
    full = rsqrt_fma(xa, m, a1, a2).astype(np.float64) * np.sqrt(xa.astype(np.float64))
    scale = np.float32(2.0 / (full.max() + full.min()))
    return float(a2), float(scale)


def search() -> tuple[int, float, float, float]:
    """Grid search of (M, A1) minimising the first step's spread, then A2 and S."""
    x = _binade_pair(211)
    best = (9.0, 0, 0.0)
    a1s = np.linspace(0.6, 3.2, 521)
    for m in range(0x5E000000, 0x5F800000, 1 << 17):
        s = _first_step_spread(m, a1s, x)
        i = int(np.argmin(s))
        if s[i] < best[0]:
            best = (s[i], m, a1s[i])
    _, m0, a0 = best
    a1s = np.linspace(a0 - 0.02, a0 + 0.02, 161).astype(np.float32).astype(np.float64)
    for m in range(m0 - (1 << 17), m0 + (1 << 17), 1 << 10):
        s = _first_step_spread(m, a1s, x)
        i = int(np.argmin(s))
        if s[i] < best[0]:
            best = (s[i], m, a1s[i])
    _, m, a1 = best
    return (m, float(np.float32(a1))) + finish(m, np.float32(a1))


def main() -> None:
    if "--search" in sys.argv:
        m, a1, a2, s = search()
        print(f"M = {m:#x}  A1 = {a1!r}  A2 = {a2!r}  S = {s!r}")
        print("bound:", error_profile(m, np.float32(a1), np.float32(a2), np.float32(s)))
    x = _binade_pair(1)
    e = rsqrt_textbook(x).astype(np.float64) * np.sqrt(x.astype(np.float64)) - 1.0
    print(f"textbook iteration (Lomont constant, a = 3/2): relative error in [{e.min():.3e}, {e.max():.3e}]")
    lo, hi = error_profile()
    print(f"shipped constants M={MAGIC:#x} A1={float(A1)!r} A2={float(A2)!r} S={float(SCALE)!r}: "
          f"relative error in [{lo:.3e}, {hi:.3e}]")


if __name__ == "__main__":
    main()
