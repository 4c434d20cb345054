"""Derivation and exhaustive check of the FMA-pipe reciprocal square root used by the kernels.

The device routine (``rsqrt_fma_half`` in ``csrc/coul_device.cuh``) takes hx = x / 2 and computes

    y0 = bits_to_float(M - (float_to_bits(hx) >> 1))
    y1 = y0 * fma(-hx, y0 * y0, A1)
    y2 = y1 * fma(-hx, y1 * y1, A2)          result: y2 ~= 1 / (S * sqrt(x))

The first line is the integer "magic constant" estimate (Blinn 1997; Lomont, "Fast Inverse
Square-Root", 2003), written for the halved argument (bits(x/2) >> 1 == (bits(x) >> 1) - 2^22).
The two steps have the Newton-Raphson form y (a - hx y^2); with a = 3/2 and Lomont's constant they
are the classic iteration.  Following the analytic-constant approach of Moroz, Walczyk et al.
("Fast calculation of inverse square root with the use of magic constant -- analytical approach",
2018), M and A1 are chosen together to minimise the relative spread of y1 * sqrt(x) about its mean
lambda (``search``); A2 = 3/2 * lambda^2 centres the second step on that scale, and S (folded into
the charge by the kernels, at no per-pair cost) removes the final scale and centres the residual
one-signed error.  Same instruction count as the classic iteration: 2 integer + 6 FP32.

Because the estimate depends only on the exponent parity and the mantissa, the relative error is
periodic over factors of 4: every FP32 value in [1, 4) covers all normal inputs.  ``error_profile``
emulates the FP32 operation sequence (products of two FP32 values are exact in FP64; the fused
multiply-add is formed in FP64 and rounded once to FP32).

    python -m ktt_b200.soft_rsqrt            # exhaustive bound of the shipped constants
    python -m ktt_b200.soft_rsqrt --search   # re-derive the constants (about a minute)
"""
from __future__ import annotations

import sys

import numpy as np

MAGIC = 0x5F1EEC00
A1 = np.float32(2.3625)
A2 = np.float32(5.8528552055)
SCALE = np.float32(0.1297434270)

# the classic iteration, for comparison
CLASSIC = (0x5F375A86 - (1 << 22), np.float32(1.5), np.float32(1.5))


def _binade_pair(step: int = 1) -> np.ndarray:
    lo = np.float32(1.0).view(np.uint32)
    hi = np.float32(4.0).view(np.uint32)
    return np.arange(lo, hi, step, dtype=np.uint32).view(np.float32)


def rsqrt_fma_half(hx, magic: int = MAGIC, a1=A1, a2=A2) -> np.ndarray:
    """FP32 emulation of the device routine for float32 hx = x / 2 (unscaled result)."""
    hx = np.asarray(hx, dtype=np.float32)
    y = (np.uint32(magic) - (hx.view(np.uint32) >> np.uint32(1))).astype(np.uint32).view(np.float32)
    h64 = hx.astype(np.float64)
    for a in (a1, a2):
        t = (y * y).astype(np.float32)
        t = (-h64 * t.astype(np.float64) + float(a)).astype(np.float32)
        y = (y * t).astype(np.float32)
    return y


def error_profile(magic: int = MAGIC, a1=A1, a2=A2, scale=SCALE, step: int = 1) -> tuple[float, float]:
    """(min, max) relative error of scale * rsqrt_fma_half(x/2) against 1/sqrt(x) over x in [1, 4)."""
    x = _binade_pair(step)
    hx = (x * np.float32(0.5)).astype(np.float32)
    y = rsqrt_fma_half(hx, magic, a1, a2).astype(np.float64) * float(scale)
    e = y * np.sqrt(x.astype(np.float64)) - 1.0
    return float(e.min()), float(e.max())


def _first_step_spread(magic: int, a1s: np.ndarray, x: np.ndarray) -> np.ndarray:
    hxf = (x * np.float32(0.5)).astype(np.float32)
    y0 = (np.uint32(magic) - (hxf.view(np.uint32) >> np.uint32(1))).astype(np.uint32).view(np.float32)
    g = y0.astype(np.float64) * np.sqrt(x.astype(np.float64))
    out = np.empty(a1s.size)
    for i, a1 in enumerate(a1s):
        r = g * (a1 - 0.5 * g * g)
        out[i] = (r.max() - r.min()) / (r.max() + r.min()) * 2.0 if r.min() > 0.3 else 9.0
    return out


def search() -> tuple[int, float, float, float]:
    """Grid search of (M, A1) minimising the first step's spread, then A2 and S."""
    x = _binade_pair(211)
    best = (9.0, 0, 0.0)
    a1s = np.linspace(1.2, 3.2, 401)
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
    a1 = np.float32(a1)
    hxf = (x * np.float32(0.5)).astype(np.float32)
    y0 = (np.uint32(m) - (hxf.view(np.uint32) >> np.uint32(1))).astype(np.uint32).view(np.float32).astype(np.float64)
    r = y0 * (float(a1) - hxf.astype(np.float64) * y0 * y0) * np.sqrt(x.astype(np.float64))
    lam = 0.5 * (r.max() + r.min())
    a2 = np.float32(1.5 * lam * lam)
    xa = _binade_pair(1)
    hxa = (xa * np.float32(0.5)).astype(np.float32)
    full = rsqrt_fma_half(hxa, m, a1, a2).astype(np.float64) * np.sqrt(xa.astype(np.float64))
    scale = np.float32(2.0 / (full.max() + full.min()))
    return m, float(a1), float(a2), float(scale)


def main() -> None:
    if "--search" in sys.argv:
        m, a1, a2, s = search()
        print(f"M = {m:#x}  A1 = {a1!r}  A2 = {a2!r}  S = {s!r}")
        print("bound:", error_profile(m, np.float32(a1), np.float32(a2), np.float32(s)))
    cm, c1, c2 = CLASSIC
    emin, emax = error_profile(cm, c1, c2, np.float32(1.0))
    print(f"classic iteration (Lomont constant, a = 3/2): relative error in [{emin:.3e}, {emax:.3e}]")
    lo, hi = error_profile()
    print(f"shipped constants M={MAGIC:#x} A1={float(A1)} A2={float(A2)} S={float(SCALE)}: "
          f"relative error in [{lo:.3e}, {hi:.3e}]")


if __name__ == "__main__":
    main()
