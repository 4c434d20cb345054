"""Error reports of a computed map against an FP64 reference.

KTT validates the Coulomb path with an absolute side-by-side threshold
(``Source/KernelRunner/ResultValidator.inl:73-90``, threshold 0.01 in
``Examples/CoulombSum3d/CoulombSum3d.cpp:226``) or a relative comparison
gated by an absolute floor of 1e-4 (``ResultValidator.inl:92-108``).  Every
result here reports, against FP64 values V* of the same points:

* ``max_abs``      max |V - V*|
* ``rel_norm``     max |V - V*| / max |V*|           (normwise; the headline tolerance 1e-5)
* ``rel_point``    max |V - V*| / max(|V*|, floor)   (pointwise with an absolute floor, stated)
* ``rel_cond``     max |V - V*| / sum_j |q_j| / r_ij (error relative to the condition of the sum,
                                                     when the caller supplies the sum of magnitudes)

The tolerance of the path is 1e-5 relative (TOLERANCE).  A pointwise relative error needs a floor
where V* crosses zero; two floors are stated, in units of rms(V*) of the checked points:

* GATE_FLOOR_RMS = 1: the gate of the FP32-pair forms.  An FP32 evaluation of one term q / r carries
  a relative rounding of about 1e-7 (r^2, the reciprocal square root, the product), so even with
  exact accumulation a point's error is about 1e-7 * sqrt(sum_j (q_j / r_ij)^2), 2e-7 .. 9e-6 on the
  benchmark maps, whatever |V*| is there: measured, the compensated forms need a floor of
  0.07 .. 0.63 rms(V*) to stay within 1e-5 everywhere.
* STRICT_FLOOR_RMS = 1e-3: met by the FP64-pair form, whose error is the FP32 rounding of the stored
  value (6e-8 relative at every point).

``gate`` reports both beside the normwise error and says which the values pass.
"""
from __future__ import annotations

import numpy as np

TOLERANCE = 1e-5
GATE_FLOOR_RMS = 1.0
STRICT_FLOOR_RMS = 1e-3


def report(values, reference, sumabs=None, floor: float | None = None) -> dict:
    v = np.asarray(values, dtype=np.float64).reshape(-1)
    r = np.asarray(reference, dtype=np.float64).reshape(-1)
    if v.shape != r.shape:
        raise ValueError(f"shape mismatch {v.shape} vs {r.shape}")
    if v.size == 0:
        return {"max_abs": 0.0, "rel_norm": 0.0, "rel_point": 0.0, "floor": 0.0, "points": 0}
    d = np.abs(v - r)
    finite = bool(np.all(np.isfinite(v)))
    scale = float(np.max(np.abs(r)))
    if floor is None:
        floor = 1e-3 * float(np.sqrt(np.mean(r * r)))
    out = {
        "max_abs": float(d.max()) if finite else float("inf"),
        "rel_norm": float(d.max() / scale) if (finite and scale > 0) else float("inf"),
        "rel_point": float(np.max(d / np.maximum(np.abs(r), floor))) if finite else float("inf"),
        "floor": float(floor),
        "points": int(v.size),
    }
    if sumabs is not None:
        s = np.asarray(sumabs, dtype=np.float64).reshape(-1)
        out["rel_cond"] = float(np.max(d / np.maximum(s, 1e-300))) if finite else float("inf")
    return out


def gate(values, reference, sumabs=None) -> dict:
    """report() at the gate floor (GATE_FLOOR_RMS * rms of the reference), plus the pointwise error at
    the strict floor and whether the values pass TOLERANCE normwise, pointwise at the gate floor and
    pointwise at the strict floor."""
    r = np.asarray(reference, dtype=np.float64).reshape(-1)
    rms = float(np.sqrt(np.mean(r * r))) if r.size else 0.0
    out = report(values, reference, sumabs=sumabs, floor=GATE_FLOOR_RMS * rms)
    strict = report(values, reference, floor=STRICT_FLOOR_RMS * rms)
    out["floor_rms"] = GATE_FLOOR_RMS
    out["rel_point_strict"] = strict["rel_point"]
    out["strict_floor"] = strict["floor"]
    out["passes_norm"] = bool(out["rel_norm"] <= TOLERANCE)
    out["passes_point"] = bool(out["rel_point"] <= TOLERANCE)
    out["passes_point_strict"] = bool(strict["rel_point"] <= TOLERANCE)
    return out
