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
"""
from __future__ import annotations

import numpy as np


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
