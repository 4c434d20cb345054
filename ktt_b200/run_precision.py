"""Precision stress: the precision forms on a cancellation-heavy map (or the uniform map).

    python -m ktt_b200.run_precision [--map clustered|uniform] [--subset 0.01] [--repeat 3]

clustered: 65,536 atoms in 64 Gaussian clusters (sigma 2 A, centres uniform in the 128 A cube),
charges +1/-1 alternating within each cluster plus N(0, 0.01), total charge exactly zero; uniform:
the benchmark's map (65,536 atoms uniform in the 128 A cube, q ~ U[-1, 1]); 256^3 grid at 0.5 A.
Each form (FP32 accumulation, compensated two-sum, FP64 merge -- MUFU-only and with part of the
rsqrts on the FMA pipe, and with the FP64 sums in shared memory -- and FP64 pairs) is timed on the device (best of --repeat) and compared with
the FP64 oracle on a seeded subset of grid points.  Prints one JSON line per form: device time, pair
rate, max abs error, max error / max |V| (rel_norm), rms error / rms V (rel_rms), the pointwise
error max |dV| / max(|V|, floor) at the gate floor rms(V) (rel_point), at 0.1 rms(V) and at the strict
floor 1e-3 rms(V) (rel_point_strict), the smallest floor every point passes at, the pass flags of
ktt_b200.errors.gate, and max error / sum_j |q_j| / r_ij (rel_cond, the error in units of the sum's
condition).
"""
from __future__ import annotations

import argparse
import json

import numpy as np

FORMS = (
    ("fp32", dict(precision=0, rsqrt_soft=0)),
    ("fp32_soft2", dict(precision=0, rsqrt_soft=2)),
    ("compensated", dict(precision=1, rsqrt_soft=0)),
    ("compensated_soft2", dict(precision=1, rsqrt_soft=2)),
    ("fp64_merge", dict(precision=2, rsqrt_soft=0)),
    ("fp64_merge_soft2", dict(precision=2, rsqrt_soft=2)),
    ("fp64_merge_shared_soft2", dict(precision=4, rsqrt_soft=2)),
    ("fp64_pairs", dict(precision=3, rsqrt_soft=0)),
)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--map", choices=["clustered", "uniform"], default="clustered")
    ap.add_argument("--subset", type=float, default=0.01)
    ap.add_argument("--repeat", type=int, default=3)
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--per-cluster", type=int, default=1024)
    ap.add_argument("--z-iterations", type=int, default=8)
    ap.add_argument("--x-points", type=int, default=2)
    args = ap.parse_args()

    import torch

    import ktt_b200
    import oracle
    from ktt_b200 import errors, workloads

    if args.map == "clustered":
        case = workloads.clustered_map(n=args.n, per_cluster=args.per_cluster, box=args.n * 0.5)
    else:
        case = workloads.uniform_map(n=args.n, box=args.n * 0.5)
    dims, h = case.dims, case.spacing
    total = dims[0] * dims[1] * dims[2]
    idx = workloads.subset_indices(total, args.subset)
    ref, sumabs = oracle.points3d(case.atoms, h, dims, idx, want_sumabs=True)
    ctx = ktt_b200.CoulombContext(0)
    atoms = torch.from_numpy(case.atoms).cuda()
    out = torch.empty((dims[2], dims[1], dims[0]), dtype=torch.float32, device="cuda")
    pairs = float(total) * case.atoms.shape[0]
    base = {"dims": list(dims), "atoms": int(case.atoms.shape[0]), "subset_points": int(idx.size),
            "ref_max_abs": float(np.max(np.abs(ref))), "ref_rms": float(np.sqrt(np.mean(ref * ref))),
            "sumabs_median": float(np.median(sumabs))}
    label = "clustered 64 x 1024, net charge 0" if args.map == "clustered" else "uniform, q ~ U[-1, 1]"
    print(json.dumps({"workload": label, **base}), flush=True)
    for name, fields in FORMS:
        tune = ktt_b200.Tune(block_x=32, block_y=4, z_iterations=args.z_iterations, x_points=args.x_points,
                             **fields)
        ms = []
        for _ in range(args.repeat):
            ctx.forward_3d(atoms, dims, h, tune=tune, out=out)
            ms.append(ctx.elapsed_ms())
        ctx.synchronize()
        got = out.reshape(-1)[torch.from_numpy(idx).cuda()].double().cpu().numpy()
        rep = errors.gate(got, ref, sumabs)
        d = got - ref
        rep["rel_rms"] = float(np.sqrt(np.mean(d * d)) / np.sqrt(np.mean(ref * ref)))
        rep["rel_point_floor_0.1rms"] = errors.report(got, ref, floor=0.1 * base["ref_rms"])["rel_point"]
        # the smallest floor (in rms(V*)) at which every checked point is within the tolerance
        need = np.abs(d) / errors.TOLERANCE
        bad = need > np.abs(ref)
        rep["floor_needed_rms"] = float(need[bad].max() / base["ref_rms"]) if bad.any() else 0.0
        print(json.dumps({"form": name, "tune": tune.as_dict(), "ms": min(ms),
                          "gpairs_per_s": pairs / (min(ms) * 1e-3) / 1e9, **rep}), flush=True)
    ctx.close()


if __name__ == "__main__":
    main()
