"""The single-slice 2D case: one z slice of a 256 x 256 grid at 0.5 A, 4,000 atoms.

    python -m ktt_b200.run_slice2d [--repeat 50] [--only BX,BY,XP,ROWS,SPLIT,SOFT]

Atoms x, y ~ U[0, 128), z ~ U[0, 32), q ~ U[-1, 1]; the slice at z = 16 A.  For each compiled 2D
tile shape: device time of the slice kernel (median of --repeat event-timed launches), pair rate,
error against the FP64 oracle over the whole slice.  Shapes include the atom-split form (a cluster
of 2 .. 16 CTAs per point tile, each streaming a share of the atoms; its queue form, a persistent
grid over (tile, atom chunk) items; its balanced form, equal ranges of the (tile, atom) space per
resident CTA) and 2/8 or 3/8 of the rsqrts on the FMA pipe.  Then the whole call as a KTT user makes it (host atoms in, dz^2 slicing on the device,
host slice out; wall clock, median) for the fastest shape, and the FP64 oracle's own time on the
host.  One JSON line per measurement.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

SHAPES = [(bx, by, xp, yi, split, soft, 0) for (bx, by) in ((32, 4), (32, 2), (64, 2), (16, 8), (32, 8), (64, 4))
          for xp in (1, 2, 4) for yi in (1, 2, 4, 8) for split in (0, 2, 4, 8, 16) for soft in (0, 2, 3)]
# the queue form of the atom split (split_form 1): chunk counts beyond a cluster's 16 as well
SHAPES += [(bx, by, xp, yi, split, soft, 1) for (bx, by) in ((32, 4), (16, 8), (64, 2), (32, 8), (64, 4))
           for xp in (1, 2, 4) for yi in (2, 4, 8) for split in (8, 16, 24, 32, 48, 64) for soft in (0, 2, 3)]
# the balanced form (split_form 2): the tile's thread layout x atom groups per CTA (at most 1024 threads)
SHAPES += [(bx, by, xp, yi, groups, soft, 2, unroll) for (bx, by) in ((32, 1), (64, 1), (32, 2), (16, 2))
           for xp in (1, 2, 4) for yi in (2, 4, 8) for groups in (4, 8, 16, 32) for soft in (0, 2, 3, 12)
           for unroll in (1, 2) if 256 <= bx * by * groups <= 1024]


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--repeat", type=int, default=50)
    ap.add_argument("--only", default="", help="one configuration: block x, block y, x points, rows, atom split, "
                                               "rsqrt share[, split form[, unroll]] (for profiling)")
    args = ap.parse_args()
    shapes = [(tuple(int(v) for v in args.only.split(",")) + (0, 1)[len(args.only.split(",")) - 6:])[:8]] \
        if args.only else SHAPES

    import torch

    import ktt_b200
    import oracle
    from ktt_b200 import errors, workloads

    case = workloads.slice_2d()
    nx, ny, h = case.nx, case.ny, case.spacing
    t0 = time.perf_counter()
    ref = oracle.slice2d(case.ktt_atoms(), h, nx, ny)
    oracle_s = time.perf_counter() - t0
    pairs = float(nx * ny * case.atoms.shape[0])

    ctx = ktt_b200.CoulombContext(0)
    atoms = torch.from_numpy(case.atoms).cuda()
    d_sliced = ctx.slice_atoms(atoms, case.z_slice)
    out = torch.empty((ny, nx), dtype=torch.float32, device="cuda")
    results = []
    for bx, by, xp, yi, split, soft, form, *rest in shapes:
        tune = ktt_b200.Tune(block_x=bx, block_y=by, x_points=xp, z_iterations=yi, atom_split=split,
                             rsqrt_soft=soft, split_form=form, unroll=rest[0] if rest else 1)
        if not ktt_b200.tune_supported_2d(tune):
            continue
        ms = []
        try:
            for _ in range(args.repeat):
                ctx.forward_2d(d_sliced, h, nx, ny, tune=tune, out=out)
                ms.append(ctx.elapsed_ms())
        except ktt_b200.CoulombError as e:
            if e.status != ktt_b200.COUL_ERR_DEVICE_LIMITS:
                raise
            continue  # e.g. a 16-CTA cluster of blocks too large to be co-resident
        ctx.synchronize()
        rep = errors.report(out.double().cpu().numpy(), ref)
        med = float(np.median(ms))
        line = {"tune": tune.as_dict(), "ms_median": med, "ms_min": min(ms),
                "gpairs_per_s": pairs / (med * 1e-3) / 1e9, "rel_norm": rep["rel_norm"]}
        results.append(line)
        print(json.dumps(line), flush=True)
    best = min(results, key=lambda r: r["ms_median"])
    tune = ktt_b200.Tune(**best["tune"])

    host_out = np.empty((ny, nx), dtype=np.float32)
    pinned_in = torch.from_numpy(case.atoms).pin_memory()
    pinned_out = torch.empty((ny, nx), dtype=torch.float32).pin_memory()
    wall = []
    for _ in range(args.repeat):
        t0 = time.perf_counter()
        d_atoms = pinned_in.to("cuda", non_blocking=True)
        s = ctx.slice_atoms(d_atoms, case.z_slice)
        ctx.forward_2d(s, h, nx, ny, tune=tune, out=out)
        pinned_out.copy_(out, non_blocking=True)
        ctx.synchronize()
        torch.cuda.synchronize()
        host_out[...] = pinned_out.numpy()
        wall.append(time.perf_counter() - t0)
    rep = errors.report(host_out, ref)
    print(json.dumps({"best_tune": best["tune"], "kernel_ms_median": best["ms_median"],
                      "kernel_gpairs_per_s": best["gpairs_per_s"],
                      "host_call_ms_median": float(np.median(wall)) * 1e3,
                      "host_call_gpairs_per_s": pairs / float(np.median(wall)) / 1e9,
                      "host_call_rel_norm": rep["rel_norm"],
                      "oracle_fp64_ms": oracle_s * 1e3, "oracle_threads": oracle.max_threads()}), flush=True)
    ctx.close()


if __name__ == "__main__":
    main()
