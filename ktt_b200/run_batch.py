"""Measure the batched persistent path on the uneven-molecule batch.

    python -m ktt_b200.run_batch [--molecules 512] [--repeat 3] [--set field=value ...]

512 molecules with atom counts log-uniform in [200, 20000] (seeded), atoms uniform in a cube of side
(n / 0.1)^(1/3) A, grids = bounding box + 8 A margin at 0.5 A.  Prints one JSON line with the
device time and pair rate of: one persistent launch, its CUDA-graph replay, and one plain launch
per molecule.
"""
from __future__ import annotations

import argparse
import json


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--molecules", type=int, default=512)
    ap.add_argument("--repeat", type=int, default=3)
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--set", action="append", default=[], metavar="FIELD=VALUE")
    args = ap.parse_args()

    import torch

    import ktt_b200
    from ktt_b200 import workloads

    mols = workloads.molecule_batch(seed=args.seed, n_mol=args.molecules)
    ctx = ktt_b200.CoulombContext(0)
    inputs = [(torch.from_numpy(m.atoms).cuda(), m.dims, m.spacing, m.origin) for m in mols]
    tune = ktt_b200.Tune(z_iterations=8, x_points=2, unroll=2, rsqrt_soft=2)
    for s in args.set:
        k, v = s.split("=", 1)
        setattr(tune, k, int(v))
    batch = ktt_b200.Batch(ctx, inputs, tune)
    out = {"molecules": len(mols), "pairs": batch.total_pairs, "work_items": batch.work_items,
           "grid_ctas": batch.grid_ctas, "tune": tune.as_dict(),
           "atoms_min": min(m.atoms.shape[0] for m in mols), "atoms_max": max(m.atoms.shape[0] for m in mols),
           "grid_min": min(min(m.dims) for m in mols), "grid_max": max(max(m.dims) for m in mols)}
    for name, mode in (("separate", ktt_b200.BATCH_SEPARATE), ("persistent", ktt_b200.BATCH_PERSISTENT),
                       ("graph", ktt_b200.BATCH_GRAPH)):
        batch.run(mode)  # warm-up (and graph instantiation)
        ctx.synchronize()
        ms = []
        for _ in range(args.repeat):
            batch.run(mode)
            ms.append(ctx.elapsed_ms())
        out[name] = {"ms": min(ms), "gpairs_per_s": batch.total_pairs / (min(ms) * 1e-3) / 1e9}
    out["speedup_graph_vs_separate"] = out["separate"]["ms"] / out["graph"]["ms"]
    print(json.dumps(out))
    batch.close()
    ctx.close()


if __name__ == "__main__":
    main()
