"""Run one forward-map case and report its device time.

    python -m ktt_b200.run_case --dims 128 128 128 --atoms 8192 [--set z_iterations=8 --set rsqrt_soft=2] [--repeat 3]

Seeded uniform atoms in a cube scaled to the grid (q ~ U[-1, 1]), one launch per repeat timed with
the context's event pair.  Used to drive profiler captures of a single kernel on a small case.
"""
from __future__ import annotations

import argparse
import json

import numpy as np


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--dims", type=int, nargs=3, default=[128, 128, 128])
    ap.add_argument("--atoms", type=int, default=8192)
    ap.add_argument("--spacing", type=float, default=0.5)
    ap.add_argument("--set", action="append", default=[], metavar="FIELD=VALUE",
                    help="coul_tune field, e.g. z_iterations=16 (repeatable)")
    ap.add_argument("--repeat", type=int, default=3)
    ap.add_argument("--seed", type=int, default=2)
    args = ap.parse_args()

    import torch

    import ktt_b200

    nx, ny, nz = args.dims
    box = args.spacing * max(args.dims)
    rng = np.random.default_rng(args.seed)
    a = np.empty((args.atoms, 4), dtype=np.float32)
    a[:, :3] = rng.uniform(0.0, box, (args.atoms, 3))
    a[:, 3] = rng.uniform(-1.0, 1.0, args.atoms)
    tune = ktt_b200.Tune(**{k: int(v) for k, v in (s.split("=", 1) for s in args.set)})
    ctx = ktt_b200.CoulombContext(0)
    atoms = torch.from_numpy(a).cuda()
    out = torch.empty((nz, ny, nx), dtype=torch.float32, device="cuda")
    ms = []
    for _ in range(args.repeat):
        ctx.forward_3d(atoms, args.dims, args.spacing, tune=tune, out=out)
        ms.append(ctx.elapsed_ms())
    ctx.synchronize()
    pairs = nx * ny * nz * args.atoms
    best = min(ms)
    print(json.dumps({"dims": args.dims, "atoms": args.atoms, "tune": tune.as_dict(), "ms": ms,
                      "gpairs_per_s": pairs / (best * 1e-3) / 1e9, "checksum": float(out.double().sum())}))
    ctx.close()


if __name__ == "__main__":
    main()
