"""Measure the N-body step (coul_nbody_step) over its configuration space.

    python -m ktt_b200.run_nbody [--n 131072] [--repeat 5] [--only BX,BP,UN,JS]

Bodies as in KTT's Nbody example (positions, masses, velocities uniform in [0, 20); dt 0.001,
damping 0.5, softening 0.1^2; 131,072 bodies by default, Examples/Nbody/Nbody.cpp:62-118).  For every
compiled configuration (block size x bodies per thread x unroll x j-split): device time (best of
--repeat event-timed steps), body-body interactions per second, and the fraction of the FP32-pipe
bound F / 12 (12 FP32 operations per interaction; F measured now by the library's microkernel).
One JSON line per configuration, then a summary line with the best.
"""
from __future__ import annotations

import argparse
import json

import numpy as np

CONFIGS = [(bx, bp, un, js) for bx in (64, 128, 256) for bp in (2, 4, 8) for un in (1, 2, 4) for js in (0, 2, 4)]


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=128 * 1024)
    ap.add_argument("--repeat", type=int, default=5)
    ap.add_argument("--only", default="", metavar="BX,BP,UN,JS",
                    help="run one configuration (block_x, bodies_per_thread, unroll, j_split), e.g. for a profiler")
    args = ap.parse_args()
    configs = [tuple(int(v) for v in args.only.split(","))] if args.only else CONFIGS

    import torch

    import ktt_b200

    rng = np.random.default_rng(11)
    pos = rng.uniform(0.0, 20.0, (args.n, 4)).astype(np.float32)
    vel = rng.uniform(0.0, 20.0, (args.n, 4)).astype(np.float32)
    vel[:, 3] = 0.0
    ctx = ktt_b200.CoulombContext(0)
    tp, tv = torch.from_numpy(pos).cuda(), torch.from_numpy(vel).cuda()
    op, ov = torch.empty_like(tp), torch.empty_like(tv)
    rsqrt_rate, ffma_rate = ctx.pipe_rates()
    bound = ffma_rate / 12.0
    interactions = float(args.n) * args.n
    rows = []
    for bx, bp, un, js in configs:
        tune = ktt_b200.NbodyTune(block_x=bx, bodies_per_thread=bp, unroll=un, j_split=js)
        if not ktt_b200.nbody_tune_supported(tune):
            continue
        ktt_b200.nbody_step(ctx, tp, tv, 0.001, 0.5, 0.01, tune, op, ov)
        ms = []
        for _ in range(args.repeat):
            ktt_b200.nbody_step(ctx, tp, tv, 0.001, 0.5, 0.01, tune, op, ov)
            ms.append(ctx.elapsed_ms())
        ctx.synchronize()
        rate = interactions / (min(ms) * 1e-3)
        row = {"tune": {"block_x": bx, "bodies_per_thread": bp, "unroll": un, "j_split": js}, "ms": min(ms),
               "ginteractions_per_s": rate / 1e9, "frac_fp32_bound": rate / bound}
        rows.append(row)
        print(json.dumps(row), flush=True)
    best = min(rows, key=lambda r: r["ms"])
    print(json.dumps({"n": args.n, "best": best, "fp32_bound_ginteractions_per_s": bound / 1e9,
                      "ffma_per_s": ffma_rate, "rsqrt_per_s": rsqrt_rate,
                      "gflops_20_per_interaction": best["ginteractions_per_s"] * 20}), flush=True)
    ctx.close()


if __name__ == "__main__":
    main()
