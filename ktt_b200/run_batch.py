"""Measure the batched persistent path on the uneven-molecule batch.

    python -m ktt_b200.run_batch [--molecules 512] [--repeat 3] [--margin 8] [--fast-fp32] [--set field=value ...]
    python -m ktt_b200.run_batch --autotune-ktt-form [--save ktt_b200/tuned/b200_batch.json]

512 molecules with atom counts log-uniform in [200, 20000] (seeded), atoms uniform in a cube of side
(n / 0.1)^(1/3) A, grids = bounding box + `margin` A on every side at 0.5 A.  Prints one JSON line
with the device time and pair rate of: one persistent launch, its CUDA-graph replay, one launch of
the same kernel form per molecule, one synchronous launch per molecule of KTT's kernel form (atoms
in __constant__ memory, all rsqrts on MUFU, FP32; what a KTT user's per-molecule Tuner::Run loop
launches), and one synchronous launch per molecule of KTT's plain reference kernel form
(directCoulombSumReference: one point per thread, Examples/CoulombSum3d/CoulombSum3dReference.cu).

The batched kernel's tile comes from `python -m ktt_b200.autotune batch` (KTT's searchers over the
tuner's coulombBatch definition), stored under "batched" (the pointwise-accurate FP64-merge form) and,
for FP32 accumulation, under "fast_fp32" (--fast-fp32 measures that one); --autotune-ktt-form searches the KTT-form
baseline's (z_iterations, x_points, CTA shape) exhaustively on the batch and stores it under
"ktt_form", so both arms run at their best tile shape.
"""
from __future__ import annotations

import argparse
import json
import os

KTT_FORMS = [(zi, xp) for zi in (4, 8, 16) for xp in (1, 2, 4)]
KTT_CTA_SHAPES = [(32, 4), (16, 8), (32, 8), (64, 4)]
DEFAULT_TUNED = os.path.join(os.path.dirname(__file__), "tuned", "b200_batch.json")


def _time_ktt_form(ctx, inputs, outs, tune, repeat, reference=False):
    """One forward call per molecule, synchronised after each, as Tuner::Run does; device time of
    the whole loop from one event pair around it.  With `reference`, the calls run the plain
    one-point-per-thread reference kernel instead of the tiled kernel form `tune`."""
    import torch
    stream = torch.cuda.current_stream()
    best = float("inf")
    for r in range(repeat + 1):
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for (atoms, dims, h, origin), out in zip(inputs, outs):
            if reference:
                ctx.forward_3d_reference(atoms, dims, h, origin, out=out)
            else:
                ctx.forward_3d(atoms, dims, h, origin, tune=tune, out=out)
            ctx.synchronize()
        stop.record(stream)
        stop.synchronize()
        if r:
            best = min(best, start.elapsed_time(stop))
    return best


def autotune_ktt_form(ctx, inputs, outs, ktt_b200, pairs):
    trials = []
    for zi, xp in KTT_FORMS:
        for bx, by in KTT_CTA_SHAPES:
            tune = ktt_b200.Tune(block_x=bx, block_y=by, z_iterations=zi, x_points=xp,
                                 atom_source=ktt_b200.ATOMS_CONSTANT)
            ms = _time_ktt_form(ctx, inputs, outs, tune, 1)
            trials.append({"tune": tune.as_dict(), "ms": ms, "gpairs_per_s": pairs / (ms * 1e-3) / 1e9})
            print(json.dumps({"ktt_form_trial": trials[-1]}), flush=True)
    return min(trials, key=lambda t: t["ms"])


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--molecules", type=int, default=512)
    ap.add_argument("--repeat", type=int, default=3)
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--margin", type=float, default=8.0, help="A of margin on every side of the bounding box")
    ap.add_argument("--set", action="append", default=[], metavar="FIELD=VALUE")
    ap.add_argument("--autotune-ktt-form", action="store_true")
    ap.add_argument("--fast-fp32", action="store_true", help="the FP32-accumulation tile of the tuned file")
    ap.add_argument("--save", default="", help="write the tuned configurations, with the new ktt_form, to this file")
    ap.add_argument("--tuned", default=DEFAULT_TUNED, help="tuned configurations to start from")
    args = ap.parse_args()

    import torch

    import ktt_b200
    from ktt_b200 import workloads

    mols = workloads.molecule_batch(seed=args.seed, n_mol=args.molecules, margin=args.margin)
    ctx = ktt_b200.CoulombContext(0)
    inputs = [(torch.from_numpy(m.atoms).cuda(), m.dims, m.spacing, m.origin) for m in mols]
    outs = [torch.empty((m.dims[2], m.dims[1], m.dims[0]), dtype=torch.float32, device="cuda") for m in mols]
    pairs = float(sum(m.pairs for m in mols))

    tuned = {}
    if args.tuned and os.path.exists(args.tuned):
        with open(args.tuned) as f:
            tuned = json.load(f)
    out = {"molecules": len(mols), "margin_per_side": args.margin}
    if args.autotune_ktt_form:
        ktt_best = autotune_ktt_form(ctx, inputs, outs, ktt_b200, pairs)
        tuned["ktt_form"] = ktt_best["tune"]
        out["ktt_form_best"] = ktt_best
        if args.save:
            with open(args.save, "w") as f:
                json.dump(tuned, f, indent=1)
                f.write("\n")
    if args.fast_fp32 and "fast_fp32" in tuned:
        tune = ktt_b200.Tune(**tuned["fast_fp32"]["batched"])
    else:
        tune = ktt_b200.Tune(**tuned.get("batched", {})) if tuned else \
            ktt_b200.Tune(block_x=8, block_y=16, z_iterations=8, x_points=2, unroll=2, rsqrt_soft=2)
    ktt_tune = ktt_b200.Tune(**tuned["ktt_form"]) if "ktt_form" in tuned else \
        ktt_b200.Tune(block_x=32, block_y=4, z_iterations=8, x_points=2, atom_source=ktt_b200.ATOMS_CONSTANT)
    for s in args.set:
        k, v = s.split("=", 1)
        setattr(tune, k, int(v))
    batch = ktt_b200.Batch(ctx, inputs, tune)
    out.update({"pairs": batch.total_pairs, "work_items": batch.work_items,
                "grid_ctas": batch.grid_ctas, "tune": tune.as_dict(), "ktt_form_tune": ktt_tune.as_dict(),
                "atoms_min": min(m.atoms.shape[0] for m in mols), "atoms_max": max(m.atoms.shape[0] for m in mols),
                "grid_min": min(min(m.dims) for m in mols), "grid_max": max(max(m.dims) for m in mols)})
    for name, mode in (("separate", ktt_b200.BATCH_SEPARATE), ("persistent", ktt_b200.BATCH_PERSISTENT),
                       ("graph", ktt_b200.BATCH_GRAPH)):
        batch.run(mode)  # warm-up (and graph instantiation)
        ctx.synchronize()
        ms = []
        for _ in range(args.repeat):
            batch.run(mode)
            ms.append(ctx.elapsed_ms())
        out[name] = {"ms": min(ms), "gpairs_per_s": batch.total_pairs / (min(ms) * 1e-3) / 1e9}
    ms = _time_ktt_form(ctx, inputs, outs, ktt_tune, args.repeat)
    out["ktt_form_separate"] = {"ms": ms, "gpairs_per_s": pairs / (ms * 1e-3) / 1e9}
    ms = _time_ktt_form(ctx, inputs, outs, None, args.repeat, reference=True)
    out["reference_separate"] = {"ms": ms, "gpairs_per_s": pairs / (ms * 1e-3) / 1e9}
    out["speedup_graph_vs_separate"] = out["separate"]["ms"] / out["graph"]["ms"]
    out["speedup_graph_vs_ktt_form"] = out["ktt_form_separate"]["ms"] / out["graph"]["ms"]
    out["speedup_graph_vs_reference"] = out["reference_separate"]["ms"] / out["graph"]["ms"]
    print(json.dumps(out))
    batch.close()
    ctx.close()


if __name__ == "__main__":
    main()
