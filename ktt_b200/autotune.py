"""Autotuner for this library's map kernels, on top of the ktt:: searchers.

    python -m ktt_b200.autotune map3d [--searcher mcmc|random|deterministic] [--budget 60] [--save]
    python -m ktt_b200.autotune batch [--searcher mcmc|random|deterministic] [--budget 40] [--save]
    python -m ktt_b200.autotune map3d --dry-run          # the configuration space only (no GPU)
    python -m ktt_b200.autotune map3d --profile --results space.json ...   # record counters of every run
    python -m ktt_b200.autotune map3d --searcher profile --model model.json # KTT's profile-based searcher

The kernel is registered with the ktt:: tuner exactly as a KTT host program registers
directCoulombSum (Examples/CoulombSum3d/CoulombSum3d.cpp:100-237) -- definition, arguments, tuning
parameters with thread modifiers and constraints -- with the B200 parameters added (X_POINTS,
RSQRT_SOFT) and a constraint that keeps the search inside the compiled variants; the batched map is
the tuner's "coulombBatch" definition.  KTT's searchers pick the configurations (MCMC by default,
Examples' ConfigurationCount budget), every configuration is validated by the tuner against a
reference computation registered through Tuner::SetReferenceComputation (Source/Tuner.h:610;
SideBySide within 1e-5 of the largest value), and the fastest valid configuration is written to
ktt_b200/tuned/b200_map3d.json or b200_batch.json with --save (the files bench.py and
ktt_b200.Batch read).  The reference computation is the caller's (tune_map3d / tune_batch take an
FP64 map function, e.g. a CPU restatement of KTT's reference computation); without one it is the
library's FP64 reference kernel (coul_forward_3d_reference_fp64: one point per thread, FP64
differences, square root and division), which shares no arithmetic with the tuned kernels.
"""
from __future__ import annotations

import argparse
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TUNED = os.path.join(HERE, "tuned")

MAP3D_SPACE = {
    "WORK_GROUP_SIZE_X": [16, 32, 64, 128],
    "WORK_GROUP_SIZE_Y": [1, 2, 4, 8],
    "Z_ITERATIONS": [4, 8, 16],
    "X_POINTS": [1, 2, 4],
    "INNER_UNROLL_FACTOR": [0, 2, 4],
    "RSQRT_SOFT": [0, 1, 2, 3, 11, 12],
}
BATCH_SPACE = {
    "WORK_GROUP_SIZE_X": [4, 8, 16, 32],
    "WORK_GROUP_SIZE_Y": [4, 8, 16, 32],
    "Z_ITERATIONS": [4, 8, 16],
    "X_POINTS": [1, 2, 4],
    "INNER_UNROLL_FACTOR": [0, 2],
    "RSQRT_SOFT": [0, 2, 12],
}


def _unroll(factor: int) -> int:
    # the tuner's INNER_UNROLL_FACTOR -> compiled unroll mapping (0 and 1: none)
    return 1 if factor <= 1 else (2 if factor < 4 else (4 if factor < 8 else 8))


def _tune_from(values, names):
    import ktt_b200
    v = dict(zip(names, values))
    return ktt_b200.Tune(block_x=v["WORK_GROUP_SIZE_X"], block_y=v["WORK_GROUP_SIZE_Y"], z_iterations=v["Z_ITERATIONS"],
                         x_points=v["X_POINTS"], unroll=_unroll(v["INNER_UNROLL_FACTOR"]), rsqrt_soft=v["RSQRT_SOFT"],
                         precision=v.get("PRECISION", 0))


def _add_space(ktt, tuner, kernel, definition, space, supported, precisions=(0,)):
    """The space's parameters, PRECISION (the accumulation forms searched), KTT's thread modifiers and
    the constraints."""
    space = dict(space, PRECISION=list(precisions))
    names = list(space)
    for name, values in space.items():
        tuner.AddParameter(kernel, name, values)
    # KTT's thread modifiers of the 3D example (the launch sizes recorded in the results)
    for dim, name in ((ktt.ModifierDimension.X, "WORK_GROUP_SIZE_X"), (ktt.ModifierDimension.Y, "WORK_GROUP_SIZE_Y")):
        tuner.AddThreadModifier(kernel, [definition], ktt.ModifierType.Local, dim, name, ktt.ModifierAction.Multiply)
        tuner.AddThreadModifier(kernel, [definition], ktt.ModifierType.Global, dim, name, ktt.ModifierAction.DivideCeil)
    tuner.AddThreadModifier(kernel, [definition], ktt.ModifierType.Global, ktt.ModifierDimension.Z, "Z_ITERATIONS",
                            ktt.ModifierAction.DivideCeil)
    tuner.AddConstraint(kernel, ["WORK_GROUP_SIZE_X", "WORK_GROUP_SIZE_Y"], lambda v: 32 <= v[0] * v[1] <= 256)
    # stay inside the compiled variants (a configuration outside them would only report CompilationFailed)
    tuner.AddConstraint(kernel, names, lambda v: supported(_tune_from(v, names)))


SEARCHERS = ["mcmc", "random", "deterministic", "profile"]


def _searcher(ktt, name, tuner=None, model="", seed=None):
    if name == "profile":
        # KTT's profile-based searcher (native, include/ktt/ProfileBasedSearcher.h) with a counter model
        # trained by ktt_b200.profile_model from results recorded with --profile
        if not model:
            raise ValueError("the profile-based searcher needs --model (see ktt_b200/profile_model.py)")
        return ktt.ProfileBasedSearcher(tuner, ktt.CounterModel.Load(model), 5, 100, 10,
                                        seed if seed is not None else int.from_bytes(os.urandom(8), "little"))
    return {"mcmc": ktt.McmcSearcher, "random": ktt.RandomSearcher, "deterministic": ktt.DeterministicSearcher}[name]()


def _run(ktt, tuner, kernel, searcher, budget, profile, results_path, model, seed):
    """The search itself: searcher, optional counters on every run, optional KTT-format results file."""
    tuner.SetSearcher(kernel, _searcher(ktt, searcher, tuner, model, seed))
    if profile:
        tuner.SetProfiling(True)
    results = tuner.Tune(kernel, ktt.ConfigurationCount(budget))
    tuner.SetProfiling(False)
    if results_path:
        base = results_path[:-5] if results_path.endswith(".json") else results_path
        tuner.SaveResults(results, base, ktt.OutputFormat.JSON)
    return results


def _summary(results, work):
    trials = []
    for r in results:
        cfg = {p.GetName(): int(p.GetValueString()) for p in r.GetConfiguration().GetPairs()}
        ns = r.GetTotalDuration()
        trials.append({"config": cfg, "status": str(r.GetStatus()).split(".")[-1],
                       "profiled": bool(r.GetResults()) and r.GetResults()[0].HasProfilingData(),
                       "ms": ns * 1e-6 if r.IsValid() else None,
                       "gpairs_per_s": work / (ns * 1e-9) / 1e9 if r.IsValid() and ns > 0 else None})
    valid = [t for t in trials if t["gpairs_per_s"] is not None]
    if not valid:
        raise RuntimeError("no configuration validated")
    best = max(valid, key=lambda t: t["gpairs_per_s"])
    return best, trials


REFERENCE_KERNEL = "FP64 reference kernel (coul_forward_3d_reference_fp64)"


def _fp64_maps(problems, reference):
    """FP64 maps of (atoms, dims, spacing, origin) problems: reference(atoms, spacing, dims, origin) when
    given, else the FP64 reference kernel on the GPU."""
    if reference is not None:
        return [np.asarray(reference(a, h, dims, origin), dtype=np.float64) for a, dims, h, origin in problems]
    import torch

    import ktt_b200
    ctx = ktt_b200.CoulombContext(0)
    try:
        maps = []
        for a, dims, h, origin in problems:
            v = ctx.forward_3d_reference_fp64(torch.from_numpy(a).cuda(), dims, h, origin)
            maps.append(v.cpu().numpy())
        return maps
    finally:
        ctx.close()


def tune_map3d(grid: int = 256, atoms: int = 65536, searcher: str = "mcmc", budget: int = 60,
               dry_run: bool = False, profile: bool = False, results_path: str = "", model: str = "",
               seed: int | None = None, reference=None, reference_name: str = "", precisions=(0,)) -> dict:
    """Searches the single-map tile space on the uniform workload (grid^3 points at 0.5 A, `atoms` atoms
    uniform in the cube the grid spans).  dry_run: only build the space and report its size.
    reference(atoms, spacing, dims, origin) -> FP64 map of shape (nz, ny, nx) is the reference
    computation every configuration is validated against (default: the FP64 reference kernel)."""
    import ktt_b200
    from ktt_b200 import pyktt as ktt
    from ktt_b200 import workloads
    w = workloads.uniform_map(n_atoms=atoms, n=grid, box=grid * 0.5)
    g, n, h = grid, atoms, w.spacing
    tuner = ktt.Tuner(0, 0, ktt.ComputeApi.CUDA)
    tuner.SetGlobalSizeType(ktt.GlobalSizeType.CUDA)
    definition = tuner.AddKernelDefinition("directCoulombSum", "", ktt.DimensionVector(g, g, g), ktt.DimensionVector())
    kernel = tuner.CreateSimpleKernel("CoulombSum", definition)
    _add_space(ktt, tuner, kernel, definition, MAP3D_SPACE, ktt_b200.tune_supported, precisions)
    if dry_run:
        return {"configurations": tuner.GetConfigurationsCount(kernel)}

    ro = ktt.ArgumentAccessType.ReadOnly
    arg_ids = [tuner.AddArgumentVectorFloat(w.atoms.reshape(-1), ro)]
    arg_ids += [tuner.AddArgumentVectorFloat(np.ascontiguousarray(w.atoms[:, c]), ro) for c in range(4)]
    arg_ids += [tuner.AddArgumentScalarInt(n), tuner.AddArgumentScalarFloat(h), tuner.AddArgumentScalarInt(g)]
    grid_id = tuner.AddArgumentVectorFloat(np.zeros(g ** 3, dtype=np.float32), ktt.ArgumentAccessType.WriteOnly)
    arg_ids.append(grid_id)
    tuner.SetArguments(definition, arg_ids)

    ref = _fp64_maps([(w.atoms, w.dims, h, None)], reference)[0].reshape(-1)

    def compute_reference(buffer):
        np.frombuffer(buffer, dtype=np.float32)[:] = ref

    tuner.SetReferenceComputation(grid_id, g ** 3 * 4, compute_reference)
    threshold = 1e-5 * float(np.abs(ref).max())
    tuner.SetValidationMethod(ktt.ValidationMethod.SideBySideComparison, threshold)
    results = _run(ktt, tuner, kernel, searcher, budget, profile, results_path, model, seed)
    best, trials = _summary(results, float(g) ** 3 * n)
    out = {
        "workload": f"{g}^3 grid, h={h} A, {n} atoms uniform in the {g * h:g} A cube",
        "device": tuner.GetCurrentDeviceInfo().GetName(),
        "selection": "fastest configuration whose map stays within 1e-5 of the largest value of the FP64 reference "
                     "map at every point",
        "reference": reference_name or (REFERENCE_KERNEL if reference is None else "caller's FP64 reference computation"),
        "source": f"ktt_b200.autotune map3d: {searcher} searcher, {len(results)} of "
                  f"{tuner.GetConfigurationsCount(kernel)} configurations, kernel time from the tuner's event pair",
        "gpairs_per_s": round(best["gpairs_per_s"], 1),
        "precisions": list(precisions),
        "tune": _tune_from([best["config"][k] for k in list(MAP3D_SPACE) + ["PRECISION"]],
                           list(MAP3D_SPACE) + ["PRECISION"]).as_dict(),
        "trials": trials,
    }
    return out


def tune_batch(molecules: int = 512, seed: int = 4, searcher: str = "mcmc", budget: int = 40,
               dry_run: bool = False, profile: bool = False, results_path: str = "", model: str = "",
               search_seed: int | None = None, reference=None, reference_name: str = "",
               precisions=(0,)) -> dict:
    """Searches the batched-map tile space (the coulombBatch definition) on the uneven molecule batch
    (`molecules` molecules of 200-20000 atoms, log-uniform, from `seed`) over the accumulation forms
    `precisions`; reference as in tune_map3d, applied to every molecule."""
    import ktt_b200
    from ktt_b200 import pyktt as ktt
    from ktt_b200 import workloads
    mols = workloads.molecule_batch(seed=seed, n_mol=molecules)
    tuner = ktt.Tuner(0, 0, ktt.ComputeApi.CUDA)
    tuner.SetGlobalSizeType(ktt.GlobalSizeType.CUDA)
    definition = tuner.AddKernelDefinition("coulombBatch", "", ktt.DimensionVector(1, 1, 2), ktt.DimensionVector())
    kernel = tuner.CreateSimpleKernel("CoulombBatch", definition)
    _add_space(ktt, tuner, kernel, definition, BATCH_SPACE, ktt_b200.batch_tune_supported, precisions)
    if dry_run:
        return {"configurations": tuner.GetConfigurationsCount(kernel)}

    atom_off = np.zeros(len(mols) + 1, dtype=np.int64)
    map_off = np.zeros(len(mols) + 1, dtype=np.int64)
    for i, m in enumerate(mols):
        atom_off[i + 1] = atom_off[i] + m.atoms.shape[0]
        # keep every map 16-byte aligned so the vectorised stores stay available
        size = m.dims[0] * m.dims[1] * m.dims[2]
        map_off[i + 1] = map_off[i] + (size + 3) // 4 * 4
    grids = np.array([[*m.dims, m.spacing, *m.origin] for m in mols], dtype=np.float32).reshape(-1)
    atoms = np.concatenate([m.atoms for m in mols]).astype(np.float32).reshape(-1)
    ro = ktt.ArgumentAccessType.ReadOnly
    ids = [tuner.AddArgumentVectorFloat(atoms, ro), tuner.AddArgumentVectorLong(atom_off, ro),
           tuner.AddArgumentVectorFloat(grids, ro)]
    maps_id = tuner.AddArgumentVectorFloat(np.zeros(int(map_off[-1]), dtype=np.float32), ktt.ArgumentAccessType.WriteOnly)
    ids += [maps_id, tuner.AddArgumentVectorLong(map_off, ro), tuner.AddArgumentScalarInt(len(mols))]
    tuner.SetArguments(definition, ids)

    ref = np.zeros(int(map_off[-1]), dtype=np.float32)
    maps = _fp64_maps([(m.atoms, m.dims, m.spacing, m.origin) for m in mols], reference)
    for i, m in enumerate(mols):
        size = m.dims[0] * m.dims[1] * m.dims[2]
        ref[map_off[i]:map_off[i] + size] = maps[i].reshape(-1)

    def compute_reference(buffer):
        np.frombuffer(buffer, dtype=np.float32)[:] = ref

    tuner.SetReferenceComputation(maps_id, ref.size * 4, compute_reference)
    tuner.SetValidationMethod(ktt.ValidationMethod.SideBySideComparison, 1e-5 * float(np.abs(ref).max()))
    results = _run(ktt, tuner, kernel, searcher, budget, profile, results_path, model, search_seed)
    pairs = float(sum(m.pairs for m in mols))
    best, trials = _summary(results, pairs)
    return {
        "batched": _tune_from([best["config"][k] for k in list(BATCH_SPACE) + ["PRECISION"]],
                              list(BATCH_SPACE) + ["PRECISION"]).as_dict(),
        "batched_gpairs_per_s": round(best["gpairs_per_s"], 1),
        "precisions": list(precisions),
        "workload": f"{len(mols)} molecules, seed {seed}, margin 8 A per side",
        "source": f"ktt_b200.autotune batch: {searcher} searcher, {len(results)} of "
                  f"{tuner.GetConfigurationsCount(kernel)} configurations of the coulombBatch definition",
        "reference": reference_name or (REFERENCE_KERNEL if reference is None else "caller's FP64 reference computation"),
        "trials": trials,
    }


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("target", choices=["map3d", "batch"])
    ap.add_argument("--searcher", choices=SEARCHERS, default="mcmc")
    ap.add_argument("--model", default="", help="counter model of the profile-based searcher")
    ap.add_argument("--search-seed", type=int, default=None, help="seed of the profile-based searcher")
    ap.add_argument("--profile", action="store_true", help="collect hardware counters on every run")
    ap.add_argument("--results", default="", help="also write the tuner's results (KTT JSON) to this file")
    ap.add_argument("--budget", type=int, default=0, help="configurations to test (default 60 map3d, 40 batch)")
    ap.add_argument("--atoms", type=int, default=65536)
    ap.add_argument("--grid", type=int, default=256)
    ap.add_argument("--molecules", type=int, default=512)
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--dry-run", action="store_true", help="report the configuration space only")
    ap.add_argument("--precisions", default="0", help="accumulation forms to search, e.g. 2,4")
    ap.add_argument("--save", action="store_true", help="write ktt_b200/tuned/b200_<target>.json")
    ap.add_argument("--out", default="", help="write the result to this file instead")
    args = ap.parse_args()
    args.budget = args.budget or (60 if args.target == "map3d" else 40)

    from ktt_b200 import pyktt as ktt
    ktt.Tuner.SetLoggingLevel(ktt.LoggingLevel.Warning)
    if args.target == "map3d":
        result = tune_map3d(args.grid, args.atoms, args.searcher, args.budget, args.dry_run, args.profile,
                            args.results, args.model, args.search_seed,
                            precisions=tuple(int(p) for p in args.precisions.split(",")))
    else:
        result = tune_batch(args.molecules, args.seed, args.searcher, args.budget, args.dry_run, args.profile,
                            args.results, args.model, args.search_seed,
                            precisions=tuple(int(p) for p in args.precisions.split(",")))
    print(json.dumps({k: v for k, v in result.items() if k != "trials"}))
    path = args.out or (os.path.join(TUNED, "b200_map3d.json" if args.target == "map3d" else "b200_batch.json")
                        if args.save else "")
    if path and not args.dry_run:
        if args.target == "batch" and os.path.exists(path):
            with open(path) as f:
                previous = json.load(f)
            # keep the KTT-form baseline tile the batch measurement compares against, and the fastest
            # FP32 tile of an earlier search
            for key in ("ktt_form", "fast_fp32"):
                if key in previous:
                    result[key] = previous[key]
        with open(path, "w") as f:
            json.dump(result, f, indent=1)
            f.write("\n")


if __name__ == "__main__":
    main()
