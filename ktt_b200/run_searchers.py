"""Convergence of the searchers on a recorded, profiled search (no GPU needed).

    python -m ktt_b200.run_searchers [--space tests/golden/b200_map3d_space_64.json] [--seeds 40] [--budget 120]

The recorded search holds, for every configuration of a tuning space, its kernel time and KTT's
default counters: a compact recording (tests/golden/make_b200_space.py) or the KTT-format results file
of `python -m ktt_b200.autotune ... --profile --results FILE`.  Each searcher is replayed through the tuner's
SimulateTuning with that many seeds: random order (KTT's RandomSearcher, drawn here without
replacement per seed), MCMC (KTT's McmcSearcher, seeded), and the profile-based searcher (KTT's
algorithm, native) with a counter model trained by ktt_b200.profile_model (KTT's recipe: half of the
profiled configurations, ExtraTreesRegressor(10)) from the same recording or, with --model-space,
from another one.  Profiled reruns count
as tested configurations.  Prints one JSON line: per searcher, the mean and median number of tested
configurations until one within 1 % / 5 % of the space's best was found, and the mean ratio of the
best time found to the space's best after 10, 20, 40 and 80 tested configurations.
"""
from __future__ import annotations

import argparse
import json
import os
import random
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_SPACE = os.path.join(os.path.dirname(HERE), "tests", "golden", "b200_map3d_space_64.json")


def load_space(path: str) -> dict:
    """A compact recording (tests/golden/make_b200_space.py) or a KTT-format result file with counters."""
    doc = json.load(open(path))
    results = doc.get("Results", [])
    if not results or "ComputationResults" not in results[0]:
        return doc
    first = next(r for r in results if r["ComputationResults"][0].get("ProfilingData"))
    names = [c["Name"] for c in first["ComputationResults"][0]["ProfilingData"]["Counters"]]
    compact = []
    for r in results:
        cr = r["ComputationResults"][0]
        values = {c["Name"]: c["Value"] for c in cr.get("ProfilingData", {}).get("Counters", [])}
        compact.append({"Configuration": [[p["Name"], p["Value"]] for p in r["Configuration"]], "Status": r["Status"],
                        "Duration": cr["Duration"], "GlobalSize": [cr["GlobalSize"][k] for k in "XYZ"],
                        "LocalSize": [cr["LocalSize"][k] for k in "XYZ"],
                        "Counters": [values.get(n) for n in names]})
    return {"Metadata": doc.get("Metadata", {}), "CounterNames": names, "Results": compact}


def write_ktt_results(space: dict, path: str) -> None:
    """The compact recording as a KTT-format result file with profiling data."""
    results = []
    for r in space["Results"]:
        cr = {"CompilationOverhead": 0.0, "Duration": r["Duration"], "GlobalSize": dict(zip("XYZ", r["GlobalSize"])),
              "KernelFunction": "directCoulombSum", "LocalSize": dict(zip("XYZ", r["LocalSize"])), "Overhead": 0.0,
              "ProfilingData": {"Counters": [{"Name": n, "Type": "Double", "Value": v}
                                             for n, v in zip(space["CounterNames"], r["Counters"])],
                                "RemainingProfilingRuns": 0}}
        results.append({"ComputationResults": [cr],
                        "Configuration": [{"Name": n, "Value": v, "ValueType": "UnsignedInt"} for n, v in r["Configuration"]],
                        "DataMovementOverhead": 0.0, "ExtraDuration": 0.0, "KernelName": "CoulombSum",
                        "SearcherOverhead": 0.0, "Status": r["Status"], "TotalDuration": r["Duration"],
                        "TotalOverhead": 0.0, "ValidationOverhead": 0.0})
    with open(path, "w") as f:
        json.dump({"Metadata": space["Metadata"], "Results": results}, f)


def build_space(ktt, tuner, space: dict):
    """The recorded configurations as a tuning space (every recorded value of every parameter, limited to
    the recorded combinations)."""
    names = [n for n, _ in space["Results"][0]["Configuration"]]
    recorded = {tuple(v for _, v in r["Configuration"]) for r in space["Results"]}
    d = tuner.AddKernelDefinition("directCoulombSum", "", ktt.DimensionVector(64, 64, 64), ktt.DimensionVector())
    k = tuner.CreateSimpleKernel("CoulombSum", d)
    for i, n in enumerate(names):
        tuner.AddParameter(k, n, sorted({c[i] for c in recorded}))
    tuner.AddConstraint(k, names, lambda v: tuple(v) in recorded)
    return k


def _curve(durations, best):
    """Tested configurations until within 1 % / 5 % of best, and best-so-far ratios."""
    running, curve = float("inf"), []
    for t in durations:
        running = min(running, t)
        curve.append(running / best)
    def first(limit):
        return next((i + 1 for i, v in enumerate(curve) if v <= limit), len(curve) + 1)
    at = {n: curve[min(n, len(curve)) - 1] for n in (10, 20, 40, 80)}
    return first(1.01), first(1.05), at


def main(argv=None) -> dict:
    ap = argparse.ArgumentParser()
    ap.add_argument("--space", default=DEFAULT_SPACE)
    ap.add_argument("--model-space", default="", help="train the counter model on this recording instead "
                    "(another input size, as KTT's models come from historical runs)")
    ap.add_argument("--seeds", type=int, default=40)
    ap.add_argument("--budget", type=int, default=120)
    ap.add_argument("--cc", default="10.0", help="compute capability of the recording's device")
    ap.add_argument("--sms", type=int, default=148, help="SM count of the recording's device")
    ap.add_argument("--xu", action="store_true", help="the profile-based searcher with the XU-pipe addition")
    args = ap.parse_args(argv)
    cc_major, cc_minor = (int(x) for x in args.cc.split("."))

    from ktt_b200 import profile_model
    from ktt_b200 import pyktt as ktt
    ktt.Tuner.SetLoggingLevel(ktt.LoggingLevel.Error)
    space = load_space(args.space)
    ok = [r for r in space["Results"] if r["Status"] == "Ok"]
    best = min(r["Duration"] for r in ok)
    times = {tuple(v for _, v in r["Configuration"]): r["Duration"] for r in ok}

    with tempfile.TemporaryDirectory() as tmp:
        results_path = os.path.join(tmp, "space.json")
        model_path = os.path.join(tmp, "model.json")
        write_ktt_results(space, results_path)
        training_path = results_path
        if args.model_space:
            training_path = os.path.join(tmp, "training.json")
            write_ktt_results(load_space(args.model_space), training_path)
        profile_model.main([training_path, "--out", model_path, "--cc", args.cc, "--multiprocessors", str(args.sms)])
        model = ktt.CounterModel.Load(model_path)

        runs = {"random": [], "mcmc": [], "profile": []}
        for seed in range(args.seeds):
            order = list(times.values())
            random.Random(seed).shuffle(order)
            runs["random"].append(order[:args.budget])
            for name in ("mcmc", "profile"):
                tuner = ktt.Tuner(0, 0, ktt.ComputeApi.CUDA)
                k = build_space(ktt, tuner, space)
                if name == "mcmc":
                    searcher = ktt.McmcSearcher(ktt.KernelConfiguration(), seed + 1)
                else:
                    searcher = ktt.ProfileBasedSearcher(tuner, model, 5, 100, 10, seed + 1)
                    searcher.SetDeviceProperties(cc_major, cc_minor, args.sms)
                    searcher.SetXuPipeAnalysis(args.xu)
                tuner.SetSearcher(k, searcher)
                rec = tuner.SimulateTuning(k, tuner.LoadResults(results_path, ktt.OutputFormat.JSON),
                                           ktt.ConfigurationCount(args.budget))
                runs[name].append([times[tuple(int(p.GetValueString()) for p in r.GetConfiguration().GetPairs())]
                                   for r in rec])

    report = {"space": os.path.relpath(args.space),
              "model_space": os.path.relpath(args.model_space or args.space), "configurations": len(ok), "seeds": args.seeds,
              "budget": args.budget, "best_ms": best}
    for name, lists in runs.items():
        stats = [_curve(d, best) for d in lists]
        report[name] = {
            "to_1pct_mean": float(np.mean([s[0] for s in stats])), "to_1pct_median": float(np.median([s[0] for s in stats])),
            "to_5pct_mean": float(np.mean([s[1] for s in stats])), "to_5pct_median": float(np.median([s[1] for s in stats])),
            "best_ratio_after": {n: float(np.mean([s[2][n] for s in stats])) for n in (10, 20, 40, 80)},
        }
    print(json.dumps(report))
    return report


if __name__ == "__main__":
    main()
