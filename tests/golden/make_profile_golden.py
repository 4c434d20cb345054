"""Golden vectors of KTT's profile-based searcher arithmetic, from KTT's own Python code.

Run from the repository root where the KTT 2.1.0 tree is mounted (no GPU, no pyktt needed):

    python tests/golden/make_profile_golden.py --ktt-root KTT_TREE   (or KTT_ROOT=KTT_TREE in the environment)

It imports ``Scripts/ProfileBasedSearcher.py`` from the KTT tree with a stand-in ``pyktt`` module
(only its class bodies refer to pyktt) and evaluates its functions on the recorded 2080 Ti counters
of ``coulomb3d_2080_space.json`` (next to this script) plus a few synthetic B200-like counter sets:

* ``analyzeBottlenecks`` (compute capability >= 7 branch) for each counter set;
* ``computeChanges`` against the counter list of KTT's shipped 2080 model
  (``Examples/CoulombSum3d/Models/2080-coulomb_output_DT.sav.metadata.json``, read as JSON; the
  pickled model itself is not loaded);
* ``scoreTuningConfigurationsPredictor`` with a stand-in model that returns the recorded counters of
  each configuration, so the scores depend only on KTT's scoring rule;
* ``weightedRandomSearchStep`` with its uniform draws fixed.

The output, ``profile_searcher_golden.json``, pins ktt::profiling (ProfileBasedSearcher.cpp) in
``tests/test_profile_searcher_cpu.py``.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _load_searcher_module(ktt_root: str):
    stub = types.ModuleType("pyktt")

    class Searcher:  # base class of PyProfilingSearcher
        def __init__(self):
            pass

    stub.Searcher = Searcher
    stub.KernelConfiguration = lambda: None
    sys.modules["pyktt"] = stub
    path = os.path.join(ktt_root, "Scripts", "ProfileBasedSearcher.py")
    spec = importlib.util.spec_from_file_location("ktt_profile_based_searcher", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


class _FixedRandom:
    def __init__(self, draws):
        self.draws = list(draws)

    def random(self):
        return self.draws.pop(0)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ktt-root", default=os.environ.get("KTT_ROOT"), required="KTT_ROOT" not in os.environ)
    args = ap.parse_args()
    mod = _load_searcher_module(args.ktt_root)
    meta = json.load(open(os.path.join(args.ktt_root, "Examples", "CoulombSum3d", "Models",
                                       "2080-coulomb_output_DT.sav.metadata.json")))
    g = json.load(open(os.path.join(HERE, "coulomb3d_2080_space.json")))
    names = ["Global size", "Local size"] + g["CounterNames"]

    def values_of(r):
        local = int(np.prod(r["LocalSize"]))
        return [float(np.prod(r["GlobalSize"]) * local), float(local)] + [float(v) for v in r["Counters"]]

    ok = [r for r in g["Results"] if r["Status"] == "Ok" and r["Counters"]]
    rng = np.random.default_rng(2021)
    picks = sorted(rng.choice(len(ok), size=12, replace=False).tolist())
    counter_sets = [{"source": "2080 Ti recorded: " + ",".join(f"{n}={v}" for n, v in ok[i]["Configuration"]),
                     "values": values_of(ok[i])} for i in picks]

    # synthetic B200-like sets: MUFU-bound (XU pipe saturated), FP32-bound, memory-bound, few threads
    base = dict(zip(names, values_of(ok[picks[0]])))
    for label, change in [
        ("xu bound", {"smsp__inst_executed_pipe_xu.avg.pct_of_peak_sustained_active": 92.0,
                      "smsp__issue_active.avg.pct_of_peak_sustained_active": 55.0}),
        ("fp32 bound", {"smsp__pipe_fma_cycles_active.avg.pct_of_peak_sustained_active": 95.0,
                        "smsp__issue_active.avg.pct_of_peak_sustained_active": 88.0,
                        "smsp__sass_thread_inst_executed_op_fp32_pred_on.sum":
                            base["smsp__inst_executed.sum"] * 32 * 0.9}),
        ("dram bound", {"dram__throughput.avg.pct_of_peak_sustained_elapsed": 91.0,
                        "dram__sectors_read.sum": 4.0e8, "dram__sectors_write.sum": 1.0e8}),
        ("few threads", {"Global size": 4096.0, "Local size": 128.0,
                         "sm__warps_active.avg.pct_of_peak_sustained_active": 12.0,
                         "smsp__cycles_active.avg.pct_of_peak_sustained_elapsed": 30.0}),
        ("integer and control", {"smsp__sass_thread_inst_executed_op_integer_pred_on.sum":
                                     base["smsp__inst_executed.sum"] * 32 * 0.8,
                                 "smsp__sass_thread_inst_executed_op_control_pred_on.sum":
                                     base["smsp__inst_executed.sum"] * 32 * 0.75,
                                 "smsp__issue_active.avg.pct_of_peak_sustained_active": 60.0}),
    ]:
        v = dict(base)
        v.update(change)
        counter_sets.append({"source": "synthetic: " + label, "values": [v[n] for n in names]})

    analysis = []
    for s in counter_sets:
        for mp, cores in [(68, 68 * 64), (148, 148 * 128)]:
            bn = mod.analyzeBottlenecks(names, s["values"], 10.0, mp, cores, 0)
            changes = mod.computeChanges(bn, meta["pc"], 10.0, 0)
            analysis.append({"source": s["source"], "multiprocessors": mp, "cores": cores, "values": s["values"],
                             "bottlenecks": {k: float(v) for k, v in bn.items()},
                             "changes": [float(c) for c in changes]})

    # scoring: candidates are recorded configurations; the stand-in model returns their recorded
    # counters (+ sizes + compilation data, in the model's counter order)
    tp = meta["tp"]
    order = [tp.index(n) for n, _ in ok[0]["Configuration"]]  # search-space order -> model order
    table = {}
    for r in ok:
        conf = {n: float(v) for n, v in r["Configuration"]}
        row = dict(zip(names, values_of(r)))
        cd = r["CompilationData"]
        row.update({"Maximum work-group size": cd["MaxWorkGroupSize"], "Local memory size": cd["LocalMemorySize"],
                    "Private memory size": cd["PrivateMemorySize"], "Constant memory size": cd["ConstantMemorySize"],
                    "Registers count": cd["RegistersCount"]})
        table[tuple(conf[n] for n in tp)] = [float(row[n]) for n in meta["pc"]]

    class TableModel:
        def predict(self, rows):
            return np.array([table[tuple(float(x) for x in row)] for row in rows])

    scoring = []
    for case in range(6):
        best = ok[int(rng.integers(len(ok)))]
        candidates = [ok[int(i)] for i in rng.choice(len(ok), size=25, replace=False)]
        best_conf = [float(v) for _, v in best["Configuration"]]
        cand_confs = [[float(v) for _, v in c["Configuration"]] for c in candidates]
        counters = analysis[(case % len(counter_sets)) * 2]
        previous = [1.0] * len(candidates)
        if case % 2:
            previous[3] = 0.0
        scores = mod.scoreTuningConfigurationsPredictor(list(counters["changes"]), order, best_conf, cand_confs,
                                                        list(previous), TableModel(), 0)
        actual = TableModel().predict([mod.reorderList(best_conf, order)])[0]
        predicted = TableModel().predict(mod.reorderTuningSpace(cand_confs, order))
        scoring.append({"changes": counters["changes"], "actual": [float(a) for a in actual],
                        "predicted": [[float(p) for p in row] for row in predicted], "previous": previous,
                        "scores": [float(s) for s in scores]})

    weighted = []
    for case in range(8):
        scores = [float(s) for s in rng.uniform(0.0, 1.0, 9) ** 8]
        if case == 7:
            scores = [0.0] * 9
        draw = float(rng.uniform())
        mod.random = _FixedRandom([draw])
        index = mod.weightedRandomSearchStep(list(scores), len(scores))
        weighted.append({"scores": scores, "u": draw, "index": int(index)})

    out = {
        "source": "Scripts/ProfileBasedSearcher.py (KTT 2.1.0) evaluated by tests/golden/make_profile_golden.py",
        "counter_names": names,
        "model_pc": meta["pc"],
        "analysis": analysis,
        "scoring": scoring,
        "weighted": weighted,
    }
    with open(os.path.join(HERE, "profile_searcher_golden.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))
        f.write("\n")
    print(f"wrote {len(analysis)} analyses, {len(scoring)} scorings, {len(weighted)} weighted draws")


if __name__ == "__main__":
    main()
