"""Counter model of the profile-based searcher, trained from results that carry profiling counters.

    python -m ktt_b200.profile_model RESULTS.json [MORE.json ...] --out MODEL.json [--cc 10.0] [--multiprocessors 148]

KTT trains its model with Scripts/PrepareModels/generate_decision_tree_model.py: the tuning
parameters of every profiled configuration are the features, its counters ("Global size",
"Local size", the CUPTI counters, then the compilation data) the targets, half of the rows
(train_test_split(test_size=0.5, random_state=7)) fit an ExtraTreesRegressor(n_estimators=10,
random_state=0), and the model is pickled next to a metadata file naming the parameters ("tp"),
counters ("pc") and compute capability ("cc").  This module trains the same forest with the same
split and writes it as JSON (format "ktt_b200.counter_forest/1": tp, pc, cc, multiprocessors and per
tree its node arrays feature / threshold / left / right / value, value given on leaves) for
ktt::CounterModel (include/ktt/ProfileBasedSearcher.h), which evaluates it in C++; nothing is pickled.

RESULTS are KTT-format JSON result files (Tuner::SaveResults; KTT's own recorded files load as they
are).  Only computations with status Ok and profiling counters are used.
"""
from __future__ import annotations

import argparse
import json
import sys

import numpy as np

FORMAT = "ktt_b200.counter_forest/1"
# KTT's names of the compilation-data columns (its CSV output and model metadata)
COMPILATION_COLUMNS = [("MaxWorkGroupSize", "Maximum work-group size"), ("LocalMemorySize", "Local memory size"),
                       ("PrivateMemorySize", "Private memory size"), ("ConstantMemorySize", "Constant memory size"),
                       ("RegistersCount", "Registers count")]


def _size(d) -> int:
    return int(d.get("X", 1)) * int(d.get("Y", 1)) * int(d.get("Z", 1))


def load_rows(paths):
    """(tp, pc, X, Y, device): one row per valid profiled result, columns in KTT's order."""
    tp, names, rows_x, rows_y, device = None, None, [], [], ""
    compilation = None
    for path in paths:
        with open(path) as f:
            doc = json.load(f)
        device = device or doc.get("Metadata", {}).get("Device", "")
        for r in doc.get("Results", []):
            if r.get("Status") != "Ok" or not r.get("ComputationResults"):
                continue
            cr = r["ComputationResults"][0]
            counters = cr.get("ProfilingData", {}).get("Counters", [])
            if not counters:
                continue
            params = [(p["Name"], float(p["Value"])) for p in r["Configuration"]]
            if tp is None:
                tp = [n for n, _ in params]
                names = [c["Name"] for c in counters]
                compilation = [k for k, _ in COMPILATION_COLUMNS if k in cr.get("CompilationData", {})]
            values = {c["Name"]: c["Value"] for c in counters}
            if [n for n, _ in params] != tp or any(n not in values for n in names):
                raise ValueError(f"{path}: results differ in their parameters or counters")
            local = _size(cr["LocalSize"])
            # "Global size" in threads: the recorded grid (blocks) times the block, as the searcher computes it
            y = [float(_size(cr["GlobalSize"]) * local), float(local)]
            y += [float("nan") if values[n] is None else float(values[n]) for n in names]
            y += [float(cr["CompilationData"][k]) for k in compilation]
            rows_x.append([v for _, v in params])
            rows_y.append(y)
    if tp is None:
        raise ValueError("no result with status Ok and profiling counters")
    pc = ["Global size", "Local size"] + names + [dict(COMPILATION_COLUMNS)[k] for k in compilation]
    return tp, pc, np.array(rows_x, dtype=np.float64), np.array(rows_y, dtype=np.float64), device


def train(x, y, test_size: float = 0.5, split_seed: int = 7, seed: int = 0, trees: int = 10):
    """KTT's estimator and split (generate_decision_tree_model.py:54-55, 85, 92); returns (model, train R^2, test R^2)."""
    from sklearn.ensemble import ExtraTreesRegressor
    from sklearn.model_selection import train_test_split
    y = np.nan_to_num(y, nan=0.0)
    if len(x) >= 4:
        x_train, x_test, y_train, y_test = train_test_split(x, y, test_size=test_size, random_state=split_seed)
    else:
        x_train, x_test, y_train, y_test = x, x, y, y
    model = ExtraTreesRegressor(n_estimators=trees, random_state=seed)
    model.fit(x_train, y_train)
    return model, float(model.score(x_train, y_train)), float(model.score(x_test, y_test))


def export(model, tp, pc, cc: float, multiprocessors: int) -> dict:
    trees = []
    for est in model.estimators_:
        t = est.tree_
        leaf = t.children_left == -1
        value = t.value.reshape(t.node_count, -1)  # (nodes, outputs) for a regressor
        trees.append({
            "feature": [-1 if leaf[i] else int(t.feature[i]) for i in range(t.node_count)],
            "threshold": [0.0 if leaf[i] else float(t.threshold[i]) for i in range(t.node_count)],
            "left": [int(v) for v in t.children_left],
            "right": [int(v) for v in t.children_right],
            "value": [[float(v) for v in value[i]] if leaf[i] else [] for i in range(t.node_count)],
        })
    return {"format": FORMAT, "cc": cc, "multiprocessors": multiprocessors, "tp": list(tp), "pc": list(pc),
            "trees": trees}


def main(argv=None) -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("results", nargs="+")
    ap.add_argument("--out", required=True)
    ap.add_argument("--cc", type=float, default=10.0, help="compute capability of the profiled device")
    ap.add_argument("--multiprocessors", type=int, default=148, help="SM count of the profiled device")
    args = ap.parse_args(argv)
    tp, pc, x, y, device = load_rows(args.results)
    model, train_score, test_score = train(x, y)
    doc = export(model, tp, pc, args.cc, args.multiprocessors)
    doc["source"] = {"results": [str(p) for p in args.results], "device": device, "rows": int(len(x)),
                     "train_r2": train_score, "test_r2": test_score}
    with open(args.out, "w") as f:
        json.dump(doc, f, separators=(",", ":"))
        f.write("\n")
    print(json.dumps({"out": str(args.out), "rows": int(len(x)), "parameters": len(tp), "counters": len(pc),
                      "train_r2": round(train_score, 4), "test_r2": round(test_score, 4)}), file=sys.stderr)


if __name__ == "__main__":
    main()
