"""Generate the committed golden fixtures from the KTT 2.1.0 source tree.

Run from the repository root, in a container where the KTT tree is mounted:

    python tests/golden/make_golden.py --ktt-root KTT_TREE   (or KTT_ROOT=KTT_TREE in the environment)

It writes, next to this script:

* ``coulomb3d_kat.json`` -- KTT's known-answer test for the Coulomb path.
  ``make -C oracle ref`` compiles ``Examples/JSON/generate-coulomb-output.c``
  from the KTT tree into ``oracle/_ref/`` and runs it; the resulting 256^3 FP32
  map ``Coulomb3d.bin`` (the file ``Examples/JSON/CoulombSum3d.json:172-181``
  validates against, threshold 0.01) is summarised here: sha256, min/max/mean,
  and the exact FP32 bit patterns of 4096 seeded sample points plus the argmin
  and argmax points.
* ``coulomb3d_2080_space.json`` -- the 210 configurations of KTT's full CUDA
  search space for ``directCoulombSum`` as measured on an RTX 2080 Ti
  (``Examples/CoulombSum3d/coulomb_2080_full_search_space.json``): each
  configuration's parameter values, status, kernel duration, total duration,
  global/local sizes, its 33 profiling counters and compilation data.  Used to pin the
  configuration-space enumeration (parameters + constraints of
  ``Examples/CoulombSum3d/CoulombSum3d.cpp:137-216``), to drive searchers
  in simulated tuning without a GPU, and to train the profile-based searcher's
  counter model as KTT trained its shipped one
  (``Examples/CoulombSum3d/Models/2080-coulomb_output_DT.sav`` is a pickle and is
  not read).
* ``ktt_prefix.json`` -- the configuration -> ``#define`` prefix expectation of
  ``Tests/KernelManagerTests.cpp:57-81``.
* ``ktt_scripts/`` -- KTT's two JSON tuning scripts for this path, parsed and
  written back unchanged in content: ``Examples/JSON/CoulombSum3d.json`` (the
  known-answer run: generated atoms, validated against ``Coulomb3d.bin`` at 0.01)
  and ``Examples/CoulombSum3d/CoulombSum3dCudaScript.json`` (simulated tuning
  over the recorded 2080 Ti results), with ``manifest.json`` naming each
  source file and its sha256.  The tuning-script loader's tests run them.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import re
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def kat(ktt_root: str) -> None:
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "ref", f"KTT_ROOT={ktt_root}"], check=True)
    path = os.path.join(REPO, "oracle", "_ref", "Coulomb3d.bin")
    raw = open(path, "rb").read()
    grid = np.frombuffer(raw, dtype=np.float32)
    assert grid.size == 256 ** 3
    rng = np.random.default_rng(20240812)
    idx = np.sort(rng.choice(grid.size, size=4096, replace=False)).astype(np.int64)
    extra = np.array([int(np.argmin(grid)), int(np.argmax(grid)), 0, grid.size - 1], dtype=np.int64)
    idx = np.unique(np.concatenate([idx, extra]))
    out = {
        "source": "Examples/JSON/generate-coulomb-output.c (KTT 2.1.0), compiled by oracle/Makefile target 'ref'",
        "cells": 256,
        "atoms": 64,
        "grid_spacing_f32": float(np.float32(0.49)),
        "validation_threshold": 0.01,
        "sha256": hashlib.sha256(raw).hexdigest(),
        "min": float(grid.min()),
        "max": float(grid.max()),
        "mean": float(grid.astype(np.float64).mean()),
        "argmin": int(np.argmin(grid)),
        "argmax": int(np.argmax(grid)),
        "index": idx.tolist(),
        "bits": grid[idx].view(np.uint32).tolist(),
    }
    with open(os.path.join(HERE, "coulomb3d_kat.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))


def space_2080(ktt_root: str) -> None:
    src = os.path.join(ktt_root, "Examples", "CoulombSum3d", "coulomb_2080_full_search_space.json")
    d = json.load(open(src))
    results = []
    # every counter, in the recorded order (the profile-based searcher and its model read them all);
    # names once, values per result
    names = [c["Name"] for c in d["Results"][0]["ComputationResults"][0]["ProfilingData"]["Counters"]]
    for r in d["Results"]:
        cr = r["ComputationResults"][0]
        recorded = {c["Name"]: c["Value"] for c in cr.get("ProfilingData", {}).get("Counters", [])}
        counters = [recorded[n] for n in names] if recorded else []
        results.append({
            "Configuration": [[p["Name"], p["Value"]] for p in r["Configuration"]],
            "Status": r["Status"],
            "TotalDuration": r["TotalDuration"],
            "Duration": cr["Duration"],
            "GlobalSize": [cr["GlobalSize"]["X"], cr["GlobalSize"]["Y"], cr["GlobalSize"]["Z"]],
            "LocalSize": [cr["LocalSize"]["X"], cr["LocalSize"]["Y"], cr["LocalSize"]["Z"]],
            "Counters": counters,
            "CompilationData": cr.get("CompilationData", {}),
        })
    out = {
        "source": "Examples/CoulombSum3d/coulomb_2080_full_search_space.json (KTT 2.1.0)",
        "Metadata": d["Metadata"],
        "problem": {"gridSize": 256, "atoms": 64, "gridSpacing": 0.5},
        "CounterNames": names,
        "Results": results,
    }
    with open(os.path.join(HERE, "coulomb3d_2080_space.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))
        f.write("\n")


def prefix(ktt_root: str) -> None:
    src = open(os.path.join(ktt_root, "Tests", "KernelManagerTests.cpp")).read()
    m = re.search(r'expectedPrefix\("([^"]*)"\)', src)
    assert m, "prefix expectation not found"
    pairs = re.findall(r'parameterPairs\.emplace_back\("(\w+)", static_cast<uint64_t>\((\d+)\)\)', src)
    out = {
        "source": "Tests/KernelManagerTests.cpp:57-81 (KTT 2.1.0)",
        "pairs": [[n, int(v)] for n, v in pairs],
        "expected": m.group(1).encode().decode("unicode_escape"),
    }
    with open(os.path.join(HERE, "ktt_prefix.json"), "w") as f:
        json.dump(out, f, indent=1)


def scripts(ktt_root: str) -> None:
    out_dir = os.path.join(HERE, "ktt_scripts")
    os.makedirs(out_dir, exist_ok=True)
    manifest = {}
    for rel in ("Examples/JSON/CoulombSum3d.json", "Examples/CoulombSum3d/CoulombSum3dCudaScript.json"):
        raw = open(os.path.join(ktt_root, rel), "rb").read()
        doc = json.loads(raw)
        name = os.path.basename(rel)
        with open(os.path.join(out_dir, name), "w") as f:
            json.dump(doc, f, indent=1)
            f.write("\n")
        manifest[name] = {"source": rel + " (KTT 2.1.0)", "sha256": hashlib.sha256(raw).hexdigest()}
    with open(os.path.join(out_dir, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1)
        f.write("\n")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ktt-root", default=os.environ.get("KTT_ROOT"), required="KTT_ROOT" not in os.environ)
    args = ap.parse_args()
    kat(args.ktt_root)
    space_2080(args.ktt_root)
    prefix(args.ktt_root)
    scripts(args.ktt_root)


if __name__ == "__main__":
    main()
