"""Compact fixture of a profiled search over this library's own tile space on a B200.

The raw recording is made on a B200 with

    python -m ktt_b200.autotune map3d --grid 64 --atoms 2048 --searcher deterministic --budget 720 \
        --profile --results b200_space_64.json

(every configuration of the 720-configuration directCoulombSum space of ktt_b200/autotune.py on a
64^3 map of 2048 seeded uniform atoms, each run once for its time and replayed for KTT's default
counters) and converted here, from the repository root:

    python tests/golden/make_b200_space.py b200_space_64.json [64]

into ``b200_map3d_space_64.json`` next to this script (``b200_map3d_space_128.json`` from the same
command with --grid 128 --atoms 4096, converted with a second argument 128): the metadata, the counter names once, and per
configuration its parameters, status, kernel duration (ms), launch grid and block, and counter values
(7 significant digits).  tests/test_profile_searcher_cpu.py replays it through the profile-based
searcher and the other searchers without a GPU.
"""
from __future__ import annotations

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(path: str, grid: str = "64") -> None:
    d = json.load(open(path))
    names = [c["Name"] for c in d["Results"][0]["ComputationResults"][0]["ProfilingData"]["Counters"]]
    results = []
    for r in d["Results"]:
        cr = r["ComputationResults"][0]
        values = {c["Name"]: c["Value"] for c in cr.get("ProfilingData", {}).get("Counters", [])}
        results.append({
            "Configuration": [[p["Name"], p["Value"]] for p in r["Configuration"]],
            "Status": r["Status"],
            "Duration": cr["Duration"],
            "GlobalSize": [cr["GlobalSize"][k] for k in "XYZ"],
            "LocalSize": [cr["LocalSize"][k] for k in "XYZ"],
            "Counters": [float(f"{values[n]:.7g}") if values.get(n) is not None else None for n in names],
        })
    atoms = {"64": 2048, "128": 4096}[grid]
    out = {"source": f"python -m ktt_b200.autotune map3d --grid {grid} --atoms {atoms} --searcher deterministic "
                     "--budget 720 --profile (B200)",
           "Metadata": d["Metadata"], "CounterNames": names, "Results": results}
    with open(os.path.join(HERE, f"b200_map3d_space_{grid}.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))
        f.write("\n")
    print(f"{len(results)} configurations, {len(names)} counters")


if __name__ == "__main__":
    main(*sys.argv[1:3])
