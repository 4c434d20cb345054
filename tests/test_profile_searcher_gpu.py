"""Hardware counters and the profile-based searcher on the B200.

A profiled tuner run collects KTT's default counters with CUPTI's range profiler (one replay of the
kernel per counter pass, before the timed run) and still validates; the autotuner records a profiled
search, trains the counter model from it (ktt_b200/profile_model.py, KTT's PrepareModels recipe) and
runs the profile-based searcher, which switches profiling on for one rerun per batch."""
import json

import numpy as np
import pytest

from ktt_b200 import autotune, profile_model
from ktt_b200 import pyktt as ktt

pytestmark = pytest.mark.gpu

ktt.Tuner.SetLoggingLevel(ktt.LoggingLevel.Error)

TILE = [("WORK_GROUP_SIZE_X", 32), ("WORK_GROUP_SIZE_Y", 4), ("Z_ITERATIONS", 8), ("X_POINTS", 2),
        ("INNER_UNROLL_FACTOR", 2), ("RSQRT_SOFT", 2)]


def kernel(tuner, grid, atoms):
    """directCoulombSum with KTT's nine arguments on a seeded uniform map of grid^3 points."""
    rng = np.random.default_rng(3)
    a = np.empty((atoms, 4), dtype=np.float32)
    a[:, :3] = rng.uniform(0.0, grid * 0.5, (atoms, 3))
    a[:, 3] = rng.uniform(-1.0, 1.0, atoms)
    tuner.SetGlobalSizeType(ktt.GlobalSizeType.CUDA)
    d = tuner.AddKernelDefinition("directCoulombSum", "", ktt.DimensionVector(grid, grid, grid), ktt.DimensionVector())
    k = tuner.CreateSimpleKernel("CoulombSum", d)
    ro = ktt.ArgumentAccessType.ReadOnly
    args = [tuner.AddArgumentVectorFloat(a.reshape(-1), ro)]
    args += [tuner.AddArgumentVectorFloat(np.ascontiguousarray(a[:, c]), ro) for c in range(4)]
    args += [tuner.AddArgumentScalarInt(atoms), tuner.AddArgumentScalarFloat(0.5), tuner.AddArgumentScalarInt(grid)]
    out = tuner.AddArgumentVectorFloat(np.zeros(grid ** 3, dtype=np.float32), ktt.ArgumentAccessType.WriteOnly)
    tuner.SetArguments(d, args + [out])
    return d, k, out


def test_profiled_run_collects_counters():
    grid, atoms = 64, 2048
    tuner = ktt.Tuner(0, 0, ktt.ComputeApi.CUDA)
    _, k, out = kernel(tuner, grid, atoms)
    for name, value in TILE:
        tuner.AddParameter(k, name, [value])
    config = tuner.CreateConfiguration(k, TILE)
    plain_map = np.zeros(grid ** 3, dtype=np.float32)
    plain = tuner.Run(k, config, [ktt.BufferOutputDescriptor(out, plain_map)])
    assert plain.IsValid() and not plain.GetResults()[0].HasProfilingData()
    tuner.SetProfiling(True)
    profiled_map = np.zeros(grid ** 3, dtype=np.float32)
    result = tuner.Run(k, config, [ktt.BufferOutputDescriptor(out, profiled_map)])
    tuner.SetProfiling(False)
    assert result.IsValid()
    # the passes run before the timed run, from reset arguments: the map is that of one run
    assert np.array_equal(profiled_map, plain_map)
    cr = result.GetResults()[0]
    assert cr.HasProfilingData() and cr.GetProfilingData().IsValid()
    counters = {c.GetName(): c.GetValueDouble() for c in cr.GetProfilingData().GetCounters()}
    assert "smsp__inst_executed_pipe_fp16.sum" not in counters  # not offered by GB100, dropped
    assert len(counters) >= 30
    assert counters["smsp__inst_executed.sum"] > 0
    assert 0 < counters["smsp__inst_executed_pipe_xu.avg.pct_of_peak_sustained_active"] <= 100
    assert 0 < counters["smsp__issue_active.avg.pct_of_peak_sustained_active"] <= 100
    assert counters["smsp__thread_inst_executed_per_inst_executed.ratio"] > 16
    # 6 of every 8 rsqrts run on MUFU (one XU instruction serves 32 lanes)
    pairs = grid ** 3 * atoms
    assert 0.5 * pairs * 6 / 8 / 32 < counters["smsp__inst_executed_pipe_xu.sum"] < 3.0 * pairs / 32
    assert result.GetProfilingRunsOverhead() > 0


def test_profile_based_search_on_device(tmp_path):
    recorded = tmp_path / "profiled_space.json"
    rec = autotune.tune_map3d(grid=64, atoms=2048, searcher="random", budget=24, profile=True,
                              results_path=str(recorded))
    assert all(t["profiled"] for t in rec["trials"])
    doc = json.load(open(recorded))
    assert len(doc["Results"]) == 24 and "ProfilingData" in doc["Results"][0]["ComputationResults"][0]
    model = tmp_path / "model.json"
    profile_model.main([str(recorded), "--out", str(model)])
    result = autotune.tune_map3d(grid=64, atoms=2048, searcher="profile", budget=18, model=str(model), seed=3)
    trials = result["trials"]
    assert len(trials) == 18 and all(t["status"] == "Ok" for t in trials)
    # batches of 5 followed by a profiled rerun of the batch's fastest
    assert [i for i, t in enumerate(trials) if t["profiled"]] == [5, 11, 17]
