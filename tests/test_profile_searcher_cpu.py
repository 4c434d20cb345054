"""The profile-based searcher without a GPU.

* Its arithmetic (ktt::profiling) against KTT's own Python functions (golden vectors of
  tests/golden/make_profile_golden.py, evaluated on the recorded 2080 Ti counters and synthetic
  B200-like counter sets).
* The counter model: trained by ktt_b200/profile_model.py as KTT trains its model, written as JSON and
  evaluated by ktt::CounterModel, against scikit-learn's own predictions.
* The searcher end to end in simulated tuning over the recorded 2080 Ti search, including KTT's
  CoulombSum3dCudaScript.json run unchanged through the tuning-script loader (its model path resolved
  to the JSON forest trained from the same recording).
* The metric list KTT profiles by default, checked against the B200's chip (GB100) on the host.
"""
import ctypes
import json
import os
import shutil

import numpy as np
import pytest

from ktt_b200 import profile_model
from ktt_b200 import pyktt as ktt

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")
SCRIPTS = os.path.join(GOLDEN, "ktt_scripts")

ktt.Tuner.SetLoggingLevel(ktt.LoggingLevel.Error)


@pytest.fixture(scope="module")
def golden():
    return json.load(open(os.path.join(GOLDEN, "profile_searcher_golden.json")))


def _write_recorded(path, with_counters=True):
    """KTT-format result file of the recorded 2080 Ti search, counters and compilation data included."""
    g = json.load(open(os.path.join(GOLDEN, "coulomb3d_2080_space.json")))
    results = []
    for r in g["Results"]:
        cr = {"CompilationData": r["CompilationData"], "Duration": r["Duration"],
              "GlobalSize": dict(zip("XYZ", r["GlobalSize"])), "KernelFunction": "directCoulombSum",
              "LocalSize": dict(zip("XYZ", r["LocalSize"])), "Overhead": 0.0}
        if with_counters and r["Counters"]:
            cr["ProfilingData"] = {"Counters": [{"Name": n, "Type": "Double", "Value": v}
                                                for n, v in zip(g["CounterNames"], r["Counters"])],
                                   "RemainingProfilingRuns": 0}
        results.append({
            "ComputationResults": [cr],
            "Configuration": [{"Name": n, "Value": v, "ValueType": "UnsignedInt"} for n, v in r["Configuration"]],
            "DataMovementOverhead": 0.0, "ExtraDuration": 0.0, "KernelName": "CoulombSum", "SearcherOverhead": 0.0,
            "Status": r["Status"], "TotalDuration": r["TotalDuration"], "TotalOverhead": 0.0, "ValidationOverhead": 0.0})
    with open(path, "w") as f:
        json.dump({"Metadata": dict(g["Metadata"]), "Results": results}, f)
    return g


@pytest.fixture(scope="module")
def recorded(tmp_path_factory):
    d = tmp_path_factory.mktemp("profiled")
    path = d / "coulomb_2080_full_search_space.json"
    g = _write_recorded(path)
    model_path = d / "coulomb_2080.model.json"
    profile_model.main([str(path), "--out", str(model_path), "--cc", "7.5", "--multiprocessors", "68"])
    ok = [r for r in g["Results"] if r["Status"] == "Ok"]
    fastest = min(r["TotalDuration"] for r in ok)
    best = [{n: v for n, v in r["Configuration"]} for r in ok if r["TotalDuration"] == fastest]
    return str(path), str(model_path), g, best


# ---- arithmetic against KTT's Python ----------------------------------------------------------

def test_analysis_matches_ktt(golden):
    for case in golden["analysis"]:
        bn = ktt.profiling.AnalyzeBottlenecks(golden["counter_names"], case["values"], case["multiprocessors"],
                                              case["cores"])
        assert set(bn) == set(case["bottlenecks"]), case["source"]
        for k, v in case["bottlenecks"].items():
            assert bn[k] == pytest.approx(v, rel=1e-12, abs=1e-15), (case["source"], k)
        # KTT's computeChanges (no XU-pipe addition) against the shipped model's counter list
        changes = ktt.profiling.ComputeChanges(case["bottlenecks"], golden["model_pc"], False)
        np.testing.assert_allclose(changes, case["changes"], rtol=1e-12, atol=1e-15, err_msg=case["source"])


def test_xu_pipe_addition(golden):
    xu = [c for c in golden["analysis"] if c["source"] == "synthetic: xu bound"][0]
    assert xu["bottlenecks"]["bnSFU"] > 0.7
    pc = golden["model_pc"] + ["smsp__inst_executed_pipe_xu.sum"]
    plain = ktt.profiling.ComputeChanges(xu["bottlenecks"], pc, False)
    extended = ktt.profiling.ComputeChanges(xu["bottlenecks"], pc, True)
    assert plain[-1] == 0.0 and extended[-1] == pytest.approx(-xu["bottlenecks"]["bnSFU"])
    assert plain[:-1] == extended[:-1]


def test_scoring_matches_ktt(golden):
    for case in golden["scoring"]:
        scores = ktt.profiling.ScoreCandidates(case["changes"], case["actual"], case["predicted"], case["previous"])
        np.testing.assert_allclose(scores, case["scores"], rtol=1e-10, atol=1e-15)
        assert all(s == 0.0 for s, p in zip(scores, case["previous"]) if p == 0.0)


def test_weighted_step_matches_ktt(golden):
    for case in golden["weighted"]:
        assert ktt.profiling.WeightedRandomStep(case["scores"], case["u"]) == case["index"]


def test_cores_per_sm():
    assert ktt.profiling.CoresPerMultiprocessor(7, 5) == 64      # KTT's table (2080 Ti)
    assert ktt.profiling.CoresPerMultiprocessor(10, 0) == 128    # B200
    assert ktt.profiling.CoresPerMultiprocessor(1, 0) == 64      # unknown: KTT's default


# ---- counter model ----------------------------------------------------------------------------

def test_model_matches_sklearn(recorded, golden):
    path, model_path, g, _ = recorded
    tp, pc, x, y, device = profile_model.load_rows([path])
    assert device == "NVIDIA GeForce RTX 2080 Ti" and len(x) == sum(r["Status"] == "Ok" for r in g["Results"])
    # KTT's metadata order: the sizes, the 33 counters, the compilation data
    assert pc == golden["model_pc"]
    sk, train_r2, test_r2 = profile_model.train(x, y)
    assert train_r2 > 0.99 and test_r2 > 0.5
    model = ktt.CounterModel.Load(model_path)
    assert model.GetParameters() == tp and model.GetCounters() == pc
    assert model.GetComputeCapability() == 7.5 and model.GetMultiprocessors() == 68
    native = np.array([model.Predict(list(row)) for row in x])
    np.testing.assert_allclose(native, sk.predict(x), rtol=1e-12, atol=1e-9)


def test_model_rejects_other_files(tmp_path):
    bad = tmp_path / "model.json"
    bad.write_text(json.dumps({"format": "something else"}))
    with pytest.raises(Exception):
        ktt.CounterModel.Load(str(bad))


# ---- the searcher in simulated tuning -----------------------------------------------------------

def _space(tuner):
    d = tuner.AddKernelDefinition("directCoulombSum", "", ktt.DimensionVector(256, 256, 256), ktt.DimensionVector())
    k = tuner.CreateSimpleKernel("CoulombSum", d)
    for name, values in [("WORK_GROUP_SIZE_X", [16, 32]), ("WORK_GROUP_SIZE_Y", [1, 2, 4, 8]), ("WORK_GROUP_SIZE_Z", [1]),
                         ("Z_ITERATIONS", [1, 2, 4, 8, 16, 32]), ("INNER_UNROLL_FACTOR", [0, 1, 2, 4, 8, 16, 32]),
                         ("USE_CONSTANT_MEMORY", [0]), ("USE_SOA", [0, 1]), ("VECTOR_SIZE", [1])]:
        tuner.AddParameter(k, name, values)
    tuner.AddConstraint(k, ["INNER_UNROLL_FACTOR", "Z_ITERATIONS"], lambda v: v[0] < v[1])
    tuner.AddConstraint(k, ["WORK_GROUP_SIZE_X", "WORK_GROUP_SIZE_Y"], lambda v: v[0] * v[1] >= 64)
    return k


def _config(configuration):
    return {p.GetName(): int(p.GetValueString()) for p in configuration.GetPairs()}


def test_simulated_search_walks_the_space(recorded):
    path, model_path, _, best = recorded
    tuner = ktt.Tuner(0, 0, ktt.ComputeApi.CUDA)
    k = _space(tuner)
    searcher = ktt.ProfileBasedSearcher(tuner, ktt.CounterModel.Load(model_path), 10, 100, 10, 5)
    searcher.SetDeviceProperties(7, 5, 68)
    tuner.SetSearcher(k, searcher)
    results = tuner.SimulateTuning(k, tuner.LoadResults(path, ktt.OutputFormat.JSON))
    # every configuration once, plus one profiled rerun of each batch's fastest
    explored = {tuple(sorted(_config(r.GetConfiguration()).items())) for r in results}
    assert len(explored) == 210 and len(results) > 210
    assert _config(tuner.GetBestConfiguration(k)) in best
    assert not tuner.GetProfiling()  # switched off again after each profiled run


def test_simulated_search_scores_batches(recorded):
    path, model_path, _, _ = recorded
    tuner = ktt.Tuner(0, 0, ktt.ComputeApi.CUDA)
    k = _space(tuner)
    searcher = ktt.ProfileBasedSearcher(tuner, ktt.CounterModel.Load(model_path), 5, 100, 10, 11)
    tuner.SetSearcher(k, searcher)  # no device: the model's (2080 Ti, 68 SMs) is used
    results = tuner.SimulateTuning(k, tuner.LoadResults(path, ktt.OutputFormat.JSON), ktt.ConfigurationCount(60))
    assert len(results) == 60
    # batches of 5, then a profiled rerun of the batch's fastest
    runs = [tuple(sorted(_config(r.GetConfiguration()).items())) for r in results]
    reruns = [i for i in range(1, len(runs)) if runs[i] in runs[:i]]
    assert reruns == list(range(5, 60, 6))


def test_ktt_cuda_script_with_profile_based_searcher(recorded, tmp_path, monkeypatch):
    """Examples/CoulombSum3d/CoulombSum3dCudaScript.json unchanged: ProfileBased searcher, batch 10,
    model ../../Examples/CoulombSum3d/Models/2080-coulomb_output_DT.sav (relative to the working
    directory, as KTT passes it), replaying the recorded search."""
    path, model_path, _, best = recorded
    work = tmp_path / "build" / "run"
    work.mkdir(parents=True)
    shutil.copy(os.path.join(SCRIPTS, "CoulombSum3dCudaScript.json"), work)
    shutil.copy(path, work / "coulomb_2080_full_search_space.json")
    models = tmp_path / "Examples" / "CoulombSum3d" / "Models"
    models.mkdir(parents=True)
    shutil.copy(model_path, models / "2080-coulomb_output_DT.sav.json")
    monkeypatch.chdir(work)
    loader = ktt.TuningLoader()
    loader.LoadTuningFile(str(work / "CoulombSum3dCudaScript.json"))
    loader.ExecuteCommands()
    results = loader.GetResults()
    explored = {tuple(sorted(_config(r.GetConfiguration()).items())) for r in results}
    assert len(explored) == 210 and len(results) > 210
    fastest = min((r for r in results if r.IsValid()), key=lambda r: r.GetTotalDuration())
    assert _config(fastest.GetConfiguration()) in best


def test_results_file_round_trips_counters(recorded, tmp_path):
    path, _, g, _ = recorded
    tuner = ktt.Tuner(0, 0, ktt.ComputeApi.CUDA)
    loaded = tuner.LoadResults(path, ktt.OutputFormat.JSON)
    first = loaded[0].GetResults()[0]
    assert first.HasProfilingData() and first.GetProfilingData().IsValid()
    counters = first.GetProfilingData().GetCounters()
    assert [c.GetName() for c in counters] == g["CounterNames"]
    assert counters[0].GetType() == ktt.ProfilingCounterType.Double
    assert counters[0].GetValueDouble() == pytest.approx(g["Results"][0]["Counters"][0])
    out = tmp_path / "again"
    tuner.SaveResults(loaded, str(out), ktt.OutputFormat.JSON)
    again = tuner.LoadResults(str(out) + ".json", ktt.OutputFormat.JSON)
    c2 = again[0].GetResults()[0].GetProfilingData().GetCounters()
    assert [(c.GetName(), c.GetValueDouble()) for c in c2] == [(c.GetName(), c.GetValueDouble()) for c in counters]


def test_configuration_from_python_integers():
    tuner = ktt.Tuner(0, 0, ktt.ComputeApi.CUDA)
    k = _space(tuner)
    c = tuner.CreateConfiguration(k, [("WORK_GROUP_SIZE_X", 32), ("Z_ITERATIONS", 8)])
    assert _config(c)["WORK_GROUP_SIZE_X"] == 32 and _config(c)["Z_ITERATIONS"] == 8


# ---- the metric list on the B200's chip (host-side check, no GPU) -------------------------------

def test_default_metrics_on_gb100(golden):
    names = [n.encode() for n in golden["counter_names"][2:]]
    names.append(b"smsp__inst_executed_pipe_xu.sum")
    lib = ctypes.CDLL(os.path.join(REPO, "ktt_b200", "libcoulktt.so"))
    arr = (ctypes.c_char_p * len(names))(*names)
    valid = (ctypes.c_int * len(names))()
    rc = lib.coul_profiler_supported(b"GB100", arr, len(names), valid)
    if rc == 3:
        pytest.skip("libcupti is not installed here")
    assert rc == 0
    unsupported = [n.decode() for n, v in zip(names, valid) if not v]
    # the FP16-pipe instruction count is not offered by GB100; KTT drops such metrics with a warning
    assert unsupported == ["smsp__inst_executed_pipe_fp16.sum"]


# ---- a profiled search recorded on the B200 ------------------------------------------------------

def test_b200_recording_and_study():
    """The profiled 720-configuration search of this library's tile space recorded on a B200
    (tests/golden/make_b200_space.py): every configuration ran and carries KTT's counters minus the
    FP16-pipe count GB100 lacks, plus the XU-pipe count; the convergence study replays it through
    every searcher."""
    from ktt_b200 import run_searchers
    space = json.load(open(os.path.join(GOLDEN, "b200_map3d_space_64.json")))
    assert len(space["Results"]) == 720 and all(r["Status"] == "Ok" for r in space["Results"])
    assert "smsp__inst_executed_pipe_fp16.sum" not in space["CounterNames"]
    assert "smsp__inst_executed_pipe_xu.sum" in space["CounterNames"]
    report = run_searchers.main(["--seeds", "2", "--budget", "30"])
    for name in ("random", "mcmc", "profile"):
        assert 1.0 <= report[name]["best_ratio_after"][10] < 3.0
        assert report[name]["best_ratio_after"][80] <= report[name]["best_ratio_after"][10]


def test_xml_results_carry_counters(recorded, tmp_path):
    """KTT's XML output (Source/Output/XmlConverters.cpp:438-535): ProfilingData > Counters > Counter."""
    import xml.etree.ElementTree as ET
    path, _, g, _ = recorded
    tuner = ktt.Tuner(0, 0, ktt.ComputeApi.CUDA)
    loaded = tuner.LoadResults(path, ktt.OutputFormat.JSON)
    tuner.SaveResults(loaded[:3], str(tmp_path / "out"), ktt.OutputFormat.XML)
    root = ET.parse(tmp_path / "out.xml").getroot()
    counters = root.findall("./Results/Result/ComputationResults/ComputationResult/ProfilingData/Counters")
    assert len(counters) == 3
    first = counters[0].findall("Counter")
    assert [c.get("Name") for c in first] == g["CounterNames"]
    assert float(first[0].get("Value")) == pytest.approx(g["Results"][0]["Counters"][0])
