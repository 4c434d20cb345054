"""The pyktt module (KTT's Python API names over the ktt:: surface) without a GPU: KTT's
CoulombSum3d configuration space built from Python (parameters, Python-callable constraints and
thread modifiers) against the recorded 2080 Ti space; simulated tuning over the recorded results
with each searcher and with a stop condition written in Python; KTT's invalid-id convention; the
JSON tuning-script loader driven from Python."""
import json
import os
import shutil

import pytest

from ktt_b200 import pyktt as ktt

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")

ktt.Tuner.SetLoggingLevel(ktt.LoggingLevel.Error)


def _space(tuner):
    d = tuner.AddKernelDefinition("directCoulombSum", "", ktt.DimensionVector(256, 256, 256), ktt.DimensionVector())
    k = tuner.CreateSimpleKernel("CoulombSum", d)
    # the parameters and constraints of Examples/CoulombSum3d/CoulombSum3d.cpp:137-216 (CUDA build)
    tuner.AddParameter(k, "WORK_GROUP_SIZE_X", [16, 32])
    tuner.AddParameter(k, "WORK_GROUP_SIZE_Y", [1, 2, 4, 8])
    tuner.AddParameter(k, "WORK_GROUP_SIZE_Z", [1])
    tuner.AddParameter(k, "Z_ITERATIONS", [1, 2, 4, 8, 16, 32])
    tuner.AddParameter(k, "INNER_UNROLL_FACTOR", [0, 1, 2, 4, 8, 16, 32])
    tuner.AddParameter(k, "USE_CONSTANT_MEMORY", [0])
    tuner.AddParameter(k, "USE_SOA", [0, 1])
    tuner.AddParameter(k, "VECTOR_SIZE", [1])
    tuner.AddThreadModifier(k, [d], ktt.ModifierType.Local, ktt.ModifierDimension.X, "WORK_GROUP_SIZE_X",
                            ktt.ModifierAction.Multiply)
    tuner.AddThreadModifier(k, [d], ktt.ModifierType.Global, ktt.ModifierDimension.Z, ["Z_ITERATIONS"],
                            lambda size, values: (size + values[0] - 1) // values[0])
    tuner.AddConstraint(k, ["INNER_UNROLL_FACTOR", "Z_ITERATIONS"], lambda v: v[0] < v[1])
    tuner.AddConstraint(k, ["WORK_GROUP_SIZE_X", "WORK_GROUP_SIZE_Y"], lambda v: v[0] * v[1] >= 64)
    return d, k


@pytest.fixture(scope="module")
def recorded(tmp_path_factory):
    d = tmp_path_factory.mktemp("rec")
    g = json.load(open(os.path.join(GOLDEN, "coulomb3d_2080_space.json")))
    results = []
    for r in g["Results"]:
        results.append({
            "ComputationResults": [{"CompilationData": {}, "Duration": r["Duration"],
                                    "GlobalSize": dict(zip("XYZ", r["GlobalSize"])), "KernelFunction": "directCoulombSum",
                                    "LocalSize": dict(zip("XYZ", r["LocalSize"])), "Overhead": 0.0}],
            "Configuration": [{"Name": n, "Value": v, "ValueType": "UnsignedInt"} for n, v in r["Configuration"]],
            "DataMovementOverhead": 0.0, "ExtraDuration": 0.0, "KernelName": "CoulombSum", "SearcherOverhead": 0.0,
            "Status": r["Status"], "TotalDuration": r["TotalDuration"], "TotalOverhead": 0.0, "ValidationOverhead": 0.0})
    path = d / "coulomb_2080_full_search_space.json"
    json.dump({"Metadata": dict(g["Metadata"]), "Results": results}, open(path, "w"))
    ok = [r for r in g["Results"] if r["Status"] == "Ok"]
    fastest = min(r["TotalDuration"] for r in ok)
    # the recording has a tie for the fastest time (WORK_GROUP_SIZE_Y 2 and 4)
    best = [{n: v for n, v in r["Configuration"]} for r in ok if r["TotalDuration"] == fastest]
    return str(path), g, best


def _config_dict(configuration):
    return {p.GetName(): int(p.GetValueString()) for p in configuration.GetPairs()}


def test_space_matches_recorded(recorded):
    _, g, _ = recorded
    tuner = ktt.Tuner(0, 0, ktt.ComputeApi.CUDA)
    _, k = _space(tuner)
    assert tuner.GetConfigurationsCount(k) == len(g["Results"]) == 210


@pytest.mark.parametrize("searcher", ["DeterministicSearcher", "RandomSearcher", "McmcSearcher"])
def test_simulated_tuning_finds_recorded_best(recorded, searcher):
    path, g, best = recorded
    tuner = ktt.Tuner(0, 0, ktt.ComputeApi.CUDA)
    _, k = _space(tuner)
    tuner.SetSearcher(k, getattr(ktt, searcher)())
    results = tuner.SimulateTuning(k, tuner.LoadResults(path, ktt.OutputFormat.JSON))
    assert len(results) == 210  # no stop condition: the whole space is walked
    fastest = min((r for r in results if r.IsValid()), key=lambda r: r.GetTotalDuration())
    assert _config_dict(fastest.GetConfiguration()) in best
    assert _config_dict(tuner.GetBestConfiguration(k)) in best


def test_python_stop_condition(recorded):
    path, _, _ = recorded

    class FirstValid(ktt.StopCondition):
        def __init__(self):
            super().__init__()
            self.seen = 0
            self.valid = False

        def IsFulfilled(self):
            return self.valid

        def Initialize(self, count):
            self.seen = 0

        def Update(self, result):
            self.seen += 1
            self.valid = result.IsValid()

        def GetStatusString(self):
            return f"stopped after {self.seen}"

    tuner = ktt.Tuner(0, 0, ktt.ComputeApi.CUDA)
    _, k = _space(tuner)
    results = tuner.SimulateTuning(k, tuner.LoadResults(path, ktt.OutputFormat.JSON), FirstValid())
    assert len(results) == 1 and results[0].IsValid()
    results = tuner.SimulateTuning(k, tuner.LoadResults(path, ktt.OutputFormat.JSON), ktt.ConfigurationCount(7))
    assert len(results) == 7


def test_invalid_ids_and_arguments():
    tuner = ktt.Tuner(0, 0, ktt.ComputeApi.CUDA)
    assert tuner.CreateSimpleKernel("x", 12345) == ktt.InvalidKernelId
    a = tuner.AddArgumentVectorFloat([1.0, 2.0, 3.0], ktt.ArgumentAccessType.ReadOnly, "atoms")
    assert a == "atoms"
    assert tuner.AddArgumentVectorFloat([1.0], ktt.ArgumentAccessType.ReadOnly, "atoms") == ktt.InvalidArgumentId
    assert tuner.AddArgumentScalarInt(64) != ktt.InvalidArgumentId
    g = tuner.AddArgumentVectorFromGenerator("i * 0.5", ktt.ArgumentDataType.Float, 16, 4, ktt.ArgumentAccessType.ReadOnly)
    assert g != ktt.InvalidArgumentId


def test_platform_and_device_info_without_a_device():
    """Tutorials/01ComputeApiInfo: one CUDA platform; with no device (this machine) an empty device
    list, and KTT's GetString layout for both descriptions."""
    tuner = ktt.Tuner(0, 0, ktt.ComputeApi.CUDA)
    platforms = tuner.GetPlatformInfo()
    assert len(platforms) == 1
    p = platforms[0]
    assert (p.GetIndex(), p.GetName(), p.GetVendor()) == (0, "NVIDIA CUDA", "NVIDIA Corporation")
    assert p.GetString().splitlines() == [
        "Information about platform with index: 0", "Name: NVIDIA CUDA", "Vendor: NVIDIA Corporation",
        f"Compute API version: {p.GetVersion()}", "Extensions: N/A"]
    assert tuner.GetDeviceInfo(0) == []
    assert tuner.GetDeviceInfo(3) == []  # no such platform: logged, empty
    d = ktt.DeviceInfo(2, "B200")
    d.SetVendor("NVIDIA Corporation")
    d.SetDeviceType(ktt.DeviceType.GPU)
    d.SetGlobalMemorySize(1 << 30)
    d.SetMaxWorkGroupSize(1024)
    d.SetMaxComputeUnits(148)
    d.SetCudaComputeCapabilityMajor(10)
    lines = d.GetString().splitlines()
    assert lines[0] == "Information about device with index: 2" and "Device type: GPU" in lines
    assert "Maximum work-group size: 1024" in lines and "Maximum parallel compute units: 148" in lines
    assert lines[-1] == "CUDA compute capability: 10.0"


def test_local_symbol_arguments_and_profiled_definitions():
    tuner = ktt.Tuner(0, 0, ktt.ComputeApi.CUDA)
    assert tuner.AddArgumentLocalFloat(1024, "lm") == "lm"
    assert tuner.AddArgumentLocalFloat(0) == ktt.InvalidArgumentId
    assert tuner.AddArgumentSymbolInt(7, symbolName="cSize", customId="sym") == "sym"
    d1, k = _space(tuner)
    d2 = tuner.AddKernelDefinition("second", "", ktt.DimensionVector(16), ktt.DimensionVector(16))
    tuner.SetProfiledDefinitions(k, [d1])  # part of the kernel: accepted silently
    tuner.SetProfiledDefinitions(k, [d2])  # not part of it: logged, kept as before
    c = tuner.CreateCompositeKernel("pair", [d1, d2])
    tuner.SetProfiledDefinitions(c, [d2])
    tuner.SetArguments(d1, ["lm"])  # local memory goes last; the argument list is accepted


def test_queues_of_a_tuner():
    """Only a tuner made from a ComputeApiInitializer takes further queues; ids follow the
    initializer's order, duplicates and the last queue are refused (logged, no exception).  The
    handles here are never used: no call below creates the device context."""
    plain = ktt.Tuner(0, 0, ktt.ComputeApi.CUDA)
    assert plain.AddComputeQueue(0x1000) == ktt.InvalidQueueId
    with pytest.raises(Exception):
        ktt.Tuner(ktt.ComputeApi.CUDA, ktt.ComputeApiInitializer(0, [0x2000]))
    init = ktt.ComputeApiInitializer(0xC000, [0x2000, 0x3000])
    assert init.GetContext() == 0xC000 and init.GetQueues() == [0x2000, 0x3000]
    tuner = ktt.Tuner(ktt.ComputeApi.CUDA, init)
    assert tuner.AddComputeQueue(0x4000) == 2
    assert tuner.AddComputeQueue(0x3000) == ktt.InvalidQueueId  # already a queue
    tuner.RemoveComputeQueue(1)
    tuner.RemoveComputeQueue(7)  # unknown id: logged
    assert tuner.AddComputeQueue(0x5000) == 3


def test_python_launchers_get_the_compute_interface():
    """SetLauncher and CreateCompositeKernel take Python launchers; they are handed the tuner's
    ComputeInterface (queues, configuration) without a copy.  These launchers launch nothing, so
    the runs need no device."""
    tuner = ktt.Tuner(0, 0, ktt.ComputeApi.CUDA)
    d = tuner.AddKernelDefinition("noop", "", ktt.DimensionVector(32), ktt.DimensionVector(32))
    k = tuner.CreateSimpleKernel("k", d)
    tuner.AddParameter(k, "P", [1, 2])
    seen = []

    def launcher(ci):
        seen.append((list(ci.GetAllQueues()), ci.GetDefaultQueue(), ci.GetCurrentConfiguration().GetString()))

    tuner.SetLauncher(k, launcher)
    assert tuner.Run(k, tuner.CreateConfiguration(k, [("P", 2)]), []).GetStatus() == ktt.ResultStatus.Ok
    c = tuner.CreateCompositeKernel("c", [d], launcher)
    assert tuner.Run(c, tuner.CreateConfiguration(c, []), []).GetStatus() == ktt.ResultStatus.Ok
    assert seen == [([0], 0, "P 2"), ([0], 0, "empty")]


def test_tuning_loader_from_python(tmp_path, recorded):
    path, _, best = recorded
    shutil.copy(os.path.join(GOLDEN, "ktt_scripts", "CoulombSum3dCudaScript.json"), tmp_path)
    shutil.copy(path, tmp_path)
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        loader = ktt.TuningLoader()
        loader.LoadTuningFile(str(tmp_path / "CoulombSum3dCudaScript.json"))
        loader.ExecuteCommands()
    finally:
        os.chdir(cwd)
    results = loader.GetResults()
    assert len(results) == 210
    fastest = min((r for r in results if r.IsValid()), key=lambda r: r.GetTotalDuration())
    assert _config_dict(fastest.GetConfiguration()) in best
    assert loader.GetTuner().GetConfigurationsCount(loader.GetKernelId()) == 210
