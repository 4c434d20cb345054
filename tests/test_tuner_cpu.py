"""CPU tests of the C++ ktt:: surface (libktt_b200.so): configuration space against KTT's recorded
2080 Ti search space, searchers through simulated tuning, stop conditions, result files, error
convention.  The test program tests/cpp/tuner_cpu_tests.cpp is compiled here against the public
headers in include/ and the built library."""
import json
import os
import shutil
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")


def _cxx():
    return shutil.which("g++") or "g++"


@pytest.fixture(scope="session")
def cpu_tests_binary(tmp_path_factory):
    from ktt_b200 import build as kb
    kb.build()
    out = tmp_path_factory.mktemp("cpp") / "tuner_cpu_tests"
    lib = os.path.join(REPO, "ktt_b200")
    subprocess.run([_cxx(), "-std=c++17", "-O1", "-Wall", "-I", os.path.join(REPO, "include"),
                    os.path.join(REPO, "tests", "cpp", "tuner_cpu_tests.cpp"), "-o", str(out), "-L", lib,
                    "-lktt_b200", "-lcoulktt", f"-Wl,-rpath,{lib}"], check=True)
    return str(out)


@pytest.fixture(scope="session")
def workdir(tmp_path_factory):
    """KTT-format result file of the recorded 2080 Ti search (from the committed golden fixture)."""
    d = tmp_path_factory.mktemp("ktt")
    g = json.load(open(os.path.join(GOLDEN, "coulomb3d_2080_space.json")))
    results = []
    for r in g["Results"]:
        results.append({
            "ComputationResults": [{
                "CompilationData": {}, "Duration": r["Duration"],
                "GlobalSize": dict(zip("XYZ", r["GlobalSize"])), "KernelFunction": "directCoulombSum",
                "LocalSize": dict(zip("XYZ", r["LocalSize"])), "Overhead": 0.0}],
            "Configuration": [{"Name": n, "Value": v, "ValueType": "UnsignedInt"} for n, v in r["Configuration"]],
            "DataMovementOverhead": 0.0, "ExtraDuration": 0.0, "KernelName": "CoulombSum", "SearcherOverhead": 0.0,
            "Status": r["Status"], "TotalDuration": r["TotalDuration"], "TotalOverhead": 0.0,
            "ValidationOverhead": 0.0})
    doc = {"Metadata": dict(g["Metadata"]), "Results": results}
    with open(d / "coulomb_2080_ktt_format.json", "w") as f:
        json.dump(doc, f)
    return str(d)


@pytest.mark.parametrize("name", ["prefix", "space", "subgroup_order", "groups", "neighbours", "deterministic",
                                  "random", "mcmc", "stop", "json", "errors"])
def test_tuner_cpu(cpu_tests_binary, workdir, name):
    r = subprocess.run([cpu_tests_binary, name, GOLDEN, workdir], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr


def test_prefix_golden_matches_reference_test():
    g = json.load(open(os.path.join(GOLDEN, "ktt_prefix.json")))
    assert g["expected"] == "#define param_two 5\n#define param_one 2\n"
    assert g["pairs"] == [["param_two", 5], ["param_one", 2]]


def test_gpu_programs_compile(tmp_path):
    """The GPU test programs build against the public headers (they run in test_tuner_gpu.py)."""
    from ktt_b200 import build as kb
    kb.build()
    lib = os.path.join(REPO, "ktt_b200")
    subprocess.run([_cxx(), "-std=c++17", "-O1", "-Wall", "-I", os.path.join(REPO, "include"),
                    os.path.join(REPO, "tests", "cpp", "tuner_gpu_tests.cpp"), "-o", str(tmp_path / "t"), "-L", lib,
                    "-lktt_b200", "-lcoulktt", f"-Wl,-rpath,{lib}"], check=True)
