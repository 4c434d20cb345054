"""GPU tests of the C++ ktt:: surface: KTT-style host programs for the Coulomb path (3D with the
full KTT space and reference-kernel validation, FP64 reference computation, 2D random search, the
iterative slice launcher, caller-owned device buffers), run against the sm_100a kernels."""
import os
import subprocess

import pytest

from test_tuner_cpu import REPO, _cxx, workdir  # noqa: F401  (fixture re-export)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="session")
def gpu_tests_binary(tmp_path_factory):
    from ktt_b200 import build as kb
    kb.build()
    out = tmp_path_factory.mktemp("cppgpu") / "tuner_gpu_tests"
    lib = os.path.join(REPO, "ktt_b200")
    subprocess.run([_cxx(), "-std=c++17", "-O2", "-I", os.path.join(REPO, "include"),
                    os.path.join(REPO, "tests", "cpp", "tuner_gpu_tests.cpp"), "-o", str(out), "-L", lib,
                    "-lktt_b200", "-lcoulktt", f"-Wl,-rpath,{lib}"], check=True)
    return str(out)


@pytest.mark.parametrize("name", ["coulomb3d_tune", "coulomb3d_reference_computation", "coulomb2d_random",
                                  "iterative_launcher", "user_buffers", "nbody_example"])
def test_tuner_gpu(gpu_tests_binary, workdir, name):  # noqa: F811
    r = subprocess.run([gpu_tests_binary, name, workdir], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-4000:]


def test_profile_based_searcher_cpp(gpu_tests_binary, tmp_path):
    """Counters and the profile-based searcher from a C++ host program; the counter model is trained
    from the B200 recording of the same tile space (tests/golden/b200_map3d_space_64.json)."""
    from ktt_b200 import profile_model, run_searchers
    space = run_searchers.load_space(os.path.join(REPO, "tests", "golden", "b200_map3d_space_64.json"))
    run_searchers.write_ktt_results(space, str(tmp_path / "space.json"))
    profile_model.main([str(tmp_path / "space.json"), "--out", str(tmp_path / "b200_64.model.json")])
    r = subprocess.run([gpu_tests_binary, "profile_based", str(tmp_path)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-4000:]
