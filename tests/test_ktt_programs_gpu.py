"""KTT's own Coulomb host programs, compiled unchanged against this library's KTT surface.

``make -C oracle kttprograms`` compiles, from the KTT tree where they lie, with -DKTT_CUDA_EXAMPLE
and no source edits, against include/Ktt.h and -lktt_b200 -lcoulktt:

* Examples/CoulombSum3d/CoulombSum3d.cpp: CUDA, profiling on (so no validation), deterministic
  search of KTT's 210-configuration CUDA space, JSON and XML result files;
* Examples/CoulombSum2d/CoulombSum2d.cpp: written for KTT's OpenCL engine, random search for 60 s,
  validated against the 2D reference kernel (SideBySide, 0.01);
* Examples/CoulombSum3dIterative/CoulombSum3dIterative.cpp: OpenCL engine, a launcher running one
  2D slice per z plane (host dz^2, UpdateBuffer, UpdateScalarArgument), validated against the 3D
  reference kernel.

Each runs on the GPU with its own command line (platform 0, device 0; its kernel source files are
not needed: definitions are matched to the built-in kernels by name and argument list).  Their
search spaces and stop conditions are fixed in their sources, so KTT_B200_CONFIGURATION_LIMIT caps
the configurations each Tune call runs.  Each program must exit 0 and save KTT's result files; the
tests read them, then run each file's best configuration again through this library's tuner on
seeded atoms and check the map against the FP64 oracle.
"""
import json
import os
import subprocess

import numpy as np
import pytest

import oracle
from ktt_b200 import errors

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PROGRAMS = os.path.join(REPO, "oracle", "_ref", "ktt_programs")
LIMIT = 6

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.isdir(PROGRAMS),
                                 reason="KTT's host programs were not built (make -C oracle kttprograms KTT_ROOT=...)")]


def _run(program, tmp_path):
    env = dict(os.environ, KTT_B200_CONFIGURATION_LIMIT=str(LIMIT))
    r = subprocess.run([os.path.join(PROGRAMS, program), "0", "0"], cwd=tmp_path, env=env, capture_output=True,
                       text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    return r


def _results(path):
    with open(path) as f:
        data = json.load(f)
    assert data["Metadata"]["KttVersion"].startswith("2.")
    return data["Results"]


def _best(results):
    ok = [r for r in results if r["Status"] == "Ok"]
    assert ok, [r["Status"] for r in results]
    best = min(ok, key=lambda r: r["TotalDuration"])
    return {c["Name"]: int(c["Value"]) for c in best["Configuration"]}


def _atoms(n, box, seed):
    rng = np.random.default_rng(seed)
    a = np.empty((n, 4), dtype=np.float32)
    a[:, :3] = rng.uniform(0.0, box, (n, 3))
    a[:, 3] = rng.uniform(-1.0, 1.0, n)
    return a


def _add_fixed_parameters(tuner, kernel, config):
    from ktt_b200 import pyktt as ktt
    for name, value in config.items():
        tuner.AddParameter(kernel, name, [value])
    return tuner.CreateConfiguration(kernel, list(config.items()))


def test_coulomb_sum_3d_program(tmp_path):
    from ktt_b200 import pyktt as ktt
    _run("CoulombSum3d", tmp_path)
    results = _results(tmp_path / "CoulombSumOutput.json")
    assert (tmp_path / "CoulombSumOutput.xml").exists()
    assert len(results) == LIMIT
    assert all(r["Status"] == "Ok" for r in results), [r["Status"] for r in results]
    # profiling is on in this program: every run carries hardware counters
    for r in results:
        assert r["ComputationResults"] and "ProfilingData" in r["ComputationResults"][0]
    config = _best(results)

    # the best configuration, again, on seeded atoms, against the FP64 oracle
    grid, n, h = 64, 700, 0.5
    atoms = _atoms(n, grid * h, seed=31)
    reference = oracle.grid3d(atoms, h, (grid, grid, grid)).reshape(-1)
    tuner = ktt.Tuner(0, 0, ktt.ComputeApi.CUDA)
    tuner.SetGlobalSizeType(ktt.GlobalSizeType.CUDA)
    d = tuner.AddKernelDefinition("directCoulombSum", "", ktt.DimensionVector(grid, grid, grid), ktt.DimensionVector())
    k = tuner.CreateSimpleKernel("CoulombSum", d)
    ro = ktt.ArgumentAccessType.ReadOnly
    args = [tuner.AddArgumentVectorFloat(atoms.reshape(-1), ro)]
    args += [tuner.AddArgumentVectorFloat(np.ascontiguousarray(atoms[:, c]), ro) for c in range(4)]
    args += [tuner.AddArgumentScalarInt(n), tuner.AddArgumentScalarFloat(h), tuner.AddArgumentScalarInt(grid)]
    out_id = tuner.AddArgumentVectorFloat(np.zeros(grid ** 3, dtype=np.float32), ktt.ArgumentAccessType.WriteOnly)
    tuner.SetArguments(d, args + [out_id])
    for dim, name in ((ktt.ModifierDimension.X, "WORK_GROUP_SIZE_X"), (ktt.ModifierDimension.Y, "WORK_GROUP_SIZE_Y")):
        tuner.AddThreadModifier(k, [d], ktt.ModifierType.Local, dim, name, ktt.ModifierAction.Multiply)
        tuner.AddThreadModifier(k, [d], ktt.ModifierType.Global, dim, name, ktt.ModifierAction.DivideCeil)
    tuner.AddThreadModifier(k, [d], ktt.ModifierType.Global, ktt.ModifierDimension.Z, "Z_ITERATIONS",
                            ktt.ModifierAction.DivideCeil)
    cfg = _add_fixed_parameters(tuner, k, config)
    out = np.zeros(grid ** 3, dtype=np.float32)
    result = tuner.Run(k, cfg, [ktt.BufferOutputDescriptor(out_id, out)])
    assert result.GetStatus() == ktt.ResultStatus.Ok, str(result.GetStatus())
    assert errors.report(out, reference)["rel_norm"] <= 1e-5, config


def test_coulomb_sum_2d_program(tmp_path):
    from ktt_b200 import pyktt as ktt
    _run("CoulombSum2d", tmp_path)
    results = _results(tmp_path / "CoulombSum2dOutput.json")
    assert len(results) == LIMIT
    statuses = [r["Status"] for r in results]
    # blocks above this library's 256-thread kernels end as DeviceLimitsExceeded; nothing fails validation
    assert set(statuses) <= {"Ok", "DeviceLimitsExceeded"}, statuses
    config = _best(results)

    nx, ny, h, n = 160, 96, 0.5, 900
    rng = np.random.default_rng(32)
    atoms = np.empty((n, 4), dtype=np.float32)
    atoms[:, :2] = rng.uniform(0.0, 80.0, (n, 2))
    atoms[:, 2] = rng.uniform(0.0, 40.0, n) ** 2  # KTT's 2D convention: .z holds dz^2
    atoms[:, 3] = rng.uniform(-1.0, 1.0, n)
    reference = oracle.slice2d(atoms, h, nx, ny).reshape(-1)
    tuner = ktt.Tuner(0, 0, ktt.ComputeApi.OpenCL)
    d = tuner.AddKernelDefinition("directCoulombSum", "", ktt.DimensionVector(nx, ny), ktt.DimensionVector())
    k = tuner.CreateSimpleKernel("CoulombSum", d)
    ro = ktt.ArgumentAccessType.ReadOnly
    args = [tuner.AddArgumentVectorFloat(atoms.reshape(-1), ro)]
    args += [tuner.AddArgumentVectorFloat(np.ascontiguousarray(atoms[:, c]), ro) for c in range(4)]
    args += [tuner.AddArgumentScalarInt(n), tuner.AddArgumentScalarFloat(h)]
    out_id = tuner.AddArgumentVectorFloat(np.zeros(nx * ny, dtype=np.float32), ktt.ArgumentAccessType.ReadWrite)
    tuner.SetArguments(d, args + [out_id])
    tuner.AddThreadModifier(k, [d], ktt.ModifierType.Global, ktt.ModifierDimension.X, "OUTER_UNROLL_FACTOR",
                            ktt.ModifierAction.Divide)
    tuner.AddThreadModifier(k, [d], ktt.ModifierType.Local, ktt.ModifierDimension.X, "WORK_GROUP_SIZE_X",
                            ktt.ModifierAction.Multiply)
    tuner.AddThreadModifier(k, [d], ktt.ModifierType.Local, ktt.ModifierDimension.Y, "WORK_GROUP_SIZE_Y",
                            ktt.ModifierAction.Multiply)
    cfg = _add_fixed_parameters(tuner, k, config)
    out = np.zeros(nx * ny, dtype=np.float32)
    result = tuner.Run(k, cfg, [ktt.BufferOutputDescriptor(out_id, out)])
    assert result.GetStatus() == ktt.ResultStatus.Ok, str(result.GetStatus())
    assert errors.report(out, reference)["rel_norm"] <= 1e-5, config


def test_coulomb_sum_3d_iterative_program(tmp_path):
    from ktt_b200 import pyktt as ktt
    _run("CoulombSum3dIterative", tmp_path)
    results = _results(tmp_path / "CoulombSum3dIterativeOutput.json")
    assert len(results) == LIMIT
    assert all(r["Status"] == "Ok" for r in results), [r["Status"] for r in results]
    # the launcher ran one slice per z plane of the 256^3 map
    assert all(r["ComputationResults"][0]["KernelFunction"] == "directCoulombSum" for r in results)
    config = _best(results)

    grid, n, h = 40, 400, 0.5
    atoms = _atoms(n, grid * h, seed=33)
    reference = oracle.grid3d(atoms, h, (grid, grid, grid)).reshape(-1)
    precomp = atoms.copy()
    z2 = np.zeros(n, dtype=np.float32)
    tuner = ktt.Tuner(0, 0, ktt.ComputeApi.OpenCL)
    d = tuner.AddKernelDefinition("directCoulombSum", "", ktt.DimensionVector(grid, grid, grid), ktt.DimensionVector())
    k = tuner.CreateSimpleKernel("CoulombSum", d)
    ro = ktt.ArgumentAccessType.ReadOnly
    precomp_id = tuner.AddArgumentVectorFloat(precomp.reshape(-1), ro)
    x_id = tuner.AddArgumentVectorFloat(np.ascontiguousarray(atoms[:, 0]), ro)
    y_id = tuner.AddArgumentVectorFloat(np.ascontiguousarray(atoms[:, 1]), ro)
    z2_id = tuner.AddArgumentVectorFloat(z2, ro)
    w_id = tuner.AddArgumentVectorFloat(np.ascontiguousarray(atoms[:, 3]), ro)
    z_id = tuner.AddArgumentScalarInt(0)
    out_id = tuner.AddArgumentVectorFloat(np.zeros(grid ** 3, dtype=np.float32), ktt.ArgumentAccessType.ReadWrite)
    tuner.SetArguments(d, [precomp_id, x_id, y_id, z2_id, w_id, tuner.AddArgumentScalarInt(n),
                           tuner.AddArgumentScalarFloat(h), z_id, out_id])
    tuner.AddThreadModifier(k, [d], ktt.ModifierType.Local, ktt.ModifierDimension.X, "WORK_GROUP_SIZE_X",
                            ktt.ModifierAction.Multiply)
    tuner.AddThreadModifier(k, [d], ktt.ModifierType.Local, ktt.ModifierDimension.Y, "WORK_GROUP_SIZE_Y",
                            ktt.ModifierAction.Multiply)
    tuner.AddThreadModifier(k, [d], ktt.ModifierType.Global, ktt.ModifierDimension.X, "OUTER_UNROLL_FACTOR",
                            ktt.ModifierAction.Divide)

    def launcher(ci):
        g = ci.GetCurrentGlobalSize(d)
        local = ci.GetCurrentLocalSize(d)
        g.SetSizeZ(1)
        for i in range(grid):
            dz2 = ((h * i) - atoms[:, 2]) ** 2
            if config["USE_SOA"] == 0:
                precomp[:, 2] = dz2
                ci.UpdateBuffer(precomp_id, precomp.reshape(-1))
            else:
                ci.UpdateBuffer(z2_id, dz2.astype(np.float32))
            ci.UpdateScalarArgumentInt(z_id, i)
            ci.RunKernel(d, g, local)

    tuner.SetLauncher(k, launcher)
    cfg = _add_fixed_parameters(tuner, k, config)
    out = np.zeros(grid ** 3, dtype=np.float32)
    result = tuner.Run(k, cfg, [ktt.BufferOutputDescriptor(out_id, out)])
    assert result.GetStatus() == ktt.ResultStatus.Ok, str(result.GetStatus())
    assert errors.report(out, reference)["rel_norm"] <= 1e-5, config
