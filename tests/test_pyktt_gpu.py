"""A KTT-style Python host program for CoulombSum3d through pyktt on the B200: the kernel
definition, arguments, KTT's tuning parameters, thread modifiers and constraints
(Examples/CoulombSum3d/CoulombSum3d.cpp:67-237, written against KTT's Python API), a reference
computation in Python (the FP64 oracle) and KTT's SideBySide validation, a random-search Tune, then
Run of the best configuration with the output downloaded into a NumPy array."""
import numpy as np
import pytest

import oracle
from ktt_b200 import errors
from ktt_b200 import pyktt as ktt

pytestmark = pytest.mark.gpu


def test_coulomb3d_python_host_program():
    grid, n, h = 128, 1024, 0.5
    rng = np.random.default_rng(21)
    atoms = np.empty((n, 4), dtype=np.float32)
    atoms[:, :3] = rng.uniform(0.0, grid * h, (n, 3))
    atoms[:, 3] = rng.uniform(-1.0, 1.0, n)
    reference = oracle.grid3d(atoms, h, (grid, grid, grid)).astype(np.float32).reshape(-1)

    ktt.Tuner.SetLoggingLevel(ktt.LoggingLevel.Warning)
    tuner = ktt.Tuner(0, 0, ktt.ComputeApi.CUDA)
    tuner.SetGlobalSizeType(ktt.GlobalSizeType.CUDA)
    tuner.SetCompilerOptions("-use_fast_math")
    d = tuner.AddKernelDefinitionFromFile("directCoulombSum", "CoulombSum3d.cu", ktt.DimensionVector(grid, grid, grid),
                                          ktt.DimensionVector())
    k = tuner.CreateSimpleKernel("CoulombSum", d)
    ro = ktt.ArgumentAccessType.ReadOnly
    args = [tuner.AddArgumentVectorFloat(atoms.reshape(-1), ro)]
    args += [tuner.AddArgumentVectorFloat(np.ascontiguousarray(atoms[:, c]), ro) for c in range(4)]
    args += [tuner.AddArgumentScalarInt(n), tuner.AddArgumentScalarFloat(h), tuner.AddArgumentScalarInt(grid)]
    grid_id = tuner.AddArgumentVectorFloat(np.zeros(grid ** 3, dtype=np.float32), ktt.ArgumentAccessType.WriteOnly)
    args.append(grid_id)
    tuner.SetArguments(d, args)

    tuner.AddParameter(k, "WORK_GROUP_SIZE_X", [16, 32])
    tuner.AddParameter(k, "WORK_GROUP_SIZE_Y", [1, 2, 4, 8])
    tuner.AddParameter(k, "WORK_GROUP_SIZE_Z", [1])
    tuner.AddParameter(k, "Z_ITERATIONS", [1, 2, 4, 8, 16, 32])
    tuner.AddParameter(k, "INNER_UNROLL_FACTOR", [0, 1, 2, 4, 8, 16, 32])
    tuner.AddParameter(k, "USE_CONSTANT_MEMORY", [0])
    tuner.AddParameter(k, "USE_SOA", [0, 1])
    tuner.AddParameter(k, "VECTOR_SIZE", [1])
    for dim, name in ((ktt.ModifierDimension.X, "WORK_GROUP_SIZE_X"), (ktt.ModifierDimension.Y, "WORK_GROUP_SIZE_Y")):
        tuner.AddThreadModifier(k, [d], ktt.ModifierType.Local, dim, name, ktt.ModifierAction.Multiply)
        tuner.AddThreadModifier(k, [d], ktt.ModifierType.Global, dim, name, ktt.ModifierAction.DivideCeil)
    tuner.AddThreadModifier(k, [d], ktt.ModifierType.Global, ktt.ModifierDimension.Z, "Z_ITERATIONS",
                            ktt.ModifierAction.DivideCeil)
    tuner.AddConstraint(k, ["INNER_UNROLL_FACTOR", "Z_ITERATIONS"], lambda v: v[0] < v[1])
    tuner.AddConstraint(k, ["WORK_GROUP_SIZE_X", "WORK_GROUP_SIZE_Y"], lambda v: v[0] * v[1] >= 64)

    def compute_reference(buffer):
        np.frombuffer(buffer, dtype=np.float32)[:] = reference

    tuner.SetReferenceComputation(grid_id, grid ** 3 * 4, compute_reference)
    tuner.SetValidationMethod(ktt.ValidationMethod.SideBySideComparison, 0.01)
    tuner.SetSearcher(k, ktt.RandomSearcher())
    results = tuner.Tune(k, ktt.ConfigurationCount(12))
    assert len(results) == 12
    assert all(r.GetStatus() == ktt.ResultStatus.Ok for r in results), [str(r.GetStatus()) for r in results]

    best = tuner.GetBestConfiguration(k)
    out = np.zeros(grid ** 3, dtype=np.float32)
    result = tuner.Run(k, best, [ktt.BufferOutputDescriptor(grid_id, out)])
    assert result.GetStatus() == ktt.ResultStatus.Ok
    assert errors.report(out, reference)["rel_norm"] <= 1e-5


def test_device_info_and_local_symbol_arguments():
    """Tutorials/01ComputeApiInfo on the B200, and a CoulombSum3d definition whose argument list ends
    in a local-memory and a symbol argument (neither is a CUDA function parameter in KTT's CUDA
    engine): it still maps onto the built-in kernel and validates."""
    tuner = ktt.Tuner(0, 0, ktt.ComputeApi.CUDA)
    devices = tuner.GetDeviceInfo(0)
    assert devices and devices[0].GetCudaComputeCapabilityMajor() == 10
    current = tuner.GetCurrentDeviceInfo()
    assert current.GetName() == devices[0].GetName() and current.GetMaxComputeUnits() >= 100
    assert current.GetMaxWorkGroupSize() == 1024 and current.GetGlobalMemorySize() > (64 << 30)
    assert current.GetDeviceTypeString() == "GPU" and "CUDA compute capability: 10." in current.GetString()
    assert int(tuner.GetPlatformInfo()[0].GetVersion()) >= 12000

    grid, n, h = 32, 96, 0.5
    rng = np.random.default_rng(5)
    atoms = np.empty((n, 4), dtype=np.float32)
    atoms[:, :3] = rng.uniform(0.0, grid * h, (n, 3))
    atoms[:, 3] = rng.uniform(-1.0, 1.0, n)
    reference = oracle.grid3d(atoms, h, (grid, grid, grid)).astype(np.float32).reshape(-1)
    tuner.SetGlobalSizeType(ktt.GlobalSizeType.CUDA)
    d = tuner.AddKernelDefinition("directCoulombSum", "", ktt.DimensionVector(grid, grid, grid), ktt.DimensionVector())
    k = tuner.CreateSimpleKernel("CoulombSum", d)
    ro = ktt.ArgumentAccessType.ReadOnly
    args = [tuner.AddArgumentVectorFloat(atoms.reshape(-1), ro)]
    args += [tuner.AddArgumentVectorFloat(np.ascontiguousarray(atoms[:, c]), ro) for c in range(4)]
    args += [tuner.AddArgumentScalarInt(n), tuner.AddArgumentScalarFloat(h), tuner.AddArgumentScalarInt(grid)]
    grid_id = tuner.AddArgumentVectorFloat(np.zeros(grid ** 3, dtype=np.float32), ktt.ArgumentAccessType.WriteOnly)
    args += [grid_id, tuner.AddArgumentSymbolInt(grid, symbolName="cGridSize"), tuner.AddArgumentLocalFloat(4096)]
    tuner.SetArguments(d, args)
    for name, value in (("WORK_GROUP_SIZE_X", 32), ("WORK_GROUP_SIZE_Y", 4), ("WORK_GROUP_SIZE_Z", 1),
                        ("Z_ITERATIONS", 8), ("INNER_UNROLL_FACTOR", 2), ("USE_CONSTANT_MEMORY", 0), ("USE_SOA", 0),
                        ("VECTOR_SIZE", 1)):
        tuner.AddParameter(k, name, [value])
    for dim, name in ((ktt.ModifierDimension.X, "WORK_GROUP_SIZE_X"), (ktt.ModifierDimension.Y, "WORK_GROUP_SIZE_Y")):
        tuner.AddThreadModifier(k, [d], ktt.ModifierType.Local, dim, name, ktt.ModifierAction.Multiply)
        tuner.AddThreadModifier(k, [d], ktt.ModifierType.Global, dim, name, ktt.ModifierAction.DivideCeil)
    tuner.AddThreadModifier(k, [d], ktt.ModifierType.Global, ktt.ModifierDimension.Z, "Z_ITERATIONS",
                            ktt.ModifierAction.DivideCeil)

    def compute_reference(buffer):
        np.frombuffer(buffer, dtype=np.float32)[:] = reference

    tuner.SetReferenceComputation(grid_id, grid ** 3 * 4, compute_reference)
    tuner.SetValidationMethod(ktt.ValidationMethod.SideBySideComparison, 0.01)
    results = tuner.Tune(k)
    assert len(results) == 1 and results[0].GetStatus() == ktt.ResultStatus.Ok, str(results[0].GetStatus())


# Run in a child process: it creates and destroys a CUDA context of its own, which the other tests'
# process-wide device state should not see.
_INITIALIZER_PROGRAM = r'''
import ctypes
import numpy as np
import oracle
from ktt_b200 import errors
from ktt_b200 import pyktt as ktt

cu = ctypes.CDLL("libcuda.so.1")


def ck(r, what):
    if r != 0:
        raise SystemExit(f"{what} failed with driver error {r}")


ck(cu.cuInit(0), "cuInit")
dev = ctypes.c_int()
ck(cu.cuDeviceGet(ctypes.byref(dev), 0), "cuDeviceGet")
ctx = ctypes.c_void_p()
ck(cu.cuCtxCreate_v2(ctypes.byref(ctx), 0, dev), "cuCtxCreate")
s1, s2 = ctypes.c_void_p(), ctypes.c_void_p()
ck(cu.cuStreamCreate(ctypes.byref(s1), 0), "cuStreamCreate")
ck(cu.cuStreamCreate(ctypes.byref(s2), 0), "cuStreamCreate")

tuner = ktt.Tuner(ktt.ComputeApi.CUDA, ktt.ComputeApiInitializer(ctx.value, [s1.value]))
assert tuner.AddComputeQueue(s2.value) == 1
grid, n, h = 32, 80, 0.5
rng = np.random.default_rng(9)
atoms = np.empty((n, 4), dtype=np.float32)
atoms[:, :3] = rng.uniform(0.0, grid * h, (n, 3))
atoms[:, 3] = rng.uniform(-1.0, 1.0, n)
reference = oracle.grid3d(atoms, h, (grid, grid, grid)).astype(np.float32).reshape(-1)
tuner.SetGlobalSizeType(ktt.GlobalSizeType.CUDA)
d = tuner.AddKernelDefinition("directCoulombSum", "", ktt.DimensionVector(grid, grid, grid), ktt.DimensionVector())
k = tuner.CreateSimpleKernel("CoulombSum", d)
ro = ktt.ArgumentAccessType.ReadOnly
args = [tuner.AddArgumentVectorFloat(atoms.reshape(-1), ro)]
args += [tuner.AddArgumentVectorFloat(np.ascontiguousarray(atoms[:, c]), ro) for c in range(4)]
args += [tuner.AddArgumentScalarInt(n), tuner.AddArgumentScalarFloat(h), tuner.AddArgumentScalarInt(grid)]
out_id = tuner.AddArgumentVectorFloat(np.zeros(grid ** 3, dtype=np.float32), ktt.ArgumentAccessType.WriteOnly)
tuner.SetArguments(d, args + [out_id])
for name, value in (("WORK_GROUP_SIZE_X", 32), ("WORK_GROUP_SIZE_Y", 4), ("Z_ITERATIONS", 8),
                    ("INNER_UNROLL_FACTOR", 2), ("USE_SOA", 0)):
    tuner.AddParameter(k, name, [value])
for dim, name in ((ktt.ModifierDimension.X, "WORK_GROUP_SIZE_X"), (ktt.ModifierDimension.Y, "WORK_GROUP_SIZE_Y")):
    tuner.AddThreadModifier(k, [d], ktt.ModifierType.Local, dim, name, ktt.ModifierAction.Multiply)
    tuner.AddThreadModifier(k, [d], ktt.ModifierType.Global, dim, name, ktt.ModifierAction.DivideCeil)
tuner.AddThreadModifier(k, [d], ktt.ModifierType.Global, ktt.ModifierDimension.Z, "Z_ITERATIONS",
                        ktt.ModifierAction.DivideCeil)
seen = []


def launcher(ci):
    seen.append(list(ci.GetAllQueues()))
    ci.RunKernelAsync(d, 1)  # on the second of the caller's streams
    ci.SynchronizeQueues()


tuner.SetLauncher(k, launcher)
out = np.zeros(grid ** 3, dtype=np.float32)
config = tuner.CreateConfiguration(k, [("WORK_GROUP_SIZE_X", 32), ("WORK_GROUP_SIZE_Y", 4), ("Z_ITERATIONS", 8),
                                       ("INNER_UNROLL_FACTOR", 2), ("USE_SOA", 0)])
result = tuner.Run(k, config, [ktt.BufferOutputDescriptor(out_id, out)])
assert result.GetStatus() == ktt.ResultStatus.Ok, str(result.GetStatus())
assert seen == [[0, 1]], seen
assert errors.report(out, reference)["rel_norm"] <= 1e-5
tuner.SynchronizeQueue(1)
tuner.RemoveComputeQueue(1)
assert tuner.GetCurrentDeviceInfo().GetCudaComputeCapabilityMajor() == 10
del tuner
ck(cu.cuStreamDestroy_v2(s1), "cuStreamDestroy")
ck(cu.cuStreamDestroy_v2(s2), "cuStreamDestroy")
ck(cu.cuCtxDestroy_v2(ctx), "cuCtxDestroy")
print("initializer ok")
'''


def test_compute_api_initializer_with_callers_context():
    """Tutorials/05ComputeApiInitializer: a tuner on a CUDA context and streams the caller created
    with the driver API; a launcher runs the kernel on the second stream (AddComputeQueue) and the
    map matches the FP64 oracle."""
    import os
    import subprocess
    import sys
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, PYTHONPATH=repo + os.pathsep + os.environ.get("PYTHONPATH", ""))
    r = subprocess.run([sys.executable, "-c", _INITIALIZER_PROGRAM], cwd=repo, env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0 and "initializer ok" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]


def test_launcher_transfers_resize_and_local_size():
    """ComputeInterface's queue transfers, ResizeBuffer (data kept), UpdateLocalArgument and
    GetProfiling from a Python launcher (Source/Api/ComputeInterface.h:202-349)."""
    tuner = ktt.Tuner(0, 0, ktt.ComputeApi.CUDA)
    d = tuner.AddKernelDefinition("noop", "", ktt.DimensionVector(32), ktt.DimensionVector(32))
    k = tuner.CreateSimpleKernel("k", d)
    rw = ktt.ArgumentAccessType.ReadWrite
    a = tuner.AddArgumentVectorFloat(np.arange(16, dtype=np.float32), rw)
    b = tuner.AddArgumentVectorFloat(np.zeros(16, dtype=np.float32), rw)
    local = tuner.AddArgumentLocalFloat(256)
    got = {}

    def launcher(ci):
        ci.UploadBufferAsync(a, 0)
        ci.UploadBufferAsync(b, 0)
        ci.WaitForTransferAction(ci.CopyBufferAsync(b, a, 0, 32))  # the first 8 floats
        ci.UpdateBufferAsync(a, 0, np.full(16, 5.0, dtype=np.float32))
        ci.ResizeBuffer(b, 128, True)  # 32 floats, the 16 old ones kept
        out_b = np.full(32, -1.0, dtype=np.float32)
        ci.DownloadBufferAsync(b, 0, out_b)
        ci.SynchronizeQueues()
        out_a = np.zeros(16, dtype=np.float32)
        ci.DownloadBuffer(a, out_a)
        ci.UpdateLocalArgument(local, 512)
        got.update(a=out_a, b=out_b, profiling=ci.GetProfiling(k))

    tuner.SetLauncher(k, launcher)
    result = tuner.Run(k, tuner.CreateConfiguration(k, []), [])
    assert result.GetStatus() == ktt.ResultStatus.Ok, str(result.GetStatus())
    assert np.array_equal(got["b"][:8], np.arange(8, dtype=np.float32))
    assert not got["b"][8:].any()
    assert np.array_equal(got["a"], np.full(16, 5.0, dtype=np.float32))
    assert got["profiling"] is False


def test_launcher_updates_hold_for_one_run_only():
    """KTT's launcher-side updates are per run (Source/KernelRunner/ComputeLayer.cpp:160-190:
    UpdateScalarArgument / UpdateLocalArgument add argument overrides dropped with the run;
    CudaEngine.cpp:430-470, 558-569: UpdateBuffer and ResizeBuffer change the device buffer only,
    and writable buffers are re-created from the host data by the next run).  The first run's
    launcher sets the atom count to 0, overwrites one buffer, resizes another and changes a local
    size; the second run's launcher changes nothing and must see the original values."""
    grid, n, h = 32, 96, 0.5
    rng = np.random.default_rng(17)
    atoms = np.empty((n, 4), dtype=np.float32)
    atoms[:, :3] = rng.uniform(0.0, grid * h, (n, 3))
    atoms[:, 3] = rng.uniform(-1.0, 1.0, n)
    reference = oracle.grid3d(atoms, h, (grid, grid, grid)).reshape(-1)

    tuner = ktt.Tuner(0, 0, ktt.ComputeApi.CUDA)
    tuner.SetGlobalSizeType(ktt.GlobalSizeType.CUDA)
    d = tuner.AddKernelDefinition("directCoulombSum", "", ktt.DimensionVector(grid, grid, grid), ktt.DimensionVector())
    side = tuner.AddKernelDefinition("noop", "", ktt.DimensionVector(32), ktt.DimensionVector(32))
    ro, rw = ktt.ArgumentAccessType.ReadOnly, ktt.ArgumentAccessType.ReadWrite
    args = [tuner.AddArgumentVectorFloat(atoms.reshape(-1), ro)]
    args += [tuner.AddArgumentVectorFloat(np.ascontiguousarray(atoms[:, c]), ro) for c in range(4)]
    n_id = tuner.AddArgumentScalarInt(n)
    args += [n_id, tuner.AddArgumentScalarFloat(h), tuner.AddArgumentScalarInt(grid)]
    map_id = tuner.AddArgumentVectorFloat(np.zeros(grid ** 3, dtype=np.float32), ktt.ArgumentAccessType.WriteOnly)
    tuner.SetArguments(d, args + [map_id])
    aux = tuner.AddArgumentVectorFloat(np.arange(16, dtype=np.float32), rw)
    grown = tuner.AddArgumentVectorFloat(np.arange(16, dtype=np.float32) + 100.0, rw)
    local = tuner.AddArgumentLocalFloat(256)
    tuner.SetArguments(side, [aux, grown, local])
    state = {"update": True}
    seen = []

    def launcher(ci):
        if state["update"]:
            ci.UpdateScalarArgumentInt(n_id, 0)
            ci.UpdateBuffer(aux, np.full(16, 5.0, dtype=np.float32))
            ci.ResizeBuffer(grown, 128, True)
            ci.UpdateLocalArgument(local, 512)
        ci.RunKernel(d)
        got_map = np.empty(grid ** 3, dtype=np.float32)
        ci.DownloadBuffer(map_id, got_map)
        got_aux = np.zeros(16, dtype=np.float32)
        ci.DownloadBuffer(aux, got_aux)
        got_grown = np.full(32, -1.0, dtype=np.float32)
        ci.DownloadBuffer(grown, got_grown)
        seen.append((got_map, got_aux, got_grown))

    k = tuner.CreateCompositeKernel("CoulombSumWithSideBuffers", [d, side], launcher)
    for name, value in (("WORK_GROUP_SIZE_X", 32), ("WORK_GROUP_SIZE_Y", 4), ("Z_ITERATIONS", 8),
                        ("INNER_UNROLL_FACTOR", 2), ("USE_SOA", 0)):
        tuner.AddParameter(k, name, [value])
    for dim, name in ((ktt.ModifierDimension.X, "WORK_GROUP_SIZE_X"), (ktt.ModifierDimension.Y, "WORK_GROUP_SIZE_Y")):
        tuner.AddThreadModifier(k, [d], ktt.ModifierType.Local, dim, name, ktt.ModifierAction.Multiply)
        tuner.AddThreadModifier(k, [d], ktt.ModifierType.Global, dim, name, ktt.ModifierAction.DivideCeil)
    tuner.AddThreadModifier(k, [d], ktt.ModifierType.Global, ktt.ModifierDimension.Z, "Z_ITERATIONS",
                            ktt.ModifierAction.DivideCeil)
    config = tuner.CreateConfiguration(k, [("WORK_GROUP_SIZE_X", 32), ("WORK_GROUP_SIZE_Y", 4), ("Z_ITERATIONS", 8),
                                           ("INNER_UNROLL_FACTOR", 2), ("USE_SOA", 0)])
    for update in (True, False):
        state["update"] = update
        result = tuner.Run(k, config, [])
        assert result.GetStatus() == ktt.ResultStatus.Ok, str(result.GetStatus())

    (map1, aux1, grown1), (map2, aux2, grown2) = seen
    # first run: no atoms, the updated buffer, the resized buffer (old values kept, the rest zero)
    assert not map1.any()
    assert np.array_equal(aux1, np.full(16, 5.0, dtype=np.float32))
    assert np.array_equal(grown1[:16], np.arange(16, dtype=np.float32) + 100.0) and not grown1[16:].any()
    # second run: the original atom count, buffer contents and buffer size
    assert errors.report(map2, reference)["rel_norm"] <= 1e-5
    assert np.array_equal(aux2, np.arange(16, dtype=np.float32))
    assert np.array_equal(grown2[:16], np.arange(16, dtype=np.float32) + 100.0)
    assert np.all(grown2[16:] == -1.0)
