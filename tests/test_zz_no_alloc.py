"""coul_batch_run_static: the batched map for callers that must not allocate device memory.

Some callers cannot let a library call cudaMalloc (their host owns all device memory through its
own pool, or they cannot afford the synchronisation of cudaFree).  This entry point keeps its work
queue and molecule table in a fixed static device array instead.  The test calls it through the C
ABI twice in a row, on two different batches, and checks each result against the allocating entry
point (coul_batch_create + coul_batch_run) within the suite's tolerance.  It lives in its own file,
collected last, and passes both alone in a fresh process and after the other tests.
"""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

import ktt_b200
from ktt_b200 import errors, workloads

pytestmark = pytest.mark.gpu

TOL_NORM = 1e-5


def _molecules(seed, n_mol):
    import torch
    mols = workloads.molecule_batch(seed=seed, n_mol=n_mol, lo=60, hi=2500)
    return [(torch.from_numpy(m.atoms).cuda(), m.dims, m.spacing, m.origin) for m in mols]


def _static_run(lib, inputs, tune):
    """Calls coul_batch_run_static through ctypes; returns the output maps."""
    import torch
    from ktt_b200._signatures import Molecule
    fn = lib.coul_batch_run_static
    fn.argtypes = [ctypes.c_void_p, ctypes.POINTER(Molecule), ctypes.c_int, ctypes.POINTER(ktt_b200._Tune),
                   ctypes.c_int, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    arr = (Molecule * len(inputs))()
    outs = []
    for i, (atoms, dims, spacing, origin) in enumerate(inputs):
        nx, ny, nz = dims
        out = torch.full((nz, ny, nx), float("nan"), dtype=torch.float32, device="cuda")
        outs.append(out)
        arr[i].d_atoms = atoms.data_ptr()
        arr[i].n_atoms = atoms.shape[0]
        arr[i].grid = ktt_b200._grid(dims, spacing, origin)
        arr[i].d_out = out.data_ptr()
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    t = tune.c()
    stream = torch.cuda.current_stream().cuda_stream
    rc = fn(ctypes.c_void_p(stream), arr, len(inputs), ctypes.byref(t), 0, ctypes.c_void_p(status.data_ptr()))
    assert rc == ktt_b200.COUL_OK, lib.coul_last_error()
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    return [o.cpu().numpy() for o in outs]


def _allocating_run(ctx, inputs, tune):
    b = ktt_b200.Batch(ctx, inputs, tune)
    b.run(ktt_b200.BATCH_PERSISTENT)
    ctx.synchronize()
    maps = [o.cpu().numpy() for o in b.outputs]
    b.close()
    return maps


def test_static_entry_point_matches_allocating_entry_point_twice():
    lib = ktt_b200.load_library()
    ctx = ktt_b200.CoulombContext(0)
    tune = ktt_b200.Tune(block_x=32, block_y=4, z_iterations=8, x_points=2, unroll=2, rsqrt_soft=2)
    first = _molecules(seed=41, n_mol=9)
    second = _molecules(seed=42, n_mol=5)  # fewer molecules: the second call must not see the first's table
    for inputs in (first, second):
        got = _static_run(lib, inputs, tune)
        want = _allocating_run(ctx, inputs, tune)
        for g, w in zip(got, want):
            assert np.all(np.isfinite(g))
            rep = errors.report(g, w)
            assert rep["rel_norm"] <= TOL_NORM, rep
    ctx.close()


# Child process: the static array has one instance per CUDA context, so calls made under the
# device's primary context, then under a context the caller created with the driver API, then under
# the primary context again must each find their own context's copy.  One molecule per call is
# checked against the FP64 oracle.
_CONTEXT_PROGRAM = r'''
import ctypes
import numpy as np
import torch
import ktt_b200
import oracle
from ktt_b200 import errors
from ktt_b200._signatures import Molecule

cu = ctypes.CDLL("libcuda.so.1")
lib = ktt_b200.load_library()
fn = lib.coul_batch_run_static
fn.argtypes = [ctypes.c_void_p, ctypes.POINTER(Molecule), ctypes.c_int, ctypes.POINTER(ktt_b200._Tune),
               ctypes.c_int, ctypes.c_void_p]
fn.restype = ctypes.c_int


def ck(r, what):
    if r != 0:
        raise SystemExit(f"{what} failed with driver error {r}")


rng = np.random.default_rng(5)
n, dims, h = 300, (40, 24, 20), 0.5
atoms = np.empty((n, 4), dtype=np.float32)
atoms[:, :3] = rng.uniform(0.0, 12.0, (n, 3))
atoms[:, 3] = rng.uniform(-1.0, 1.0, n)
want = oracle.grid3d(atoms, h, dims)
tune = ktt_b200.Tune(block_x=32, block_y=4, z_iterations=8, x_points=2, unroll=2, rsqrt_soft=2).c()
out_bytes = dims[0] * dims[1] * dims[2] * 4


def run(d_atoms, d_out, stream):
    m = (Molecule * 1)()
    m[0].d_atoms, m[0].n_atoms, m[0].d_out = d_atoms, n, d_out
    m[0].grid = ktt_b200._grid(dims, h, None)
    rc = fn(ctypes.c_void_p(stream), m, 1, ctypes.byref(tune), 0, None)
    assert rc == ktt_b200.COUL_OK, lib.coul_last_error()


def primary_call():
    a = torch.from_numpy(atoms).cuda()
    o = torch.full((dims[2], dims[1], dims[0]), float("nan"), device="cuda")
    run(a.data_ptr(), o.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return o.cpu().numpy()


def own_context_call():
    dev = ctypes.c_int()
    ck(cu.cuDeviceGet(ctypes.byref(dev), 0), "cuDeviceGet")
    ctx = ctypes.c_void_p()
    ck(cu.cuCtxCreate_v2(ctypes.byref(ctx), 0, dev), "cuCtxCreate")  # current on this thread
    d_atoms, d_out = ctypes.c_uint64(), ctypes.c_uint64()
    ck(cu.cuMemAlloc_v2(ctypes.byref(d_atoms), ctypes.c_size_t(atoms.nbytes)), "cuMemAlloc")
    ck(cu.cuMemAlloc_v2(ctypes.byref(d_out), ctypes.c_size_t(out_bytes)), "cuMemAlloc")
    ck(cu.cuMemcpyHtoD_v2(d_atoms, atoms.ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(atoms.nbytes)), "HtoD")
    ck(cu.cuMemsetD32_v2(d_out, 0x7fc00000, ctypes.c_size_t(out_bytes // 4)), "cuMemsetD32")
    run(d_atoms.value, d_out.value, 0)  # the legacy default stream of the current (own) context
    ck(cu.cuCtxSynchronize(), "cuCtxSynchronize")
    got = np.empty((dims[2], dims[1], dims[0]), dtype=np.float32)
    ck(cu.cuMemcpyDtoH_v2(got.ctypes.data_as(ctypes.c_void_p), d_out, ctypes.c_size_t(out_bytes)), "DtoH")
    ck(cu.cuMemFree_v2(d_atoms), "cuMemFree")
    ck(cu.cuMemFree_v2(d_out), "cuMemFree")
    ck(cu.cuCtxDestroy_v2(ctx), "cuCtxDestroy")
    return got


maps = [primary_call(), own_context_call()]
torch.cuda.synchronize()  # back on the primary context
maps.append(primary_call())
for got in maps:
    assert np.all(np.isfinite(got))
    rep = errors.report(got, want)
    assert rep["rel_norm"] <= 1e-5, rep
print("contexts ok")
'''


def test_static_entry_point_under_callers_own_context():
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, PYTHONPATH=repo + os.pathsep + os.environ.get("PYTHONPATH", ""))
    r = subprocess.run([sys.executable, "-c", _CONTEXT_PROGRAM], cwd=repo, env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0 and "contexts ok" in r.stdout, r.stdout + r.stderr


def test_static_entry_point_rejects_oversized_batch():
    lib = ktt_b200.load_library()
    fn = lib.coul_batch_run_static
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ktt_b200._Tune), ctypes.c_int,
                   ctypes.c_void_p]
    fn.restype = ctypes.c_int
    t = ktt_b200.Tune(z_iterations=8, x_points=2, unroll=2, rsqrt_soft=2).c()
    assert fn(None, None, 1025, ctypes.byref(t), 0, None) == ktt_b200.COUL_ERR_INVALID_ARGUMENT
    assert b"1024" in lib.coul_last_error()
