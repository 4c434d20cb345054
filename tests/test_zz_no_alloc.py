"""coul_batch_run_static: the batched map for callers that must not allocate device memory.

Some callers cannot let a library call cudaMalloc (their host owns all device memory through its
own pool, or they cannot afford the synchronisation of cudaFree).  This entry point keeps its work
queue and molecule table in a fixed static device array instead.  The test calls it through the C
ABI twice in a row, on two different batches, and checks each result against the allocating entry
point (coul_batch_create + coul_batch_run) within the suite's tolerance.  It lives in its own file,
collected last, and passes both alone in a fresh process and after the other tests.
"""
import ctypes

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


def test_static_entry_point_rejects_oversized_batch():
    lib = ktt_b200.load_library()
    fn = lib.coul_batch_run_static
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ktt_b200._Tune), ctypes.c_int,
                   ctypes.c_void_p]
    fn.restype = ctypes.c_int
    t = ktt_b200.Tune(z_iterations=8, x_points=2, unroll=2, rsqrt_soft=2).c()
    assert fn(None, None, 1025, ctypes.byref(t), 0, None) == ktt_b200.COUL_ERR_INVALID_ARGUMENT
    assert b"1024" in lib.coul_last_error()
