"""CPU oracle for the direct Coulomb summation path -- TEST INFRASTRUCTURE ONLY.

Only the test-suite, ``__graft_entry__.smoke()`` (as the checker) and
``bench.py``'s CPU-baseline leg import this package.  The product path
(``ktt_b200`` / ``libcoulktt.so``) never calls it and has no CPU fallback.

The numerical code lives in ``coulomb_oracle.c`` (FP64 restatement of KTT's
reference computation: ``Examples/CoulombSum3d/CoulombSum3dReference.cu:11-26``,
``Examples/CoulombSum2d/CoulombSum2dReference.cl:8-20``) and
``coulomb_oracle_fp32.c`` (FP32 restatement of
``Examples/JSON/generate-coulomb-output.c:5-38``), built by ``oracle/Makefile``
into ``liboracle.so``.  Pinning: the FP32 restatement reproduces the output of
the reference's own generator (compiled from its source by ``make -C oracle
ref``) bit for bit; the sampled golden vectors of that output are committed in
``tests/golden/coulomb3d_kat.json``.  ``nbody_oracle.c`` restates the N-body step of KTT's Nbody
example (``Examples/Nbody/NbodyReference.cu:36-75``) in FP64.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")


def build() -> str:
    """Compile liboracle.so with the system gcc (OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    lib = ctypes.CDLL(_LIB_PATH)
    vp = ctypes.c_void_p
    i64 = ctypes.c_int64
    lib.oracle_max_threads.restype = ctypes.c_int
    lib.oracle_set_threads.argtypes = [ctypes.c_int]
    lib.oracle_grid3d.argtypes = [_f32p, i64, ctypes.c_float, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f64p]
    lib.oracle_points3d.argtypes = [_f32p, i64, ctypes.c_float, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    _i64p, i64, _f64p, vp]
    lib.oracle_slice2d.argtypes = [_f32p, i64, ctypes.c_float, ctypes.c_int, ctypes.c_int, _f64p]
    lib.oracle_adjoint3d.argtypes = [_f32p, i64, ctypes.c_float, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     vp, _f32p, vp, i64, vp, vp, vp, vp]
    lib.oracle_loss_perturbed.argtypes = [_f32p, i64, i64, _f64p, ctypes.c_float, vp, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, vp, _f32p, _f64p, vp]
    lib.oracle_kat_atoms.argtypes = [ctypes.c_int, _f32p]
    lib.oracle_kat_fp32.argtypes = [_f32p, ctypes.c_int, ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    _f32p]
    lib.oracle_nbody_step.argtypes = [_f32p, _f32p, i64, ctypes.c_float, ctypes.c_float, ctypes.c_float, vp, i64,
                                      _f64p, _f64p, _f64p]
    for name in ("oracle_grid3d", "oracle_points3d", "oracle_slice2d", "oracle_adjoint3d", "oracle_loss_perturbed",
                 "oracle_nbody_step"):
        getattr(lib, name).restype = ctypes.c_int
    _lib = lib
    return lib


def _atoms(a) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float32).reshape(-1, 4))
    return a


def _origin(origin):
    if origin is None:
        return None, None
    arr = np.ascontiguousarray(np.asarray(origin, dtype=np.float32).reshape(3))
    return arr, arr.ctypes.data_as(ctypes.c_void_p)


def _check(rc: int, what: str):
    if rc != 0:
        raise RuntimeError(f"{what} failed with status {rc}")


def max_threads() -> int:
    return int(_load().oracle_max_threads())


def set_threads(n: int) -> None:
    _load().oracle_set_threads(int(n))


def grid3d(atoms, h: float, dims, origin=None) -> np.ndarray:
    """FP64 map of shape (nz, ny, nx); dims = (nx, ny, nz)."""
    lib = _load()
    a = _atoms(atoms)
    nx, ny, nz = (int(d) for d in dims)
    out = np.empty(nx * ny * nz, dtype=np.float64)
    keep, optr = _origin(origin)
    _check(lib.oracle_grid3d(a, a.shape[0], np.float32(h), optr, nx, ny, nz, out), "oracle_grid3d")
    del keep
    return out.reshape(nz, ny, nx)


def points3d(atoms, h: float, dims, idx, origin=None, want_sumabs: bool = False):
    """FP64 potential at linear grid indices idx (x fastest); optionally sum_j |q_j|/r_ij."""
    lib = _load()
    a = _atoms(atoms)
    nx, ny, nz = (int(d) for d in dims)
    idx = np.ascontiguousarray(np.asarray(idx, dtype=np.int64).reshape(-1))
    out = np.empty(idx.shape[0], dtype=np.float64)
    sabs = np.empty(idx.shape[0], dtype=np.float64) if want_sumabs else None
    keep, optr = _origin(origin)
    rc = lib.oracle_points3d(a, a.shape[0], np.float32(h), optr, nx, ny, nz, idx, idx.shape[0], out,
                             sabs.ctypes.data_as(ctypes.c_void_p) if sabs is not None else None)
    del keep
    _check(rc, "oracle_points3d")
    return (out, sabs) if want_sumabs else out


def slice2d(atoms_xy_dz2_q, h: float, nx: int, ny: int) -> np.ndarray:
    """FP64 2D slice in KTT's 2D convention (atom .z holds dz^2); shape (ny, nx)."""
    lib = _load()
    a = _atoms(atoms_xy_dz2_q)
    out = np.empty(int(nx) * int(ny), dtype=np.float64)
    _check(lib.oracle_slice2d(a, a.shape[0], np.float32(h), int(nx), int(ny), out), "oracle_slice2d")
    return out.reshape(int(ny), int(nx))


def adjoint3d(atoms, h: float, dims, target, weight=None, sel=None, origin=None, want_map: bool = False):
    """FP64 loss and gradient of L = 0.5*sum w (V - target)^2 wrt charges and positions.

    Returns (loss, dq[nsel], dr[nsel, 3]) and the FP64 map if want_map.
    """
    lib = _load()
    a = _atoms(atoms)
    nx, ny, nz = (int(d) for d in dims)
    total = nx * ny * nz
    tgt = np.ascontiguousarray(np.asarray(target, dtype=np.float32).reshape(-1))
    assert tgt.shape[0] == total
    w = None if weight is None else np.ascontiguousarray(np.asarray(weight, dtype=np.float32).reshape(-1))
    s = None if sel is None else np.ascontiguousarray(np.asarray(sel, dtype=np.int64).reshape(-1))
    m = a.shape[0] if s is None else s.shape[0]
    loss = np.zeros(1, dtype=np.float64)
    dq = np.empty(m, dtype=np.float64)
    dr = np.empty((m, 3), dtype=np.float64)
    vmap = np.empty(total, dtype=np.float64) if want_map else None
    keep, optr = _origin(origin)
    vp = ctypes.c_void_p
    rc = lib.oracle_adjoint3d(a, a.shape[0], np.float32(h), optr, nx, ny, nz,
                              w.ctypes.data_as(vp) if w is not None else None, tgt,
                              s.ctypes.data_as(vp) if s is not None else None, m,
                              loss.ctypes.data_as(vp), dq.ctypes.data_as(vp), dr.ctypes.data_as(vp),
                              vmap.ctypes.data_as(vp) if vmap is not None else None)
    del keep
    _check(rc, "oracle_adjoint3d")
    if want_map:
        return float(loss[0]), dq, dr, vmap.reshape(nz, ny, nx)
    return float(loss[0]), dq, dr


def loss_perturbed(atoms, j: int, new_atom, h: float, dims, target, vmap, weight=None, origin=None) -> float:
    """FP64 loss after replacing atom j by new_atom (x, y, z, q as float64), given the FP64 map."""
    lib = _load()
    a = _atoms(atoms)
    nx, ny, nz = (int(d) for d in dims)
    tgt = np.ascontiguousarray(np.asarray(target, dtype=np.float32).reshape(-1))
    v = np.ascontiguousarray(np.asarray(vmap, dtype=np.float64).reshape(-1))
    w = None if weight is None else np.ascontiguousarray(np.asarray(weight, dtype=np.float32).reshape(-1))
    na = np.ascontiguousarray(np.asarray(new_atom, dtype=np.float64).reshape(4))
    out = np.zeros(1, dtype=np.float64)
    keep, optr = _origin(origin)
    vp = ctypes.c_void_p
    rc = lib.oracle_loss_perturbed(a, a.shape[0], int(j), na, np.float32(h), optr, nx, ny, nz,
                                   w.ctypes.data_as(vp) if w is not None else None, tgt, v, out.ctypes.data_as(vp))
    del keep
    _check(rc, "oracle_loss_perturbed")
    return float(out[0])


def kat_atoms(n: int = 64) -> np.ndarray:
    """The deterministic atoms of KTT's JSON known-answer test (generate-coulomb-output.c:15-20)."""
    out = np.empty(4 * n, dtype=np.float32)
    _load().oracle_kat_atoms(int(n), out)
    return out.reshape(n, 4)


def kat_fp32(atoms, gs: float = 0.49, cells: int = 256, z0: int = 0, z1: int | None = None) -> np.ndarray:
    """FP32 restatement of generate-coulomb-output.c:22-31 for slices [z0, z1); shape (z1-z0, cells, cells)."""
    a = _atoms(atoms)
    z1 = cells if z1 is None else int(z1)
    out = np.empty((z1 - z0) * cells * cells, dtype=np.float32)
    _load().oracle_kat_fp32(a, a.shape[0], np.float32(gs), int(cells), int(z0), z1, out)
    return out.reshape(z1 - z0, cells, cells)


def nbody_step(pos_mass, vel, dt: float, damping: float, softening_sqr: float, idx=None):
    """FP64 N-body step for all bodies or the bodies idx: returns (pos', vel', acc) with shapes
    (k, 4), (k, 4), (k, 3); the j sum always runs over all bodies."""
    lib = _load()
    p = np.ascontiguousarray(np.asarray(pos_mass, dtype=np.float32).reshape(-1, 4))
    v = np.ascontiguousarray(np.asarray(vel, dtype=np.float32).reshape(-1, 4))
    n = p.shape[0]
    if idx is None:
        sel, ptr, k = None, None, n
    else:
        sel = np.ascontiguousarray(np.asarray(idx, dtype=np.int64).reshape(-1))
        ptr, k = sel.ctypes.data_as(ctypes.c_void_p), sel.shape[0]
    pos_out = np.empty((k, 4))
    vel_out = np.empty((k, 4))
    acc = np.empty((k, 3))
    rc = lib.oracle_nbody_step(p.reshape(-1), v.reshape(-1), n, np.float32(dt), np.float32(damping),
                               np.float32(softening_sqr), ptr, k, pos_out.reshape(-1), vel_out.reshape(-1),
                               acc.reshape(-1))
    del sel
    _check(rc, "oracle_nbody_step")
    return pos_out, vel_out, acc
