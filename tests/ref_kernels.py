"""Test infrastructure: run KTT's own CUDA Coulomb kernels (built by oracle/build_ref_kernels.py into
oracle/_ref/kernels/, the way KTT compiles them) through the CUDA driver API, with KTT's launch
geometry for CoulombSum3d under GlobalSizeType::CUDA and its thread modifiers
(Examples/CoulombSum3d/CoulombSum3d.cpp:70-72, 102, 145-181): block (WGX, WGY, 1), grid
(ceil(G / WGX), ceil(G / WGY), ceil(G / Z_ITERATIONS)); the reference kernel with block (16, 16)
and grid (G / 16, G / 16, G)."""
from __future__ import annotations

import ctypes
import json
import os

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KDIR = os.path.join(REPO, "oracle", "_ref", "kernels")

_modules = {}


def available() -> bool:
    return os.path.exists(os.path.join(KDIR, "manifest.json"))


def space():
    """KTT's 210-configuration CUDA space for CoulombSum3d as dicts (Z, IUF, SOA, WGX, WGY)."""
    out = []
    for z in (1, 2, 4, 8, 16, 32):
        for u in (0, 1, 2, 4, 8, 16, 32):
            if u >= z:
                continue
            for s in (0, 1):
                for wx in (16, 32):
                    for wy in (1, 2, 4, 8):
                        if wx * wy >= 64:
                            out.append({"WORK_GROUP_SIZE_X": wx, "WORK_GROUP_SIZE_Y": wy, "Z_ITERATIONS": z,
                                        "INNER_UNROLL_FACTOR": u, "USE_SOA": s})
    return out


def _check(res):
    from cuda.bindings import driver as cu
    err = res[0] if isinstance(res, tuple) else res
    if err != cu.CUresult.CUDA_SUCCESS:
        raise RuntimeError(f"CUDA driver call failed: {err}")
    return res[1] if isinstance(res, tuple) and len(res) > 1 else None


def _function(fname: str, kernel: str):
    from cuda.bindings import driver as cu
    if fname not in _modules:
        mod = _check(cu.cuModuleLoad(os.path.join(KDIR, fname).encode()))
        _modules[fname] = mod
    # kernels that are not extern "C" are looked up by the lowered name recorded at build time
    kernel = manifest()["kernels"].get(fname, {}).get("function", kernel)
    return _check(cu.cuModuleGetFunction(_modules[fname], kernel.encode()))


def run_tuned(cfg: dict, atoms, soa_cols, n_atoms: int, spacing: float, grid: int, out, stream=None):
    """One launch of directCoulombSum (out += V).  atoms: (n, 4) float32 CUDA tensor; soa_cols: four
    float32 CUDA tensors (x, y, z, w); out: grid^3 float32 CUDA tensor."""
    import torch
    from cuda.bindings import driver as cu
    fn = _function(f"coulomb3d_z{cfg['Z_ITERATIONS']}_u{cfg['INNER_UNROLL_FACTOR']}_soa{cfg['USE_SOA']}.cubin",
                   "directCoulombSum")
    wx, wy, z = cfg["WORK_GROUP_SIZE_X"], cfg["WORK_GROUP_SIZE_Y"], cfg["Z_ITERATIONS"]
    s = stream or torch.cuda.current_stream()
    args = ((atoms.data_ptr(), *(c.data_ptr() for c in soa_cols), int(n_atoms), float(spacing), int(grid),
             out.data_ptr()),
            (ctypes.c_void_p,) * 5 + (ctypes.c_int, ctypes.c_float, ctypes.c_int, ctypes.c_void_p))
    _check(cu.cuLaunchKernel(fn, -(-grid // wx), -(-grid // wy), -(-grid // z), wx, wy, 1, 0,
                             cu.CUstream(s.cuda_stream), args, 0))


def run_reference(atoms, n_atoms: int, spacing: float, grid: int, out, stream=None):
    """One launch of directCoulombSumReference (out += V); grid must be a multiple of 16."""
    import torch
    from cuda.bindings import driver as cu
    if grid % 16:
        raise ValueError("the reference kernel's launch needs a grid size that is a multiple of 16")
    fn = _function("coulomb3d_reference.cubin", "directCoulombSumReference")
    s = stream or torch.cuda.current_stream()
    args = ((atoms.data_ptr(), int(n_atoms), float(spacing), int(grid), out.data_ptr()),
            (ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_int, ctypes.c_void_p))
    _check(cu.cuLaunchKernel(fn, grid // 16, grid // 16, grid, 16, 16, 1, 0, cu.CUstream(s.cuda_stream), args, 0))


def manifest() -> dict:
    with open(os.path.join(KDIR, "manifest.json")) as f:
        return json.load(f)


# ---- KTT's N-body example (Examples/Nbody) ----

class DeviceLimitsExceeded(Exception):
    """The configuration cannot be launched on this device (KTT's ResultStatus::DeviceLimitsExceeded)."""

def nbody_configs():
    """The compiled sample of the tuned N-body kernel's space (manifest entries), as dicts."""
    return [dict(v) for k, v in manifest()["kernels"].items() if k.startswith("nbody_") and "reference" not in v]


def _nbody_name(cfg):
    keys = ("WORK_GROUP_SIZE_X", "WORK_GROUP_SIZE_Y", "OUTER_UNROLL_FACTOR", "INNER_UNROLL_FACTOR1",
            "INNER_UNROLL_FACTOR2", "USE_SOA", "LOCAL_MEM", "USE_CONSTANT_MEMORY", "VECTOR_TYPE")
    return "nbody_" + "_".join(str(cfg[k]) for k in keys) + ".cubin"


def run_nbody_tuned(cfg, dt, pos4, posx, posy, posz, mass, new_pos4, vel4, velx, vely, velz, new_vel4, damping,
                    eps2, n, stream=None):
    """One launch of KTT's nbody_kernel (Examples/Nbody/Nbody.cu:260-275) with the example's launch
    geometry (Examples/Nbody/Nbody.cpp:126-160, OpenCL global size n x 1): grid n / (OUTER_UNROLL_FACTOR *
    WORK_GROUP_SIZE_X), block (WORK_GROUP_SIZE_X, WORK_GROUP_SIZE_Y).  n must be a multiple of
    WORK_GROUP_SIZE_X * OUTER_UNROLL_FACTOR and of WORK_GROUP_SIZE_X * VECTOR_TYPE."""
    import torch
    from cuda.bindings import driver as cu
    wx, wy, ouf, vt = cfg["WORK_GROUP_SIZE_X"], cfg["WORK_GROUP_SIZE_Y"], cfg["OUTER_UNROLL_FACTOR"], cfg["VECTOR_TYPE"]
    if n % (wx * ouf) or n % (wx * vt):
        raise ValueError("body count not divisible by the configuration's tile")
    fn = _function(_nbody_name(cfg), "nbody_kernel")
    # a block beyond what the compiled kernel's registers allow is KTT's DeviceLimitsExceeded: refuse it
    # before launching rather than let the launch fail
    limit = _check(cu.cuFuncGetAttribute(cu.CUfunction_attribute.CU_FUNC_ATTRIBUTE_MAX_THREADS_PER_BLOCK, fn))
    if wx * wy > limit:
        raise DeviceLimitsExceeded(f"{wx * wy} threads per block, the kernel allows {limit}")
    s = stream or torch.cuda.current_stream()
    ptrs = [pos4, posx, posy, posz, mass, new_pos4, vel4, velx, vely, velz, new_vel4]
    args = ((float(dt), *(t.data_ptr() for t in ptrs), float(damping), float(eps2), int(n)),
            (ctypes.c_float,) + (ctypes.c_void_p,) * 11 + (ctypes.c_float, ctypes.c_float, ctypes.c_int))
    _check(cu.cuLaunchKernel(fn, n // (wx * ouf), 1, 1, wx, wy, 1, 0, cu.CUstream(s.cuda_stream), args, 0))


def run_nbody_reference(dt, pos4, new_pos4, vel4, new_vel4, damping, eps2, n, stream=None):
    """One launch of nbody_kernel_reference (Examples/Nbody/NbodyReference.cu:36-75) with the example's
    64-thread blocks; n must be a multiple of 64."""
    import torch
    from cuda.bindings import driver as cu
    if n % 64:
        raise ValueError("the reference N-body kernel needs a multiple of 64 bodies")
    fn = _function("nbody_reference.cubin", "nbody_kernel_reference")
    s = stream or torch.cuda.current_stream()
    args = ((float(dt), pos4.data_ptr(), new_pos4.data_ptr(), vel4.data_ptr(), new_vel4.data_ptr(), float(damping),
             float(eps2)),
            (ctypes.c_float,) + (ctypes.c_void_p,) * 4 + (ctypes.c_float, ctypes.c_float))
    _check(cu.cuLaunchKernel(fn, n // 64, 1, 1, 64, 1, 1, 0, cu.CUstream(s.cuda_stream), args, 0))
