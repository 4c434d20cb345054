"""ktt_b200 -- B200-native direct Coulomb summation behind a KTT-compatible surface.

Python binding of the C ABI in ``include/coulktt.h`` (``libcoulktt.so``,
built by ``python -m ktt_b200.build``).  Tensors are PyTorch CUDA tensors;
PyTorch provides device memory and streams only -- every computation runs in
the library's own sm_100a kernels.  There is no CPU fallback: if the library
or a B200 is missing, the calls raise.

The C++ ``ktt::Tuner`` surface (``include/Ktt.h``, ``libktt_b200.so``) is
the drop-in for KTT host programs; this module is the drop-in for KTT's
Python examples (``Examples/CoulombSum2d/CoulombSum2d.py``) at the level of
the kernel call, and hosts the ``torch.autograd.Function`` of the adjoint.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field, fields

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcoulktt.so")

COUL_OK = 0
COUL_ERR_INVALID_ARGUMENT = 1
COUL_ERR_CUDA = 2
COUL_ERR_UNSUPPORTED = 3
COUL_ERR_DEVICE_LIMITS = 4
COUL_ERR_TIMEOUT = 5
COUL_ERR_NO_DEVICE = 6
COUL_ERR_OUT_OF_MEMORY = 7

ATOMS_SHARED_TMA = 0
ATOMS_CONSTANT = 1
PREC_FP32 = 0
PREC_COMPENSATED = 1
PREC_FP64_MERGE = 2
PREC_FP64_PAIRS = 3
PREC_FP64_MERGE_SHARED = 4  # PREC_FP64_MERGE with the FP64 sums in shared memory (same values, fewer registers)


class CoulombError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


class _Tune(ctypes.Structure):
    _fields_ = [("block_x", ctypes.c_int), ("block_y", ctypes.c_int), ("z_iterations", ctypes.c_int),
                ("x_points", ctypes.c_int), ("unroll", ctypes.c_int), ("atom_source", ctypes.c_int),
                ("precision", ctypes.c_int), ("rsqrt_soft", ctypes.c_int), ("atom_split", ctypes.c_int),
                ("split_form", ctypes.c_int)]


class _PipeRates(ctypes.Structure):
    _fields_ = [("rsqrt_per_s", ctypes.c_double), ("ffma_per_s", ctypes.c_double),
                ("ffma2_lanes_per_s", ctypes.c_double), ("dfma_per_s", ctypes.c_double),
                ("rsqrt_mix6_per_s", ctypes.c_double), ("sm_count", ctypes.c_int),
                ("max_sm_clock_khz", ctypes.c_int)]


class _Grid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("spacing", ctypes.c_float),
                ("origin", ctypes.c_float * 3)]


@dataclass
class Tune:
    """Forward-kernel configuration; field names follow coul_tune (KTT parameter in brackets).

    block_x [WORK_GROUP_SIZE_X], block_y [WORK_GROUP_SIZE_Y], z_iterations [Z_ITERATIONS],
    x_points [VECTOR_SIZE / OUTER_UNROLL_FACTOR], unroll [INNER_UNROLL_FACTOR],
    atom_source [USE_CONSTANT_MEMORY], precision, rsqrt_soft, atom_split (atom chunks per point tile
    in the atom-split form, or atom groups per CTA in its balanced form; 0 = off), split_form (0: a
    thread-block cluster per tile, 1: a persistent grid over (tile, chunk) items from a device queue,
    2: a resident grid whose CTAs take equal ranges of the (tile, atom) space, the block being
    block_x x block_y x atom_split threads).
    """
    block_x: int = 32
    block_y: int = 4
    z_iterations: int = 16
    x_points: int = 4
    unroll: int = 1
    atom_source: int = ATOMS_SHARED_TMA
    precision: int = PREC_FP32
    rsqrt_soft: int = 0
    atom_split: int = 0
    split_form: int = 0

    def c(self) -> _Tune:
        return _Tune(*(int(getattr(self, f.name)) for f in fields(self)))

    def as_dict(self) -> dict:
        return {f.name: int(getattr(self, f.name)) for f in fields(self)}


def tuned(name: str, key: str = "tune") -> Tune | None:
    """A configuration the autotuner stored under ktt_b200/tuned/<name>.json (None if absent)."""
    import json
    path = os.path.join(os.path.dirname(__file__), "tuned", name + ".json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        entry = json.load(f).get(key)
    return Tune(**entry) if entry else None


_lib = None


def library_path() -> str:
    return LIB_PATH


def load_library():
    """Load libcoulktt.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise CoulombError(COUL_ERR_NO_DEVICE, f"{LIB_PATH} is missing; run `python -m ktt_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    vp, i64, ci, cf = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_float
    T, G = ctypes.POINTER(_Tune), ctypes.POINTER(_Grid)
    sig = {
        "coul_ctx_create": [ci, ctypes.POINTER(vp)],
        "coul_ctx_destroy": [vp],
        "coul_ctx_set_stream": [vp, vp],
        "coul_ctx_device_info": [vp, ctypes.POINTER(ci), ctypes.POINTER(ci), ctypes.POINTER(ci)],
        "coul_synchronize": [vp],
        "coul_elapsed_ms": [vp, ctypes.POINTER(ctypes.c_double)],
        "coul_tune_supported": [T],
        "coul_tune_supported_2d": [T],
        "coul_batch_tune_supported": [T],
        "coul_variant_count": [],
        "coul_variant_get": [ci, T, ctypes.POINTER(ci), ctypes.POINTER(ci)],
        "coul_forward_3d": [vp, vp, i64, G, T, ci, vp],
        "coul_forward_3d_slab": [vp, vp, i64, G, ci, ci, T, ci, vp],
        "coul_forward_3d_soa": [vp, vp, vp, vp, vp, i64, G, T, ci, vp],
        "coul_forward_3d_reference": [vp, vp, i64, G, ci, vp],
        "coul_forward_3d_reference_fp64": [vp, vp, i64, G, vp],
        "coul_forward_2d": [vp, vp, i64, cf, ci, ci, T, ci, vp],
        "coul_slice_atoms": [vp, vp, i64, cf, vp],
        "coul_forward_3d_host": [vp, vp, i64, G, T, vp],
        "coul_probe_bounded_wait": [vp, ci, ctypes.c_uint64],
        "coul_measure_pipe_rates": [vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)],
        "coul_measure_pipe_rates_ex": [vp, ctypes.POINTER(_PipeRates)],
    }
    for name, args in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = ci
    for name in ("coul_ctx_get_stream", "coul_ctx_own_stream"):
        getattr(lib, name).argtypes = [vp]
        getattr(lib, name).restype = vp
    lib.coul_last_error.restype = ctypes.c_char_p
    lib.coul_status_string.argtypes = [ci]
    lib.coul_status_string.restype = ctypes.c_char_p
    lib.coul_tune_default.argtypes = [T]
    lib.coul_tune_default.restype = None
    _register_optional(lib)
    _lib = lib
    return lib


def _register_optional(lib) -> None:
    """Signatures of entry points added by later units (batched, adjoint, ...)."""
    try:
        from . import _signatures  # noqa: F401
        _signatures.register(lib)
    except ImportError:
        pass


def _check(rc: int) -> None:
    if rc != COUL_OK:
        msg = _lib.coul_last_error().decode(errors="replace") if _lib is not None else ""
        raise CoulombError(rc, msg or "error")


def variants() -> list[tuple[Tune, bool, bool]]:
    """All compiled forward variants as (tune, is_2d, is_soa)."""
    lib = load_library()
    out = []
    for i in range(lib.coul_variant_count()):
        t = _Tune()
        d2, soa = ctypes.c_int(), ctypes.c_int()
        _check(lib.coul_variant_get(i, ctypes.byref(t), ctypes.byref(d2), ctypes.byref(soa)))
        out.append((Tune(*(getattr(t, n) for n, _ in _Tune._fields_)), bool(d2.value), bool(soa.value)))
    return out


def tune_supported(tune: Tune) -> bool:
    lib = load_library()
    return lib.coul_tune_supported(ctypes.byref(tune.c())) == COUL_OK


def batch_tune_supported(tune: Tune) -> bool:
    """Whether the persistent batched kernel has a compiled variant for this tile shape."""
    return load_library().coul_batch_tune_supported(ctypes.byref(tune.c())) == COUL_OK


def tune_supported_2d(tune: Tune) -> bool:
    """Whether coul_forward_2d has a compiled variant for this configuration."""
    lib = load_library()
    return lib.coul_tune_supported_2d(ctypes.byref(tune.c())) == COUL_OK


def _grid(dims, spacing, origin) -> _Grid:
    nx, ny, nz = (int(d) for d in dims)
    o = (0.0, 0.0, 0.0) if origin is None else tuple(float(v) for v in origin)
    return _Grid(nx, ny, nz, float(spacing), (ctypes.c_float * 3)(*o))


def _ptr(t) -> int:
    return int(t.data_ptr())


class CoulombContext:
    """One CUDA device; calls are enqueued on PyTorch's current stream of that device."""

    def __init__(self, device: int = 0):
        self._lib = load_library()
        self._ctx = ctypes.c_void_p()
        _check(self._lib.coul_ctx_create(int(device), ctypes.byref(self._ctx)))
        self.device = int(device)
        sm, ma, mi = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(self._lib.coul_ctx_device_info(self._ctx, ctypes.byref(sm), ctypes.byref(ma), ctypes.byref(mi)))
        self.sm_count, self.cc = sm.value, (ma.value, mi.value)

    # -- plumbing ---------------------------------------------------------------------------
    def close(self) -> None:
        if self._ctx:
            self._lib.coul_ctx_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._ctx

    def _bind_stream(self) -> None:
        import torch
        s = torch.cuda.current_stream(self.device)
        _check(self._lib.coul_ctx_set_stream(self._ctx, ctypes.c_void_p(s.cuda_stream)))

    def probe_bounded_wait(self, arrive: bool, budget_ns: int) -> int:
        """Status of the bounded-wait self-test kernel (COUL_OK, or COUL_ERR_TIMEOUT when nothing arrives)."""
        return int(self._lib.coul_probe_bounded_wait(self._ctx, 1 if arrive else 0, int(budget_ns)))

    def pipe_rates(self) -> tuple[float, float]:
        """(MUFU rsqrt/s, FP32 FMA/s) of the whole GPU, measured now by throughput microkernels (the
        FMA rate is the larger of the scalar and the packed-FFMA2 rate)."""
        m, f = ctypes.c_double(), ctypes.c_double()
        _check(self._lib.coul_measure_pipe_rates(self._ctx, ctypes.byref(m), ctypes.byref(f)))
        return m.value, f.value

    def pipe_rates_ex(self) -> dict:
        """All pipe rates of coul_measure_pipe_rates_ex (per second, whole GPU) with the SM count and
        the maximum SM clock."""
        r = _PipeRates()
        _check(self._lib.coul_measure_pipe_rates_ex(self._ctx, ctypes.byref(r)))
        return {name: getattr(r, name) for name, _ in _PipeRates._fields_}

    def synchronize(self) -> None:
        _check(self._lib.coul_synchronize(self._ctx))

    def elapsed_ms(self) -> float:
        ms = ctypes.c_double()
        _check(self._lib.coul_elapsed_ms(self._ctx, ctypes.byref(ms)))
        return ms.value

    @staticmethod
    def _check_atoms(atoms, cols: int = 4):
        import torch
        if not (isinstance(atoms, torch.Tensor) and atoms.is_cuda and atoms.dtype == torch.float32):
            raise CoulombError(COUL_ERR_INVALID_ARGUMENT, "atoms must be a float32 CUDA tensor")
        if atoms.dim() != 2 or atoms.shape[1] != cols or not atoms.is_contiguous():
            raise CoulombError(COUL_ERR_INVALID_ARGUMENT, f"atoms must be a contiguous (n, {cols}) tensor")

    @staticmethod
    def _out(out, shape, device):
        import torch
        if out is None:
            return torch.empty(shape, dtype=torch.float32, device=device)
        if tuple(out.shape) != tuple(shape) or out.dtype != torch.float32 or not out.is_contiguous():
            raise CoulombError(COUL_ERR_INVALID_ARGUMENT, f"out must be a contiguous float32 tensor of shape {shape}")
        return out

    # -- forward ------------------------------------------------------------------------------
    def forward_3d(self, atoms, dims, spacing, origin=None, tune: Tune | None = None, out=None,
                   accumulate: bool = False):
        """Map of shape (nz, ny, nx) for dims = (nx, ny, nz)."""
        self._check_atoms(atoms)
        nx, ny, nz = (int(d) for d in dims)
        out = self._out(out, (nz, ny, nx), atoms.device)
        self._bind_stream()
        g = _grid(dims, spacing, origin)
        t = (tune or Tune()).c()
        _check(self._lib.coul_forward_3d(self._ctx, _ptr(atoms), atoms.shape[0], ctypes.byref(g), ctypes.byref(t),
                                         1 if accumulate else 0, _ptr(out)))
        return out

    def forward_3d_slab(self, atoms, dims, spacing, z_begin: int, z_end: int, origin=None,
                        tune: Tune | None = None, out=None, accumulate: bool = False):
        """Slab z in [z_begin, z_end) of the map of dims = (nx, ny, nz): shape (z_end - z_begin, ny, nx),
        the full grid's point coordinates (slabs starting at multiples of tune.z_iterations put together
        equal forward_3d bit for bit)."""
        self._check_atoms(atoms)
        nx, ny, nz = (int(d) for d in dims)
        out = self._out(out, (int(z_end) - int(z_begin), ny, nx), atoms.device)
        self._bind_stream()
        g = _grid(dims, spacing, origin)
        t = (tune or Tune()).c()
        _check(self._lib.coul_forward_3d_slab(self._ctx, _ptr(atoms), atoms.shape[0], ctypes.byref(g), int(z_begin),
                                              int(z_end), ctypes.byref(t), 1 if accumulate else 0, _ptr(out)))
        return out

    def forward_3d_soa(self, x, y, z, q, dims, spacing, origin=None, tune: Tune | None = None, out=None,
                       accumulate: bool = False):
        nx, ny, nz = (int(d) for d in dims)
        out = self._out(out, (nz, ny, nx), x.device)
        self._bind_stream()
        g = _grid(dims, spacing, origin)
        t = (tune or Tune()).c()
        _check(self._lib.coul_forward_3d_soa(self._ctx, _ptr(x), _ptr(y), _ptr(z), _ptr(q), x.shape[0],
                                             ctypes.byref(g), ctypes.byref(t), 1 if accumulate else 0, _ptr(out)))
        return out

    def forward_3d_reference(self, atoms, dims, spacing, origin=None, out=None, accumulate: bool = False):
        self._check_atoms(atoms)
        nx, ny, nz = (int(d) for d in dims)
        out = self._out(out, (nz, ny, nx), atoms.device)
        self._bind_stream()
        g = _grid(dims, spacing, origin)
        _check(self._lib.coul_forward_3d_reference(self._ctx, _ptr(atoms), atoms.shape[0], ctypes.byref(g),
                                                   1 if accumulate else 0, _ptr(out)))
        return out

    def forward_3d_reference_fp64(self, atoms, dims, spacing, origin=None, out=None):
        """The map in FP64 (float64 tensor of shape (nz, ny, nx)), one point per thread: the
        validation kernel of coul_forward_3d_reference_fp64."""
        import torch
        self._check_atoms(atoms)
        nx, ny, nz = (int(d) for d in dims)
        if out is None:
            out = torch.empty((nz, ny, nx), dtype=torch.float64, device=atoms.device)
        elif out.dtype != torch.float64 or not out.is_contiguous() or out.numel() != nx * ny * nz:
            raise ValueError("out must be a contiguous float64 tensor of nx * ny * nz elements")
        self._bind_stream()
        g = _grid(dims, spacing, origin)
        _check(self._lib.coul_forward_3d_reference_fp64(self._ctx, _ptr(atoms), atoms.shape[0], ctypes.byref(g),
                                                        _ptr(out)))
        return out

    def forward_2d(self, atoms_xy_dz2_q, spacing, nx, ny, tune: Tune | None = None, out=None,
                   accumulate: bool = False):
        """Slice of shape (ny, nx) in KTT's 2D convention (atom column 2 holds dz^2)."""
        self._check_atoms(atoms_xy_dz2_q)
        out = self._out(out, (int(ny), int(nx)), atoms_xy_dz2_q.device)
        self._bind_stream()
        t = (tune or Tune(block_x=32, block_y=4, z_iterations=4, x_points=4)).c()
        _check(self._lib.coul_forward_2d(self._ctx, _ptr(atoms_xy_dz2_q), atoms_xy_dz2_q.shape[0], float(spacing),
                                         int(nx), int(ny), ctypes.byref(t), 1 if accumulate else 0, _ptr(out)))
        return out

    def slice_atoms(self, atoms, z_slice: float, out=None):
        import torch
        self._check_atoms(atoms)
        out = torch.empty_like(atoms) if out is None else out
        self._bind_stream()
        _check(self._lib.coul_slice_atoms(self._ctx, _ptr(atoms), atoms.shape[0], float(z_slice), _ptr(out)))
        return out

    def forward_3d_host(self, atoms_np, dims, spacing, origin=None, tune: Tune | None = None, out_np=None):
        """Host (numpy) buffers in and out; copies are part of the call (KTT Tuner::Run semantics)."""
        import numpy as np
        a = np.ascontiguousarray(np.asarray(atoms_np, dtype=np.float32).reshape(-1, 4))
        nx, ny, nz = (int(d) for d in dims)
        out = np.empty((nz, ny, nx), dtype=np.float32) if out_np is None else out_np
        assert out.flags.c_contiguous and out.dtype == np.float32 and out.size == nx * ny * nz
        g = _grid(dims, spacing, origin)
        t = (tune or Tune()).c()
        _check(self._lib.coul_forward_3d_host(self._ctx, a.ctypes.data, a.shape[0], ctypes.byref(g), ctypes.byref(t),
                                              out.ctypes.data))
        return out


@dataclass
class NbodyTune:
    """N-body step configuration (coul_nbody_tune; KTT parameter in brackets): block_x
    [WORK_GROUP_SIZE_X], bodies_per_thread [OUTER_UNROLL_FACTOR], unroll [INNER_UNROLL_FACTOR1],
    j_split (cluster of CTAs sharing a tile of bodies, splitting the bodies j) [WORK_GROUP_SIZE_Y]."""
    block_x: int = 128
    bodies_per_thread: int = 4
    unroll: int = 2
    j_split: int = 0

    def c(self):
        from ._signatures import NbodyTuneC
        return NbodyTuneC(self.block_x, self.bodies_per_thread, self.unroll, self.j_split)


def nbody_tune_supported(tune: NbodyTune) -> bool:
    return load_library().coul_nbody_tune_supported(ctypes.byref(tune.c())) == COUL_OK


def nbody_step(ctx: "CoulombContext", pos_mass, vel, dt: float, damping: float, softening_sqr: float,
               tune: NbodyTune | None = None, out_pos=None, out_vel=None):
    """One step of KTT's N-body example (coul_nbody_step): pos_mass and vel are (n, 4) float32 CUDA
    tensors; returns (pos_mass', vel')."""
    import torch
    CoulombContext._check_atoms(pos_mass)
    CoulombContext._check_atoms(vel)
    n = pos_mass.shape[0]
    if vel.shape[0] != n:
        raise CoulombError(COUL_ERR_INVALID_ARGUMENT, "pos_mass and vel must hold the same number of bodies")
    out_pos = torch.empty_like(pos_mass) if out_pos is None else out_pos
    out_vel = torch.empty_like(vel) if out_vel is None else out_vel
    ctx._bind_stream()
    t = (tune or NbodyTune()).c()
    _check(ctx._lib.coul_nbody_step(ctx.handle, _ptr(pos_mass), _ptr(vel), n, float(dt), float(damping),
                                    float(softening_sqr), ctypes.byref(t), _ptr(out_pos), _ptr(out_vel)))
    return out_pos, out_vel


def adjoint_3d(ctx: "CoulombContext", atoms, dims, spacing, grad_map, origin=None):
    """dL/dr and dL/dq for G = dL/dV on the map: returns an (n, 4) tensor (dx, dy, dz, dq)."""
    import torch
    CoulombContext._check_atoms(atoms)
    nx, ny, nz = (int(d) for d in dims)
    g = grad_map.contiguous().to(torch.float32)
    if g.numel() != nx * ny * nz or not g.is_cuda:
        raise CoulombError(COUL_ERR_INVALID_ARGUMENT, "grad_map must be a CUDA tensor with nx*ny*nz elements")
    n = atoms.shape[0]
    grad_q = torch.empty(n, dtype=torch.float32, device=atoms.device)
    grad_xyz = torch.empty((n, 3), dtype=torch.float32, device=atoms.device)
    ctx._bind_stream()
    grid = _grid(dims, spacing, origin)
    _check(ctx._lib.coul_adjoint_3d(ctx.handle, _ptr(atoms), n, ctypes.byref(grid), _ptr(g), _ptr(grad_q),
                                    _ptr(grad_xyz)))
    return torch.cat([grad_xyz, grad_q[:, None]], dim=1)


def _autograd_function():
    import torch

    class CoulombMapFunction(torch.autograd.Function):
        """V = map(atoms) with atoms (n, 4) = (x, y, z, q); backward through the sm_100a adjoint
        kernel (1/r recomputed, FP64 partial sums) -- gradients for positions and charges."""

        @staticmethod
        def forward(fctx, atoms, ctx, dims, spacing, origin, tune):
            a = atoms.detach().contiguous()
            out = ctx.forward_3d(a, dims, spacing, origin, tune=tune)
            fctx.save_for_backward(a)
            fctx.coul = (ctx, dims, spacing, origin)
            return out

        @staticmethod
        def backward(fctx, grad_out):
            (a,) = fctx.saved_tensors
            ctx, dims, spacing, origin = fctx.coul
            grad = adjoint_3d(ctx, a, dims, spacing, grad_out, origin)
            return grad, None, None, None, None, None

    return CoulombMapFunction


_MAP_FUNCTION = None


def coulomb_map(atoms, ctx: "CoulombContext", dims, spacing, origin=None, tune: Tune | None = None):
    """Differentiable potential map: a torch.autograd.Function over the forward and adjoint kernels.

    atoms: (n, 4) float32 CUDA tensor (x, y, z, q), may require grad; returns (nz, ny, nx)."""
    global _MAP_FUNCTION
    if _MAP_FUNCTION is None:
        _MAP_FUNCTION = _autograd_function()
    return _MAP_FUNCTION.apply(atoms, ctx, tuple(int(d) for d in dims), float(spacing), origin, tune)


BATCH_PERSISTENT = 0
BATCH_GRAPH = 1
BATCH_SEPARATE = 2


class Batch:
    """Many molecules evaluated by one persistent launch from a (molecule, tile) work queue.

    molecules: list of (atoms (n, 4) float32 CUDA tensor, dims (nx, ny, nz), spacing, origin).
    The batch allocates one output map per molecule (``outputs``, shapes (nz, ny, nx)).
    """

    def __init__(self, ctx: "CoulombContext", molecules, tune: Tune | None = None):
        import torch
        from ._signatures import Molecule
        self._ctx = ctx
        self._lib = ctx._lib
        self.atoms = [m[0] for m in molecules]
        self.outputs = []
        arr = (Molecule * len(molecules))()
        for i, (atoms, dims, spacing, origin) in enumerate(molecules):
            CoulombContext._check_atoms(atoms)
            nx, ny, nz = (int(d) for d in dims)
            out = torch.empty((nz, ny, nx), dtype=torch.float32, device=atoms.device)
            self.outputs.append(out)
            arr[i].d_atoms = atoms.data_ptr()
            arr[i].n_atoms = atoms.shape[0]
            arr[i].grid = _grid(dims, spacing, origin)
            arr[i].d_out = out.data_ptr()
        self.tune = tune or tuned("b200_batch", "batched") or Tune(z_iterations=8, x_points=2, unroll=2,
                                                                  rsqrt_soft=2)
        t = self.tune.c()
        self._handle = ctypes.c_void_p()
        ctx._bind_stream()
        _check(self._lib.coul_batch_create(ctx.handle, arr, len(molecules), ctypes.byref(t), ctypes.byref(self._handle)))
        items, ctas, pairs = ctypes.c_int64(), ctypes.c_int(), ctypes.c_double()
        _check(self._lib.coul_batch_info(self._handle, ctypes.byref(items), ctypes.byref(ctas), ctypes.byref(pairs)))
        self.work_items, self.grid_ctas, self.total_pairs = items.value, ctas.value, pairs.value

    def run(self, mode: int = BATCH_PERSISTENT, accumulate: bool = False) -> None:
        self._ctx._bind_stream()
        _check(self._lib.coul_batch_run(self._ctx.handle, self._handle, int(mode), 1 if accumulate else 0))

    def close(self) -> None:
        if self._handle:
            self._lib.coul_batch_destroy(self._handle)
            self._handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
