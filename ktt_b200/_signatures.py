"""ctypes signatures of the C ABI entry points beyond the single-map forward calls."""
import ctypes


class Molecule(ctypes.Structure):
    pass


class NbodyTuneC(ctypes.Structure):
    _fields_ = [("block_x", ctypes.c_int), ("bodies_per_thread", ctypes.c_int), ("unroll", ctypes.c_int),
                ("j_split", ctypes.c_int)]


def register(lib) -> None:
    from . import _Grid, _Tune

    Molecule._fields_ = [("d_atoms", ctypes.c_void_p), ("n_atoms", ctypes.c_int64), ("grid", _Grid),
                         ("d_out", ctypes.c_void_p)]
    vp, ci = ctypes.c_void_p, ctypes.c_int
    sig = {
        "coul_batch_create": [vp, ctypes.POINTER(Molecule), ci, ctypes.POINTER(_Tune), ctypes.POINTER(vp)],
        "coul_batch_destroy": [vp],
        "coul_batch_run": [vp, vp, ci, ci],
        "coul_batch_info": [vp, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ci), ctypes.POINTER(ctypes.c_double)],
        "coul_pack_atoms": [vp, vp, vp, vp, vp, ctypes.c_int64, vp],
        "coul_adjoint_3d": [vp, vp, ctypes.c_int64, ctypes.POINTER(_Grid), vp, vp, vp],
        "coul_nbody_tune_default": [ctypes.POINTER(NbodyTuneC)],
        "coul_nbody_tune_supported": [ctypes.POINTER(NbodyTuneC)],
        "coul_nbody_step": [vp, vp, vp, ctypes.c_int64, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                            ctypes.POINTER(NbodyTuneC), vp, vp],
        "coul_buffer_alloc": [vp, ctypes.c_size_t, ctypes.POINTER(vp)],
        "coul_buffer_free": [vp, vp],
        "coul_buffer_upload": [vp, vp, vp, ctypes.c_size_t],
        "coul_buffer_download": [vp, vp, vp, ctypes.c_size_t],
        "coul_buffer_copy": [vp, vp, vp, ctypes.c_size_t],
        "coul_buffer_memset": [vp, vp, ci, ctypes.c_size_t],
    }
    for name, args in sig.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.argtypes = args
        fn.restype = ci
