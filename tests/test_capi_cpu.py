"""C ABI checks that need no GPU: the library loads, exports every entry point the
public headers declare, and validates configurations before any device work."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

import ktt_b200

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols(header: str) -> list[str]:
    text = open(header).read()
    return sorted(set(re.findall(r"COUL_API\s+[\w\s\*]+?\b(coul_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = ktt_b200.load_library()
    names = []
    for h in glob.glob(os.path.join(REPO, "include", "*.h")):
        names += declared_symbols(h)
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_no_cpu_fallback_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(ktt_b200.CoulombError) as e:
        ktt_b200.CoulombContext(0)
    assert e.value.status == ktt_b200.COUL_ERR_NO_DEVICE


def test_tune_validation_without_device():
    T = ktt_b200.Tune
    assert ktt_b200.tune_supported(T())
    assert ktt_b200.tune_supported(T(z_iterations=32, x_points=1, unroll=8))
    assert ktt_b200.tune_supported(T(atom_source=ktt_b200.ATOMS_CONSTANT, z_iterations=4, x_points=2))
    assert not ktt_b200.tune_supported(T(z_iterations=3))              # no such variant
    assert not ktt_b200.tune_supported(T(block_x=64, block_y=8))       # 512 threads > launch bound
    assert not ktt_b200.tune_supported(T(precision=7))
    lib = ktt_b200.load_library()
    t = T(block_x=0).c()
    assert lib.coul_tune_supported(ctypes.byref(t)) == ktt_b200.COUL_ERR_DEVICE_LIMITS
    assert b"block" in lib.coul_last_error()
    # atom-split form: cluster sizes 2..16 (above 8 non-portable), FP32 shared-memory atoms only
    split = dict(z_iterations=8, x_points=2, rsqrt_soft=2)
    for s in (2, 3, 5, 8, 9, 16):
        assert ktt_b200.tune_supported(T(atom_split=s, **split))
    assert ktt_b200.tune_supported(T(atom_split=1, z_iterations=16, x_points=4))  # 1 = off
    assert not ktt_b200.tune_supported(T(atom_split=17, **split))
    assert not ktt_b200.tune_supported(T(atom_split=-1, **split))
    assert not ktt_b200.tune_supported(T(atom_split=4, precision=ktt_b200.PREC_FP64_MERGE, **split))
    assert not ktt_b200.tune_supported(T(atom_split=4, z_iterations=4, x_points=1,
                                         atom_source=ktt_b200.ATOMS_CONSTANT))
    assert ktt_b200.tune_supported_2d(T(z_iterations=2, x_points=1, atom_split=4))
    assert ktt_b200.tune_supported_2d(T(z_iterations=4, x_points=4))
    assert not ktt_b200.tune_supported_2d(T(z_iterations=8, x_points=2, atom_split=4))
    # the queue form of the atom split: any chunk count 2..256, no clusters
    for s in (2, 17, 64, 256):
        assert ktt_b200.tune_supported(T(atom_split=s, split_form=1, **split))
        assert ktt_b200.tune_supported_2d(T(z_iterations=4, x_points=2, rsqrt_soft=2, atom_split=s, split_form=1))
    assert not ktt_b200.tune_supported(T(atom_split=257, split_form=1, **split))
    assert not ktt_b200.tune_supported(T(atom_split=4, split_form=1, precision=ktt_b200.PREC_FP64_MERGE, **split))
    # the balanced form: 2..32 atom groups per CTA, tile threads x groups <= 1024
    for g in (2, 4, 16, 32):
        assert ktt_b200.tune_supported(T(block_x=32, block_y=1, atom_split=g, split_form=2, **split))
        assert ktt_b200.tune_supported_2d(T(block_x=32, block_y=1, z_iterations=4, x_points=2, rsqrt_soft=2,
                                            atom_split=g, split_form=2))
    assert ktt_b200.tune_supported(T(block_x=32, block_y=4, atom_split=8, split_form=2, **split))
    assert not ktt_b200.tune_supported(T(block_x=32, block_y=4, atom_split=16, split_form=2, **split))
    assert not ktt_b200.tune_supported(T(block_x=32, block_y=1, atom_split=33, split_form=2, **split))
    assert not ktt_b200.tune_supported(T(atom_split=4, split_form=3, **split))
    assert not ktt_b200.tune_supported(T(block_x=32, block_y=1, atom_split=4, split_form=2,
                                         precision=ktt_b200.PREC_COMPENSATED, **split))


def test_variant_inventory():
    vs = ktt_b200.variants()
    assert len(vs) == ktt_b200.load_library().coul_variant_count()
    keys = {(t.z_iterations, t.x_points, t.unroll, t.atom_source, t.precision, t.rsqrt_soft, d2, soa)
            for t, d2, soa in vs if t.atom_split == 0}
    split_keys = {(t.z_iterations, t.x_points, t.unroll, t.rsqrt_soft, t.split_form, d2)
                  for t, d2, soa in vs if t.atom_split}
    assert len(keys) + len(split_keys) == len(vs)  # no duplicates
    # the atom-split forms (cluster, queue, balanced): FP32, float4 atoms through shared memory, 2D and 3D
    assert all(t.precision == 0 and t.atom_source == 0 and not soa for t, _, soa in vs if t.atom_split)
    for form in (0, 1, 2):
        assert any(d2 for *_, f, d2 in split_keys if f == form) and any(not d2 for *_, f, d2 in split_keys if f == form)
    # the KTT CUDA space of CoulombSum3d.cpp: Z_ITERATIONS x unroll x USE_SOA, all present for x_points 1
    for zi in (1, 2, 4, 8, 16, 32):
        for un in (1, 2, 4, 8):
            for soa in (False, True):
                assert (zi, 1, un, 0, 0, 0, False, soa) in keys
    for prec in (1, 2):
        assert any(t.precision == prec for t, _, _ in vs)
    assert any(d2 for _, d2, _ in vs)


def test_status_strings():
    lib = ktt_b200.load_library()
    assert lib.coul_status_string(0) == b"ok"
    assert lib.coul_status_string(5).startswith(b"device-side wait")


def test_fma_pipe_rsqrt_bound_and_constants_match_device_code():
    """The FMA-pipe reciprocal square root: exhaustive FP32 bound over every input in [1, 4)
    (the error is periodic over factors of 4), and the constants in the device header are the
    ones that bound was computed for."""
    from ktt_b200 import soft_rsqrt as sr
    lo, hi = sr.error_profile()
    assert -5e-7 < lo < 0 < hi < 5e-7
    src = open(os.path.join(REPO, "ktt_b200", "csrc", "coul_device.cuh")).read()
    assert f"kSoftRsqrtMagic = {sr.MAGIC:#x}u" in src
    for name, val in (("A1", sr.A1), ("A2", sr.A2), ("Scale", sr.SCALE)):
        m = re.search(rf"kSoftRsqrt{name} = ([0-9.eE+-]+)f;", src)
        assert m and np.float32(float(m.group(1))) == val, name
