"""The oracle is pinned before it is trusted.

* Its FP32 restatement of KTT's known-answer generator
  (Examples/JSON/generate-coulomb-output.c:22-31) must reproduce the golden
  FP32 bit patterns sampled from the reference program's own output.
* Its FP64 map must agree with that output within KTT's validation threshold
  of the known-answer test (0.01 absolute, Examples/JSON/CoulombSum3d.json:172-181)
  and, much tighter, within the FP32 rounding of the generator.
* The 2D and adjoint routines are checked against independent numpy
  evaluations on small cases.
"""
import json
import os

import numpy as np
import pytest

import oracle


@pytest.fixture(scope="module")
def kat(golden_dir):
    with open(os.path.join(golden_dir, "coulomb3d_kat.json")) as f:
        return json.load(f)


def test_kat_atoms_follow_generator():
    a = oracle.kat_atoms(64)
    i = np.arange(64, dtype=np.float32)
    assert np.array_equal(a[:, 0], np.float32(1.0) + i * np.float32(0.1))
    assert np.array_equal(a[:, 3], (np.arange(64) % 10).astype(np.float32) * np.float32(0.1))


def test_fp32_restatement_bit_exact_on_golden_samples(kat):
    a = oracle.kat_atoms(64)
    idx = np.asarray(kat["index"], dtype=np.int64)
    bits = np.asarray(kat["bits"], dtype=np.uint32)
    cells = kat["cells"]
    z = idx // (cells * cells)
    # evaluate whole slices that contain sampled points, a band at a time
    got = np.empty(idx.size, dtype=np.float32)
    for z0 in np.unique(z):
        sl = oracle.kat_fp32(a, kat["grid_spacing_f32"], cells, int(z0), int(z0) + 1)[0].reshape(-1)
        m = z == z0
        got[m] = sl[idx[m] % (cells * cells)]
    assert np.array_equal(got.view(np.uint32), bits)


def test_fp64_oracle_against_golden(kat):
    a = oracle.kat_atoms(64)
    idx = np.asarray(kat["index"], dtype=np.int64)
    ref = np.asarray(kat["bits"], dtype=np.uint32).view(np.float32).astype(np.float64)
    cells = kat["cells"]
    v = oracle.points3d(a, kat["grid_spacing_f32"], (cells, cells, cells), idx)
    d = np.abs(v - ref)
    assert d.max() <= kat["validation_threshold"]
    # the generator sums 64 FP32 terms: its error is a few ulps of the result
    assert np.max(d / np.abs(v)) < 2e-6


def test_fp64_oracle_full_map_statistics(kat):
    a = oracle.kat_atoms(64)
    cells = kat["cells"]
    v = oracle.grid3d(a, kat["grid_spacing_f32"], (cells, cells, cells))
    assert abs(v.min() - kat["min"]) < 1e-4 and abs(v.max() - kat["max"]) < 1e-3
    assert abs(v.mean() - kat["mean"]) < 1e-6
    assert int(np.argmax(v)) == kat["argmax"]


def _numpy_map(atoms, h, dims, origin=(0, 0, 0)):
    nx, ny, nz = dims
    a = atoms.astype(np.float64)
    gx = np.array([np.fmaf(np.float32(i), np.float32(h), np.float32(origin[0])) if hasattr(np, "fmaf") else
                   np.float32(np.float64(np.float32(i)) * np.float32(h) + np.float32(origin[0])) for i in range(nx)],
                  dtype=np.float64)
    gy = np.array([np.float32(np.float64(np.float32(i)) * np.float32(h) + np.float32(origin[1])) for i in range(ny)],
                  dtype=np.float64)
    gz = np.array([np.float32(np.float64(np.float32(i)) * np.float32(h) + np.float32(origin[2])) for i in range(nz)],
                  dtype=np.float64)
    d2 = ((gz[:, None, None, None] - a[None, None, None, :, 2]) ** 2 +
          (gy[None, :, None, None] - a[None, None, None, :, 1]) ** 2 +
          (gx[None, None, :, None] - a[None, None, None, :, 0]) ** 2)
    return np.sum(a[:, 3] / np.sqrt(d2), axis=-1)


def test_grid3d_matches_numpy_with_origin():
    rng = np.random.default_rng(0)
    atoms = rng.uniform(0, 6, (37, 4)).astype(np.float32)
    atoms[:, 3] -= 3.0
    dims, h, origin = (7, 5, 3), 0.75, (-1.25, 0.5, 2.0)
    ref = _numpy_map(atoms, h, dims, origin)
    got = oracle.grid3d(atoms, h, dims, origin)
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12)
    idx = np.array([0, 5, 17, 104], dtype=np.int64)
    pts, sabs = oracle.points3d(atoms, h, dims, idx, origin, want_sumabs=True)
    np.testing.assert_allclose(pts, got.reshape(-1)[idx], rtol=1e-14)
    assert np.all(sabs >= np.abs(pts))


def test_slice2d_convention():
    rng = np.random.default_rng(1)
    a = rng.uniform(0, 10, (50, 4)).astype(np.float32)
    a[:, 3] -= 5.0
    h = 0.5
    got = oracle.slice2d(a, h, 9, 6)
    gx = np.arange(9, dtype=np.float32) * np.float32(h)
    gy = np.arange(6, dtype=np.float32) * np.float32(h)
    ad = a.astype(np.float64)
    d2 = ((gy[:, None, None] - ad[None, None, :, 1]) ** 2 + (gx[None, :, None] - ad[None, None, :, 0]) ** 2 +
          ad[None, None, :, 2])
    np.testing.assert_allclose(got, np.sum(ad[:, 3] / np.sqrt(d2), axis=-1), rtol=1e-12)


def test_adjoint_oracle_against_finite_differences():
    rng = np.random.default_rng(2)
    n = 12
    a = np.empty((n, 4), dtype=np.float32)
    a[:, :3] = rng.uniform(0.3, 3.7, (n, 3))
    a[:, 3] = rng.uniform(-1, 1, n)
    dims, h = (9, 8, 7), 0.5
    target = rng.normal(0, 1, dims[::-1]).astype(np.float32)
    weight = (rng.uniform(0, 1, dims[::-1]) > 0.2).astype(np.float32)
    loss, dq, dr, vmap = oracle.adjoint3d(a, h, dims, target, weight, want_map=True)
    ref = _numpy_map(a, h, dims)
    np.testing.assert_allclose(vmap, ref, rtol=1e-12)
    assert abs(loss - 0.5 * np.sum(weight * (ref - target) ** 2)) < 1e-9 * max(1.0, loss)
    eps = 1e-4
    for j in range(n):
        for c in range(4):
            plus = a[j].astype(np.float64).copy()
            minus = plus.copy()
            plus[c] += eps
            minus[c] -= eps
            lp = oracle.loss_perturbed(a, j, plus, h, dims, target, vmap, weight)
            lm = oracle.loss_perturbed(a, j, minus, h, dims, target, vmap, weight)
            fd = (lp - lm) / (2 * eps)
            an = dq[j] if c == 3 else dr[j, c]
            assert abs(fd - an) <= 1e-5 * max(1.0, abs(an)), (j, c, fd, an)
