"""The atom-split forms of the forward kernel against the FP64 oracle and against the
one-CTA-per-tile form: the thread-block cluster form (cluster sizes 2..16, above 8 the B200's
non-portable cluster sizes), the queue form (a persistent grid over (tile, chunk) items, 2..256
chunks) and the balanced form (equal ranges of the (tile, atom) space per resident CTA, 2..32 atom
groups per CTA); 3D maps and 2D slices, ragged atom counts (fewer atoms than chunks included), accumulate
semantics, run-to-run determinism, and the two forms equal bit for bit for the same chunk count."""
import numpy as np
import pytest

import ktt_b200
import oracle
from ktt_b200 import errors, workloads

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _atoms(n, seed, box=20.0):
    rng = np.random.default_rng(seed)
    a = np.zeros((max(n, 0), 4), dtype=np.float32)
    a[:, :3] = rng.uniform(0.0, box, (n, 3))
    a[:, 3] = rng.uniform(-1.0, 1.0, n)
    return a


@pytest.mark.parametrize("n_atoms", [0, 1, 3, 7, 255, 257, 4000, 8195])
@pytest.mark.parametrize("split", [2, 3, 4, 8, 12, 16])
def test_split_3d_matches_oracle(ctx, n_atoms, split):
    import torch
    a = _atoms(n_atoms, seed=n_atoms + 31)
    dims, h, origin = (37, 29, 19), 0.5, (-1.0, 0.5, 2.0)
    tune = ktt_b200.Tune(block_x=32, block_y=4, z_iterations=8, x_points=2, rsqrt_soft=2, atom_split=split)
    atoms = torch.from_numpy(a).cuda() if n_atoms else torch.zeros((0, 4), device="cuda")
    out = torch.full((dims[2], dims[1], dims[0]), float("nan"), device="cuda")
    ctx.forward_3d(atoms, dims, h, origin, tune=tune, out=out)
    got = out.cpu().numpy()
    if n_atoms == 0:
        assert np.all(got == 0.0)
        return
    ref = oracle.grid3d(a, h, dims, origin)
    assert errors.report(got, ref)["rel_norm"] <= TOL
    plain = ctx.forward_3d(atoms, dims, h, origin, tune=ktt_b200.Tune(block_x=32, block_y=4, z_iterations=8,
                                                                      x_points=2, rsqrt_soft=2))
    assert float((out - plain).abs().max()) <= TOL * max(float(plain.abs().max()), 1e-30)


@pytest.mark.parametrize("shape", [(1, 1, 1), (2, 1, 1), (4, 1, 2), (2, 2, 2), (1, 2, 4)])
@pytest.mark.parametrize("split", [2, 4, 8, 16])
def test_split_2d_slice_matches_oracle(ctx, shape, split):
    import torch
    zi, xp, un = shape
    case = workloads.slice_2d(n_atoms=4000, n=256)
    ref = oracle.slice2d(case.ktt_atoms(), case.spacing, case.nx, case.ny)
    sliced = ctx.slice_atoms(torch.from_numpy(case.atoms).cuda(), case.z_slice)
    tune = ktt_b200.Tune(block_x=32, block_y=4, z_iterations=zi, x_points=xp, unroll=un, atom_split=split)
    got = ctx.forward_2d(sliced, case.spacing, case.nx, case.ny, tune=tune)
    assert errors.report(got.cpu().numpy(), ref)["rel_norm"] <= TOL
    again = ctx.forward_2d(sliced, case.spacing, case.nx, case.ny, tune=tune)
    assert torch.equal(got, again)


def test_split_2d_ragged_slice_and_accumulate(ctx):
    import torch
    a = _atoms(1234, seed=8)
    nx, ny, h, zs = 101, 75, 0.5, 7.0
    kat = a.copy()
    kat[:, 2] = (np.float32(zs) - a[:, 2]) ** 2
    ref = oracle.slice2d(kat, h, nx, ny)
    sliced = ctx.slice_atoms(torch.from_numpy(a).cuda(), zs)
    tune = ktt_b200.Tune(block_x=16, block_y=8, z_iterations=2, x_points=2, atom_split=3)
    v = ctx.forward_2d(sliced, h, nx, ny, tune=tune)
    assert errors.report(v.cpu().numpy(), ref)["rel_norm"] <= TOL
    base = torch.linspace(-2, 2, nx * ny, device="cuda").reshape(ny, nx)
    acc = base.clone()
    ctx.forward_2d(sliced, h, nx, ny, tune=tune, out=acc, accumulate=True)
    assert torch.equal(acc, base + v)


def test_split_slab_equals_split_map(ctx):
    import torch
    a = _atoms(900, seed=12)
    dims, h = (40, 33, 48), 0.5
    tune = ktt_b200.Tune(block_x=32, block_y=4, z_iterations=8, x_points=1, rsqrt_soft=2, atom_split=4)
    atoms = torch.from_numpy(a).cuda()
    full = ctx.forward_3d(atoms, dims, h, tune=tune)
    slab = ctx.forward_3d_slab(atoms, dims, h, 16, 40, tune=tune)
    assert torch.equal(slab, full[16:40])


@pytest.mark.parametrize("n_atoms", [0, 1, 5, 300, 4000, 8195])
@pytest.mark.parametrize("chunks", [2, 16, 64, 256])
def test_queue_split_3d_matches_oracle(ctx, n_atoms, chunks):
    import torch
    a = _atoms(n_atoms, seed=n_atoms + 57)
    dims, h, origin = (37, 29, 19), 0.5, (-1.0, 0.5, 2.0)
    tune = ktt_b200.Tune(block_x=32, block_y=4, z_iterations=8, x_points=2, rsqrt_soft=2, atom_split=chunks,
                         split_form=1)
    atoms = torch.from_numpy(a).cuda() if n_atoms else torch.zeros((0, 4), device="cuda")
    out = torch.full((dims[2], dims[1], dims[0]), float("nan"), device="cuda")
    ctx.forward_3d(atoms, dims, h, origin, tune=tune, out=out)
    got = out.cpu().numpy()
    if n_atoms == 0:
        assert np.all(got == 0.0)
        return
    ref = oracle.grid3d(a, h, dims, origin)
    assert errors.report(got, ref)["rel_norm"] <= TOL
    again = ctx.forward_3d(atoms, dims, h, origin, tune=tune)
    assert torch.equal(out, again)  # the chunk order of the sums does not depend on scheduling


@pytest.mark.parametrize("shape", [(2, 2, 0), (4, 2, 2), (4, 1, 2), (8, 2, 2)])
@pytest.mark.parametrize("chunks", [4, 16, 48])
def test_queue_split_2d_slice(ctx, shape, chunks):
    import torch
    zi, xp, soft = shape
    case = workloads.slice_2d(n_atoms=4000, n=256)
    ref = oracle.slice2d(case.ktt_atoms(), case.spacing, case.nx, case.ny)
    sliced = ctx.slice_atoms(torch.from_numpy(case.atoms).cuda(), case.z_slice)
    tune = ktt_b200.Tune(block_x=32, block_y=4, z_iterations=zi, x_points=xp, rsqrt_soft=soft, atom_split=chunks,
                         split_form=1)
    got = ctx.forward_2d(sliced, case.spacing, case.nx, case.ny, tune=tune)
    assert errors.report(got.cpu().numpy(), ref)["rel_norm"] <= TOL
    if chunks <= 16:
        # the cluster form with as many CTAs per tile adds the same partials in the same order
        cluster = ktt_b200.Tune(**dict(tune.as_dict(), split_form=0))
        if ktt_b200.tune_supported_2d(cluster):
            assert torch.equal(got, ctx.forward_2d(sliced, case.spacing, case.nx, case.ny, tune=cluster))
    base = torch.linspace(-2, 2, case.nx * case.ny, device="cuda").reshape(case.ny, case.nx)
    acc = base.clone()
    ctx.forward_2d(sliced, case.spacing, case.nx, case.ny, tune=tune, out=acc, accumulate=True)
    assert torch.equal(acc, base + got)


@pytest.mark.parametrize("n_atoms", [0, 1, 5, 9, 1023, 1025, 4000, 8195])
@pytest.mark.parametrize("block,groups", [((32, 1), 2), ((32, 1), 32), ((32, 2), 8), ((64, 1), 16)])
def test_balanced_split_3d_matches_oracle(ctx, n_atoms, block, groups):
    import torch
    a = _atoms(n_atoms, seed=n_atoms + 77)
    dims, h, origin = (37, 29, 19), 0.5, (-1.0, 0.5, 2.0)
    tune = ktt_b200.Tune(block_x=block[0], block_y=block[1], z_iterations=8, x_points=2, rsqrt_soft=2,
                         atom_split=groups, split_form=2)
    atoms = torch.from_numpy(a).cuda() if n_atoms else torch.zeros((0, 4), device="cuda")
    out = torch.full((dims[2], dims[1], dims[0]), float("nan"), device="cuda")
    ctx.forward_3d(atoms, dims, h, origin, tune=tune, out=out)
    got = out.cpu().numpy()
    if n_atoms == 0:
        assert np.all(got == 0.0)
        return
    ref = oracle.grid3d(a, h, dims, origin)
    assert errors.report(got, ref)["rel_norm"] <= TOL
    again = ctx.forward_3d(atoms, dims, h, origin, tune=tune)
    assert torch.equal(out, again)  # fixed ranges per CTA, pieces added in CTA order


@pytest.mark.parametrize("shape", [(4, 2, 0), (4, 2, 2), (4, 2, 3), (2, 2, 2), (8, 2, 2), (4, 4, 2), (2, 4, 2),
                                   (8, 1, 2)])
@pytest.mark.parametrize("block,groups", [((32, 1), 32), ((32, 1), 8), ((64, 1), 16), ((32, 2), 4)])
def test_balanced_split_2d_slice(ctx, shape, block, groups):
    import torch
    zi, xp, soft = shape
    case = workloads.slice_2d(n_atoms=4000, n=256)
    ref = oracle.slice2d(case.ktt_atoms(), case.spacing, case.nx, case.ny)
    sliced = ctx.slice_atoms(torch.from_numpy(case.atoms).cuda(), case.z_slice)
    tune = ktt_b200.Tune(block_x=block[0], block_y=block[1], z_iterations=zi, x_points=xp, rsqrt_soft=soft,
                         atom_split=groups, split_form=2)
    got = ctx.forward_2d(sliced, case.spacing, case.nx, case.ny, tune=tune)
    assert errors.report(got.cpu().numpy(), ref)["rel_norm"] <= TOL
    assert torch.equal(got, ctx.forward_2d(sliced, case.spacing, case.nx, case.ny, tune=tune))
    base = torch.linspace(-2, 2, case.nx * case.ny, device="cuda").reshape(case.ny, case.nx)
    acc = base.clone()
    ctx.forward_2d(sliced, case.spacing, case.nx, case.ny, tune=tune, out=acc, accumulate=True)
    assert torch.equal(acc, base + got)


def test_balanced_split_ragged_slice_and_slab(ctx):
    import torch
    a = _atoms(1234, seed=18)
    nx, ny, h, zs = 101, 75, 0.5, 7.0
    kat = a.copy()
    kat[:, 2] = (np.float32(zs) - a[:, 2]) ** 2
    ref = oracle.slice2d(kat, h, nx, ny)
    sliced = ctx.slice_atoms(torch.from_numpy(a).cuda(), zs)
    tune = ktt_b200.Tune(block_x=32, block_y=1, z_iterations=4, x_points=2, rsqrt_soft=2, atom_split=16,
                         split_form=2)
    v = ctx.forward_2d(sliced, h, nx, ny, tune=tune)
    assert errors.report(v.cpu().numpy(), ref)["rel_norm"] <= TOL
    # a z slab of a 3D map equals the same planes of the whole map
    b = _atoms(900, seed=19)
    dims = (40, 33, 48)
    t3 = ktt_b200.Tune(block_x=32, block_y=1, z_iterations=8, x_points=1, rsqrt_soft=2, atom_split=8, split_form=2)
    atoms = torch.from_numpy(b).cuda()
    full = ctx.forward_3d(atoms, dims, h, tune=t3)
    ref3 = oracle.grid3d(b, h, dims)
    assert errors.report(full.cpu().numpy(), ref3)["rel_norm"] <= TOL
    slab = ctx.forward_3d_slab(atoms, dims, h, 16, 40, tune=t3)
    assert errors.report(slab.cpu().numpy(), ref3[16:40])["rel_norm"] <= TOL


def test_balanced_split_counters_across_forms_and_grids(ctx):
    """The balanced form zeroes its counters as it completes; launches of other grids, the queue
    form's use of the same workspace and tiny maps (fewer units than CTAs) in between stay exact."""
    import torch
    a = _atoms(700, seed=23)
    b = _atoms(3, seed=24)
    atoms_a = torch.from_numpy(a).cuda()
    atoms_b = torch.from_numpy(b).cuda()
    bal = ktt_b200.Tune(block_x=32, block_y=1, z_iterations=8, x_points=2, rsqrt_soft=2, atom_split=16,
                        split_form=2)
    queue = ktt_b200.Tune(block_x=32, block_y=4, z_iterations=8, x_points=2, rsqrt_soft=2, atom_split=16,
                          split_form=1)
    cases = [((33, 17, 9), atoms_a, a, bal), ((33, 17, 9), atoms_a, a, bal), ((5, 4, 3), atoms_b, b, bal),
             ((33, 17, 9), atoms_a, a, queue), ((33, 17, 9), atoms_a, a, bal), ((64, 40, 24), atoms_a, a, bal),
             ((5, 4, 3), atoms_b, b, bal), ((64, 40, 24), atoms_a, a, bal)]
    first = {}
    for dims, atoms, host, tune in cases:
        got = ctx.forward_3d(atoms, dims, 0.5, tune=tune)
        ref = oracle.grid3d(host, 0.5, dims)
        assert errors.report(got.cpu().numpy(), ref)["rel_norm"] <= TOL
        key = (dims, tune.split_form)
        if key in first:
            assert torch.equal(got, first[key])
        first.setdefault(key, got)


def test_balanced_split_alternating_sizes_and_contexts(ctx):
    """The persistent forms keep their occupancy per context and only ever raise a kernel's shared
    memory limit: configurations of one kernel with large and small shared memory, alternated within a
    context and across two contexts on the same device, all stay launchable and exact."""
    import torch
    a = _atoms(2100, seed=29)
    dims, h = (45, 31, 26), 0.5
    atoms = torch.from_numpy(a).cuda()
    ref = oracle.grid3d(a, h, dims)
    big = ktt_b200.Tune(block_x=64, block_y=1, z_iterations=8, x_points=2, rsqrt_soft=2, atom_split=16, split_form=2)
    small = ktt_b200.Tune(block_x=32, block_y=1, z_iterations=8, x_points=2, rsqrt_soft=2, atom_split=2, split_form=2)
    other = ktt_b200.CoulombContext(0)
    try:
        first = {}
        for c, tune in ((ctx, big), (ctx, small), (other, small), (ctx, big), (other, big), (ctx, small)):
            got = c.forward_3d(atoms, dims, h, tune=tune)
            assert errors.report(got.cpu().numpy(), ref)["rel_norm"] <= TOL
            key = tune.atom_split
            if key in first:
                assert torch.equal(got, first[key])
            first.setdefault(key, got)
    finally:
        other.close()
