"""z-slab sharding on one GPU: the slabs of a map, each evaluated by coul_forward_3d_slab as the
ranks of a sharded run would, put together equal the single-launch map bit for bit; and the
molecule-sharded batch on one rank equals one batch of all molecules."""
import numpy as np
import pytest

import ktt_b200
import oracle
from ktt_b200 import errors, sharding

pytestmark = pytest.mark.gpu

TUNES = [
    ktt_b200.Tune(block_x=32, block_y=4, z_iterations=8, x_points=2, unroll=2, rsqrt_soft=2),
    ktt_b200.Tune(block_x=32, block_y=4, z_iterations=8, x_points=2, precision=ktt_b200.PREC_FP64_MERGE),
    ktt_b200.Tune(block_x=32, block_y=4, z_iterations=4, x_points=1, atom_source=ktt_b200.ATOMS_CONSTANT),
]


def _case(seed=9, n=700, dims=(70, 45, 61), h=0.5, origin=(-1.0, 2.0, 0.25)):
    rng = np.random.default_rng(seed)
    a = np.empty((n, 4), dtype=np.float32)
    a[:, :3] = rng.uniform(0.0, 30.0, (n, 3))
    a[:, 3] = rng.uniform(-1.0, 1.0, n)
    return a, dims, h, origin


@pytest.mark.parametrize("world", [2, 3, 5])
@pytest.mark.parametrize("ti", range(len(TUNES)))
def test_slabs_equal_single_map(ctx, world, ti):
    import torch
    tune = TUNES[ti]
    a, dims, h, origin = _case()
    atoms = torch.from_numpy(a).cuda()
    full = ctx.forward_3d(atoms, dims, h, origin, tune=tune)
    parts = []
    for z0, z1 in sharding.slab_plan(dims[2], world, tune.z_iterations):
        if z1 > z0:
            parts.append(ctx.forward_3d_slab(atoms, dims, h, z0, z1, origin, tune=tune))
    joined = torch.cat(parts, dim=0)
    ctx.synchronize()
    assert torch.equal(joined, full)
    # and against the oracle on a subset
    ref = oracle.grid3d(a, h, dims, origin)
    assert errors.report(joined.cpu().numpy(), ref)["rel_norm"] <= 1e-5


def test_unaligned_slab_and_single_rank_sharded(ctx):
    import torch
    tune = TUNES[0]
    a, dims, h, origin = _case(seed=4)
    atoms = torch.from_numpy(a).cuda()
    full = ctx.forward_3d(atoms, dims, h, origin, tune=tune)
    # a boundary off the tile depth: same points, but a point may take its rsqrt from the other pipe
    s = ctx.forward_3d_slab(atoms, dims, h, 13, 50, origin, tune=tune)
    assert float((s - full[13:50]).abs().max()) <= 1e-6 * float(full.abs().max())
    mufu = ktt_b200.Tune(block_x=32, block_y=4, z_iterations=8, x_points=2)
    s = ctx.forward_3d_slab(atoms, dims, h, 13, 50, origin, tune=mufu)
    assert torch.equal(s, ctx.forward_3d(atoms, dims, h, origin, tune=mufu)[13:50])
    slab, (z0, z1), whole = sharding.forward_3d_sharded(ctx, atoms, dims, h, origin, tune=tune)
    assert (z0, z1) == (0, dims[2]) and torch.equal(whole, full)


@pytest.mark.parametrize("z0,z1", [(-1, 4), (5, 5), (6, 3), (0, 62)])
def test_bad_slab_rejected(ctx, z0, z1):
    import torch
    a, dims, h, origin = _case()
    with pytest.raises(ktt_b200.CoulombError):
        ctx.forward_3d_slab(torch.from_numpy(a).cuda(), dims, h, z0, z1, origin,
                            out=torch.empty((max(z1 - z0, 1), dims[1], dims[0]), device="cuda"))


def test_batch_sharded_single_rank_equals_batch(ctx):
    """One rank (no process group): batch_sharded evaluates every molecule, in the plan's order, with
    the same maps bit for bit as one Batch of all of them."""
    import torch
    from ktt_b200 import workloads
    mols = workloads.molecule_batch(seed=31, n_mol=6, lo=50, hi=2000)
    inputs = [(torch.from_numpy(m.atoms).cuda(), m.dims, m.spacing, m.origin) for m in mols]
    idx, outs = sharding.batch_sharded(ctx, inputs)
    assert sorted(idx) == list(range(len(mols)))
    b = ktt_b200.Batch(ctx, inputs)
    b.run(ktt_b200.BATCH_PERSISTENT)
    ctx.synchronize()
    for i, o in zip(idx, outs):
        assert torch.equal(o, b.outputs[i])
    b.close()
