"""The batched persistent path: (molecule, tile) work items from a device queue, one launch,
optionally replayed from a CUDA graph, against one plain launch per molecule and the FP64 oracle."""
import numpy as np
import pytest

import oracle
from ktt_b200 import errors, workloads
import ktt_b200

pytestmark = pytest.mark.gpu


def _small_batch(seed=21, n_mol=24, lo=50, hi=3000):
    return workloads.molecule_batch(seed=seed, n_mol=n_mol, lo=lo, hi=hi)


@pytest.mark.parametrize("tune", [
    ktt_b200.Tune(z_iterations=8, x_points=2, unroll=2, rsqrt_soft=2),
    ktt_b200.Tune(z_iterations=16, x_points=1, rsqrt_soft=2, block_x=64, block_y=2),
    ktt_b200.Tune(z_iterations=8, x_points=2, precision=ktt_b200.PREC_FP64_MERGE, rsqrt_soft=2),
    ktt_b200.Tune(z_iterations=8, x_points=2, unroll=2, rsqrt_soft=12),
    # one x-y point per thread: linear x-y tiles in the batch, the block's own tiles one launch per molecule
    ktt_b200.Tune(z_iterations=16, x_points=1, unroll=2, rsqrt_soft=12, block_x=8, block_y=4),
    ktt_b200.Tune(z_iterations=8, x_points=1, rsqrt_soft=12, block_x=16, block_y=4),
])
def test_persistent_graph_and_separate_agree_bitwise(ctx, tune):
    import torch
    mols = _small_batch()
    inputs = [(torch.from_numpy(m.atoms).cuda(), m.dims, m.spacing, m.origin) for m in mols]
    b = ktt_b200.Batch(ctx, inputs, tune)
    assert b.work_items > 0 and b.grid_ctas >= ctx.sm_count
    maps = {}
    for mode in (ktt_b200.BATCH_SEPARATE, ktt_b200.BATCH_PERSISTENT, ktt_b200.BATCH_GRAPH):
        for o in b.outputs:
            o.fill_(float("nan"))
        b.run(mode)
        ctx.synchronize()
        maps[mode] = [o.cpu().numpy().copy() for o in b.outputs]
    for a, p, g in zip(maps[ktt_b200.BATCH_SEPARATE], maps[ktt_b200.BATCH_PERSISTENT], maps[ktt_b200.BATCH_GRAPH]):
        assert np.array_equal(a.view(np.uint32), p.view(np.uint32))
        assert np.array_equal(a.view(np.uint32), g.view(np.uint32))
    # graph replay again (accumulate) adds the same map on top
    b.run(ktt_b200.BATCH_GRAPH, accumulate=True)
    ctx.synchronize()
    for o, ref in zip(b.outputs, maps[ktt_b200.BATCH_GRAPH]):
        np.testing.assert_allclose(o.cpu().numpy(), 2 * ref, rtol=1e-6, atol=1e-6)
    b.close()


@pytest.mark.parametrize("tune", [None, ktt_b200.Tune(z_iterations=16, x_points=1, unroll=2, rsqrt_soft=2, block_x=8,
                                                     block_y=4)])
def test_batched_against_oracle(ctx, tune):
    import torch
    mols = _small_batch(seed=22, n_mol=10)
    inputs = [(torch.from_numpy(m.atoms).cuda(), m.dims, m.spacing, m.origin) for m in mols]
    b = ktt_b200.Batch(ctx, inputs, tune) if tune is not None else ktt_b200.Batch(ctx, inputs)
    b.run(ktt_b200.BATCH_GRAPH)
    ctx.synchronize()
    for m, out in zip(mols, b.outputs):
        total = int(np.prod(m.dims))
        idx = workloads.subset_indices(total, min(1.0, 3000 / total), seed=5)
        ref = oracle.points3d(m.atoms, m.spacing, m.dims, idx, origin=m.origin)
        rep = errors.report(out.cpu().numpy().reshape(-1)[idx], ref)
        assert rep["rel_norm"] <= 1e-5, rep
    b.close()


def test_batch_rejects_unsupported_shape(ctx):
    import torch
    mols = _small_batch(n_mol=2)
    inputs = [(torch.from_numpy(m.atoms).cuda(), m.dims, m.spacing, m.origin) for m in mols]
    with pytest.raises(ktt_b200.CoulombError) as e:
        ktt_b200.Batch(ctx, inputs, ktt_b200.Tune(z_iterations=32, x_points=4, rsqrt_soft=1))
    assert e.value.status == ktt_b200.COUL_ERR_UNSUPPORTED


def test_batch_outlives_its_context():
    """Destroying a context releases its live batches' device resources; the batch handles can still
    be destroyed afterwards, and a run on them is refused."""
    import torch
    mols = _small_batch(n_mol=3)
    c = ktt_b200.CoulombContext(0)
    inputs = [(torch.from_numpy(m.atoms).cuda(), m.dims, m.spacing, m.origin) for m in mols]
    kept = ktt_b200.Batch(c, inputs)
    closed = ktt_b200.Batch(c, inputs)
    closed.close()
    kept.run(ktt_b200.BATCH_PERSISTENT)
    c.synchronize()
    c.close()
    lib = ktt_b200.load_library()
    assert lib.coul_batch_run(None, kept._handle, ktt_b200.BATCH_PERSISTENT, 0) == ktt_b200.COUL_ERR_INVALID_ARGUMENT
    kept.close()


def test_precise_batch_with_shared_sums(ctx):
    """The batch in the FP64-merge form with its sums in shared memory: bit-identical to the same form
    with register sums and to one forward launch per molecule, and within the pointwise gate of the
    FP64 oracle."""
    import torch
    mols = _small_batch(seed=25, n_mol=8)
    inputs = [(torch.from_numpy(m.atoms).cuda(), m.dims, m.spacing, m.origin) for m in mols]
    maps = {}
    for prec in (ktt_b200.PREC_FP64_MERGE, ktt_b200.PREC_FP64_MERGE_SHARED):
        tune = ktt_b200.Tune(block_x=8, block_y=4, z_iterations=8, x_points=2, rsqrt_soft=2, precision=prec)
        b = ktt_b200.Batch(ctx, inputs, tune)
        for mode in (ktt_b200.BATCH_PERSISTENT, ktt_b200.BATCH_SEPARATE):
            b.run(mode)
            ctx.synchronize()
            maps[(prec, mode)] = [o.cpu().numpy().copy() for o in b.outputs]
        b.close()
    ref_maps = maps[(ktt_b200.PREC_FP64_MERGE, ktt_b200.BATCH_PERSISTENT)]
    for key, got in maps.items():
        for a, r in zip(got, ref_maps):
            assert np.array_equal(a.view(np.uint32), r.view(np.uint32)), key
    for m, out in zip(mols, maps[(ktt_b200.PREC_FP64_MERGE_SHARED, ktt_b200.BATCH_PERSISTENT)]):
        total = int(np.prod(m.dims))
        idx = workloads.subset_indices(total, min(1.0, 3000 / total), seed=6)
        ref, sabs = oracle.points3d(m.atoms, m.spacing, m.dims, idx, origin=m.origin, want_sumabs=True)
        rep = errors.gate(out.reshape(-1)[idx], ref, sumabs=sabs)
        assert rep["passes_norm"] and rep["passes_point"], rep
