"""The N-body step (coul_nbody_step, the sibling of KTT's Nbody example) against the FP64 oracle:
ragged body counts (not multiples of any tile), every compiled bodies-per-thread / unroll form, the
cluster j-split, run-to-run determinism, KTT's own example size (128 K bodies) on a seeded subset,
and argument errors.  The accelerations themselves are checked through a step with zero velocities
and dt = 1, whose velocity update is v' = fma(1, a, 0) = a exactly."""
import numpy as np
import pytest

import ktt_b200
import oracle

pytestmark = pytest.mark.gpu

DT, DAMPING, EPS2 = 0.001, 0.5, 0.1 * 0.1


def _bodies(n, seed):
    # KTT's Nbody.cpp:96-118: positions, masses and velocities uniform in [0, 20)
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0.0, 20.0, (n, 4)).astype(np.float32)
    vel = rng.uniform(0.0, 20.0, (n, 4)).astype(np.float32)
    vel[:, 3] = 0.0
    return pos, vel


def _check(pos, vel, new_pos, new_vel, idx=None, dt=DT):
    ref_pos, ref_vel, ref_acc = oracle.nbody_step(pos, vel, dt, DAMPING, EPS2, idx)
    sel = slice(None) if idx is None else idx
    assert np.abs(new_vel[sel].astype(np.float64) - ref_vel).max() <= 1e-5 * np.abs(ref_vel).max()
    assert np.abs(new_pos[sel].astype(np.float64) - ref_pos).max() <= 1e-5 * np.abs(ref_pos).max()
    assert np.array_equal(new_pos[sel, 3], pos[sel, 3]) and np.all(new_vel[sel, 3] == 0.0)


TUNES = [ktt_b200.NbodyTune(block_x=bx, bodies_per_thread=bp, unroll=un)
         for bx, bp, un in ((128, 2, 1), (128, 2, 4), (64, 4, 2), (256, 4, 4), (128, 8, 1), (32, 8, 2))]


@pytest.mark.parametrize("n", [1, 7, 255, 257, 1000, 4099])
@pytest.mark.parametrize("ti", range(len(TUNES)))
def test_nbody_matches_oracle(ctx, n, ti):
    import torch
    pos, vel = _bodies(n, seed=n)
    tp = torch.from_numpy(pos).cuda()
    p, v = ktt_b200.nbody_step(ctx, tp, torch.from_numpy(vel).cuda(), DT, DAMPING, EPS2, TUNES[ti])
    _check(pos, vel, p.cpu().numpy(), v.cpu().numpy())
    # accelerations: zero velocities and dt = 1 make the velocity update equal to a
    still = np.zeros_like(vel)
    _, a = ktt_b200.nbody_step(ctx, tp, torch.from_numpy(still).cuda(), 1.0, DAMPING, EPS2, TUNES[ti])
    _, _, ref_acc = oracle.nbody_step(pos, still, 1.0, DAMPING, EPS2)
    assert np.abs(a.cpu().numpy()[:, :3].astype(np.float64) - ref_acc).max() <= 1e-5 * max(np.abs(ref_acc).max(), 1e-30)


@pytest.mark.parametrize("split", [2, 3, 8, 16])
def test_nbody_j_split(ctx, split):
    import torch
    pos, vel = _bodies(3001, seed=5)
    tp, tv = torch.from_numpy(pos).cuda(), torch.from_numpy(vel).cuda()
    tune = ktt_b200.NbodyTune(block_x=128, bodies_per_thread=4, unroll=2, j_split=split)
    p, v = ktt_b200.nbody_step(ctx, tp, tv, DT, DAMPING, EPS2, tune)
    _check(pos, vel, p.cpu().numpy(), v.cpu().numpy())
    p2, v2 = ktt_b200.nbody_step(ctx, tp, tv, DT, DAMPING, EPS2, tune)
    assert torch.equal(p, p2) and torch.equal(v, v2)


def test_nbody_ktt_example_size(ctx):
    """131,072 bodies (Examples/Nbody/Nbody.cpp:62), 512 seeded bodies checked."""
    import torch
    n = 128 * 1024
    pos, vel = _bodies(n, seed=11)
    p, v = ktt_b200.nbody_step(ctx, torch.from_numpy(pos).cuda(), torch.from_numpy(vel).cuda(), DT, DAMPING, EPS2)
    idx = np.sort(np.random.default_rng(3).choice(n, 512, replace=False))
    _check(pos, vel, p.cpu().numpy(), v.cpu().numpy(), idx)


def test_nbody_rejects_bad_arguments(ctx):
    import torch
    pos, vel = _bodies(64, seed=1)
    tp, tv = torch.from_numpy(pos).cuda(), torch.from_numpy(vel).cuda()
    with pytest.raises(ktt_b200.CoulombError):
        ktt_b200.nbody_step(ctx, tp, tv, DT, DAMPING, EPS2, out_pos=tp)  # output aliases input
    with pytest.raises(ktt_b200.CoulombError):
        ktt_b200.nbody_step(ctx, tp, tv, DT, DAMPING, 0.0)  # no softening: the j = i term divides by zero
    with pytest.raises(ktt_b200.CoulombError):
        ktt_b200.nbody_step(ctx, tp, tv, DT, DAMPING, EPS2, ktt_b200.NbodyTune(bodies_per_thread=3))
    with pytest.raises(ktt_b200.CoulombError):
        ktt_b200.nbody_step(ctx, tp, tv, DT, DAMPING, EPS2, ktt_b200.NbodyTune(block_x=48))
