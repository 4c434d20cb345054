"""The multi-GPU layout's host logic on CPU: the z-slab plan, and world-size 2 and 3 gloo process
groups running the sharded map (slabs evaluated by the FP64 oracle standing in for the GPU kernel),
its all-gather, and the max-over-ranks timing reduction the benchmark uses."""
import os
import socket

import numpy as np
import pytest

from ktt_b200 import sharding


@pytest.mark.parametrize("nz", [0, 1, 7, 8, 9, 64, 255, 256, 257])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
@pytest.mark.parametrize("align", [1, 4, 8, 16])
def test_slab_plan_covers_once_aligned_balanced(nz, world, align):
    plan = sharding.slab_plan(nz, world, align)
    assert len(plan) == world
    z = 0
    for z0, z1 in plan:
        assert z0 == z and z1 >= z0
        assert z0 % align == 0 or z0 == nz
        assert z1 % align == 0 or z1 == nz
        z = z1
    assert z == nz
    units = [(z1 - z0 + align - 1) // align for z0, z1 in plan]
    assert max(units) - min(units) <= 1


def test_slab_plan_rejects_bad_arguments():
    for args in ((-1, 2, 1), (8, 0, 1), (8, 2, 0)):
        with pytest.raises(ValueError):
            sharding.slab_plan(*args)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, result_dir):
    import torch
    import torch.distributed as dist

    import oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        rng = np.random.default_rng(5)
        atoms = np.empty((37, 4), dtype=np.float32)
        atoms[:, :3] = rng.uniform(0.0, 6.0, (37, 3))
        atoms[:, 3] = rng.uniform(-1.0, 1.0, 37)
        dims, h, origin = (9, 7, 23), 0.5, (-0.5, 0.25, 0.0)
        full_ref = oracle.grid3d(atoms, h, dims, origin)  # (nz, ny, nx) FP64

        class Tune:  # only the z depth matters for the plan
            z_iterations = 4

        def compute(z0, z1):
            return torch.from_numpy(full_ref[z0:z1].astype(np.float32))

        slab, (z0, z1), full = sharding.forward_3d_sharded(None, torch.zeros((1, 4)), dims, h, origin, tune=Tune(),
                                                          compute=compute)
        assert slab.shape == (z1 - z0, dims[1], dims[0])
        ok_full = bool(np.array_equal(full.numpy(), full_ref.astype(np.float32)))
        worst = sharding.max_over_ranks(10.0 * (rank + 1))
        sharding.barrier()
        np.save(os.path.join(result_dir, f"r{rank}.npy"),
                np.array([z0, z1, float(ok_full), worst], dtype=np.float64))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_map_gloo(tmp_path, world):
    import torch.multiprocessing as mp
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    rows = [np.load(tmp_path / f"r{r}.npy") for r in range(world)]
    plan = sharding.slab_plan(23, world, 4)
    for r, row in enumerate(rows):
        assert (int(row[0]), int(row[1])) == plan[r]
        assert row[2] == 1.0, f"rank {r}: gathered map differs from the oracle's"
        assert row[3] == 10.0 * world


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_molecule_plan_deals_every_molecule_once_balanced(world):
    rng = np.random.default_rng(7)
    pairs = list(rng.lognormal(20.0, 1.5, 137))
    plan = sharding.molecule_plan(pairs, world)
    assert len(plan) == world
    dealt = sorted(i for part in plan for i in part)
    assert dealt == list(range(len(pairs)))
    loads = [sum(pairs[i] for i in part) for part in plan]
    # longest processing time first: no rank exceeds the average by more than the largest molecule
    assert max(loads) <= sum(pairs) / world + max(pairs)
    assert sharding.molecule_plan(pairs, world) == plan  # deterministic
    with pytest.raises(ValueError):
        sharding.molecule_plan(pairs, 0)
