"""Multi-GPU layout: one process per GPU, one map split into z slabs, or a batch of molecules dealt
out to the ranks.

Grid points are independent, so a map shards by z slabs with no collective on the data path: every
rank holds all atoms, evaluates its slab with coul_forward_3d_slab (the full grid's coordinates, so
the slabs put together equal the single-GPU map bit for bit), and writes it to its own memory.  An
optional all-gather assembles the whole map on every rank (NCCL over NVLink on GPUs, gloo on CPU).
The reference has no multi-device path for this computation (KTT tunes one kernel on one device,
Source/Api/Tuner.h:83 takes one platform/device index).

A batch of molecules shards by molecule (molecule_plan: longest first, each to the least-loaded
rank), each rank running its share through one persistent launch, again with no collective.

The timing helpers (barrier, max over ranks) are the ones the benchmark uses.
"""
from __future__ import annotations

from typing import Callable


def slab_plan(nz: int, world: int, align: int = 1) -> list[tuple[int, int]]:
    """Contiguous z ranges, one per rank, covering [0, nz) once.  Boundaries fall on multiples of
    `align` (the kernel tile's z depth, so no slab pays for a partial tile in its middle); the
    units of `align` planes are dealt out as evenly as possible, earlier ranks taking the extra
    ones.  Ranks beyond the number of units get an empty range (z0 == z1)."""
    if nz < 0 or world < 1 or align < 1:
        raise ValueError("nz >= 0, world >= 1 and align >= 1 required")
    units = (nz + align - 1) // align
    per, extra = divmod(units, world)
    plan, u = [], 0
    for r in range(world):
        k = per + (1 if r < extra else 0)
        plan.append((min(u * align, nz), min((u + k) * align, nz)))
        u += k
    return plan


def rank_world(group=None) -> tuple[int, int]:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


def barrier(group=None) -> None:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.barrier(group=group)


def max_over_ranks(x: float, group=None, device=None) -> float:
    """The maximum of a per-rank scalar (device times are reported as the slowest rank's)."""
    import torch
    import torch.distributed as dist
    rank, world = rank_world(group)
    if world == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def forward_3d_sharded(ctx, atoms, dims, spacing, origin=None, tune=None, group=None, gather: bool = True,
                       compute: Callable | None = None):
    """This rank's slab of the map, and (gather=True) the whole map assembled on every rank.

    Returns (slab, (z0, z1), full): slab has shape (z1 - z0, ny, nx); full is (nz, ny, nx) or None.
    `compute(z0, z1)` evaluates a slab; the default is ctx.forward_3d_slab with `tune`.
    """
    import torch
    import torch.distributed as dist
    nx, ny, nz = (int(d) for d in dims)
    rank, world = rank_world(group)
    align = int(tune.z_iterations) if tune is not None else 1
    plan = slab_plan(nz, world, align)
    z0, z1 = plan[rank]
    if compute is None:
        def compute(a, b):
            return ctx.forward_3d_slab(atoms, dims, spacing, a, b, origin, tune=tune)
    if z1 > z0:
        slab = compute(z0, z1)
    else:
        slab = torch.empty((0, ny, nx), dtype=torch.float32, device=atoms.device)
    if not gather:
        return slab, (z0, z1), None
    if world == 1:
        return slab, (z0, z1), slab
    depth = max(b - a for a, b in plan)
    padded = torch.zeros((depth, ny, nx), dtype=slab.dtype, device=slab.device)
    padded[: z1 - z0] = slab
    parts = [torch.empty_like(padded) for _ in range(world)]
    dist.all_gather(parts, padded, group=group)
    full = torch.cat([p[: b - a] for p, (a, b) in zip(parts, plan)], dim=0)
    return slab, (z0, z1), full


def molecule_plan(pairs: list[float], world: int) -> list[list[int]]:
    """Molecules of a batch dealt to ranks, longest processing time first: each molecule in
    decreasing order of pair count goes to the rank with the fewest pairs so far (ties: the lower
    rank), so every rank's share stays within one molecule of the average.  Deterministic; returns
    each rank's molecule indices in the order they were dealt."""
    if world < 1:
        raise ValueError("world >= 1 required")
    order = sorted(range(len(pairs)), key=lambda i: (-pairs[i], i))
    load = [0.0] * world
    plan: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        plan[r].append(i)
        load[r] += pairs[i]
    return plan


def batch_sharded(ctx, molecules, tune=None, group=None):
    """This rank's molecules of a batch (molecule_plan over the ranks' count), evaluated by one
    persistent launch on this rank's GPU; no collective on the data path.  `molecules` as for
    ktt_b200.Batch.  Returns (indices, outputs): the molecule indices this rank evaluated and their
    maps, in the same order."""
    import ktt_b200
    rank, world = rank_world(group)
    pairs = [float(m[0].shape[0]) * int(m[1][0]) * int(m[1][1]) * int(m[1][2]) for m in molecules]
    mine = molecule_plan(pairs, world)[rank]
    if not mine:
        return [], []
    batch = ktt_b200.Batch(ctx, [molecules[i] for i in mine], tune)
    try:
        batch.run(ktt_b200.BATCH_PERSISTENT)
        ctx.synchronize()
        return mine, list(batch.outputs)
    finally:
        batch.close()
