"""KTT's own CUDA kernels, compiled the way KTT compiles them, run on the same inputs as this
library's kernels: the known-answer map against the golden output (KTT's 0.01 criterion) and
against this library's map; a seeded uniform map over every configuration of KTT's CUDA space
against this library's map and the FP64 oracle.

With KTT_REF_SWEEP_OUT=<path> the last test also times KTT's whole 210-configuration space on the
256^3 x 65,536-atom map and writes the device times to <path> (JSON)."""
import json
import os

import numpy as np
import pytest

import ktt_b200
import oracle
import ref_kernels
from ktt_b200 import errors, workloads

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_kernels.available(),
                                 reason="KTT's kernels are not built (make -C oracle refkernels)")]


def _cols(a):
    import torch
    return [torch.from_numpy(np.ascontiguousarray(a[:, k])).cuda() for k in range(4)]


@pytest.fixture(scope="module")
def kat(golden_dir):
    with open(os.path.join(golden_dir, "coulomb3d_kat.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("cfg", [
    {"WORK_GROUP_SIZE_X": 32, "WORK_GROUP_SIZE_Y": 2, "Z_ITERATIONS": 16, "INNER_UNROLL_FACTOR": 0, "USE_SOA": 0},
    {"WORK_GROUP_SIZE_X": 16, "WORK_GROUP_SIZE_Y": 4, "Z_ITERATIONS": 32, "INNER_UNROLL_FACTOR": 8, "USE_SOA": 1},
])
def test_ktt_kernel_on_the_known_answer_map(ctx, kat, cfg):
    import torch
    cells, h = kat["cells"], kat["grid_spacing_f32"]
    atoms = oracle.kat_atoms(64)
    ta = torch.from_numpy(atoms).cuda()
    ref_out = torch.zeros(cells ** 3, device="cuda")
    ref_kernels.run_tuned(cfg, ta, _cols(atoms), 64, h, cells, ref_out)
    ours = ctx.forward_3d(ta, (cells, cells, cells), h).reshape(-1)
    torch.cuda.synchronize()
    v = ref_out.cpu().numpy()
    idx = np.asarray(kat["index"], dtype=np.int64)
    golden = np.asarray(kat["bits"], dtype=np.uint32).view(np.float32)
    assert np.max(np.abs(v[idx] - golden)) <= kat["validation_threshold"]
    # KTT's kernel steps z by repeated addition of the spacing (CoulombSum3d.cu:39), this library
    # evaluates each coordinate directly, so near an atom the two differ by more than rounding of the
    # sum; KTT's own criterion for this map (SideBySide 0.01) applies
    assert float((ref_out - ours).abs().max()) <= kat["validation_threshold"]


def test_ktt_space_matches_this_library_and_fp64(ctx):
    """All 42 compiled forms of KTT's space (two launch shapes each) on a 256^3 map of 2,048 seeded
    atoms, and KTT's reference kernel, against this library's map (1e-5 normwise) and the FP64 oracle
    on a seeded subset (1e-5)."""
    import torch
    w = workloads.uniform_map(n_atoms=2048)
    g = w.dims[0]
    ta = torch.from_numpy(w.atoms).cuda()
    cols = _cols(w.atoms)
    ours = ctx.forward_3d(ta, w.dims, w.spacing, tune=ktt_b200.Tune(z_iterations=8, x_points=2)).reshape(-1)
    idx = workloads.subset_indices(g ** 3, 2e-4, seed=3)
    ref64 = oracle.points3d(w.atoms, w.spacing, w.dims, idx)
    scale = float(ours.abs().max())
    seen = set()
    failures = []
    for cfg in ref_kernels.space():
        key = (cfg["Z_ITERATIONS"], cfg["INNER_UNROLL_FACTOR"], cfg["USE_SOA"])
        shape = (cfg["WORK_GROUP_SIZE_X"], cfg["WORK_GROUP_SIZE_Y"])
        if (key, shape) in seen or shape not in ((32, 2), (16, 8)):
            continue
        seen.add((key, shape))
        out = torch.zeros(g ** 3, device="cuda")
        ref_kernels.run_tuned(cfg, ta, cols, w.atoms.shape[0], w.spacing, g, out)
        torch.cuda.synchronize()
        d = float((out - ours).abs().max()) / scale
        e = errors.report(out.cpu().numpy()[idx], ref64)["rel_norm"]
        if d > 1e-5 or e > 1e-5:
            failures.append((cfg, d, e))
    assert len(seen) == 84
    out = torch.zeros(g ** 3, device="cuda")
    ref_kernels.run_reference(ta, w.atoms.shape[0], w.spacing, g, out)
    torch.cuda.synchronize()
    assert float((out - ours).abs().max()) / scale <= 1e-5
    assert not failures, failures[:5]


@pytest.mark.skipif(not os.environ.get("KTT_REF_SWEEP_OUT"), reason="timing sweep is opt-in")
def test_time_ktt_space_on_the_full_map(ctx):
    """Device time of every configuration of KTT's CUDA space on the 256^3 x 65,536 map (one
    warm-up, best of two timed launches each), and of this library's chosen configuration."""
    import torch
    w = workloads.uniform_map()
    g = w.dims[0]
    ta = torch.from_numpy(w.atoms).cuda()
    cols = _cols(w.atoms)
    out = torch.zeros(g ** 3, device="cuda")
    pairs = float(g ** 3) * w.atoms.shape[0]
    rows = []
    for cfg in ref_kernels.space():
        times = []
        for rep in range(3):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            ref_kernels.run_tuned(cfg, ta, cols, w.atoms.shape[0], w.spacing, g, out)
            b.record()
            b.synchronize()
            if rep:
                times.append(a.elapsed_time(b))
        rows.append({**cfg, "ms": min(times), "gpairs_per_s": pairs / (min(times) * 1e-3) / 1e9})
    best = min(rows, key=lambda r: r["ms"])
    ref = []
    for rep in range(2):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        ref_kernels.run_reference(ta, w.atoms.shape[0], w.spacing, g, out)
        b.record()
        b.synchronize()
        ref.append(a.elapsed_time(b))
    tuned = ktt_b200.tuned("b200_map3d")
    mine = []
    for rep in range(3):
        ctx.forward_3d(ta, w.dims, w.spacing, tune=tuned, out=out.reshape(g, g, g))
        mine.append(ctx.elapsed_ms())
    result = {"workload": "256^3 grid, h 0.5, 65,536 atoms U[0,128)^3 (seed 2)", "configurations": rows,
              "best": best, "reference_kernel_ms": min(ref),
              "this_library": {"tune": tuned.as_dict(), "ms": min(mine[1:]),
                               "gpairs_per_s": pairs / (min(mine[1:]) * 1e-3) / 1e9},
              "nvrtc_options": ref_kernels.manifest()["options"]}
    with open(os.environ["KTT_REF_SWEEP_OUT"], "w") as f:
        json.dump(result, f, indent=1)
    assert best["ms"] > 0


@pytest.mark.skipif(not os.environ.get("KTT_REF_BATCH_OUT"), reason="timing comparison is opt-in")
def test_time_batch_against_ktt_kernels(ctx):
    """The 512-molecule uneven batch (seed 4, 8 A margin per side): this library's batched persistent
    kernel replayed from its CUDA graph, against one synchronous launch per molecule (what a loop of
    Tuner::Run calls does) of KTT's own directCoulombSum at its best B200 configuration and of
    directCoulombSumReference.  KTT's kernels evaluate cubic grids from a zero origin only
    (CoulombSum3d.cu:3-15), so each molecule runs on the cube of its largest side (a multiple of 16 for
    the reference kernel's launch) with its atoms shifted by the origin; rates count the pairs of the
    molecule's own grid (useful pairs) and, for KTT's kernels, also the cube's (evaluated pairs).
    Device time of each whole mode from one event pair, best of two; results to KTT_REF_BATCH_OUT."""
    import torch
    mols = workloads.molecule_batch(seed=4, n_mol=512)
    useful = float(sum(m.pairs for m in mols))
    tune = ktt_b200.tuned("b200_batch", "batched")
    inputs = [(torch.from_numpy(m.atoms).cuda(), m.dims, m.spacing, m.origin) for m in mols]
    batch = ktt_b200.Batch(ctx, inputs, tune)
    batch.run(ktt_b200.BATCH_GRAPH)
    ctx.synchronize()
    graph = []
    for _ in range(2):
        batch.run(ktt_b200.BATCH_GRAPH)
        graph.append(ctx.elapsed_ms())
    batch.close()

    with open(os.path.join(ref_kernels.REPO, "profiles", "ktt_kernel_space_b200.json")) as f:
        best = json.load(f)["best"]
    cfg = {k: best[k] for k in ("WORK_GROUP_SIZE_X", "WORK_GROUP_SIZE_Y", "Z_ITERATIONS", "INNER_UNROLL_FACTOR",
                                "USE_SOA")}
    shifted = []
    for m in mols:
        a = m.atoms.copy()
        a[:, :3] -= np.asarray(m.origin, dtype=np.float32)
        g = max(m.dims)
        shifted.append((torch.from_numpy(a).cuda(), _cols(a), a.shape[0], m.spacing, g, (g + 15) // 16 * 16))
    largest = max(s[5] for s in shifted)
    out = torch.zeros(largest ** 3, device="cuda")

    def loop(reference):
        stream = torch.cuda.current_stream()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for atoms, cols, n, h, g, g16 in shifted:
            if reference:
                ref_kernels.run_reference(atoms, n, h, g16, out)
            else:
                ref_kernels.run_tuned(cfg, atoms, cols, n, h, g, out)
            torch.cuda.synchronize()
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b)

    result = {"molecules": len(mols), "useful_pairs": useful, "batched_tune": tune.as_dict(),
              "graph_ms": min(graph), "graph_gpairs_per_s": useful / (min(graph) * 1e-3) / 1e9, "ktt_config": cfg}
    for name, reference, cubes in (("ktt_best", False, [s[4] for s in shifted]),
                                   ("ktt_reference", True, [s[5] for s in shifted])):
        loop(reference)  # warm-up: module loads
        ms = min(loop(reference) for _ in range(2))
        evaluated = float(sum(g ** 3 * s[2] for g, s in zip(cubes, shifted)))
        result[name] = {"ms": ms, "useful_gpairs_per_s": useful / (ms * 1e-3) / 1e9,
                        "evaluated_gpairs_per_s": evaluated / (ms * 1e-3) / 1e9,
                        "graph_speedup": ms / min(graph)}
    with open(os.environ["KTT_REF_BATCH_OUT"], "w") as f:
        json.dump(result, f, indent=1)
    assert result["ktt_best"]["graph_speedup"] > 0


# ---- KTT's N-body example ----

def _nbody_inputs(n, seed=11):
    import torch
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0.0, 20.0, (n, 4)).astype(np.float32)
    vel = rng.uniform(0.0, 20.0, (n, 4)).astype(np.float32)
    vel[:, 3] = 0.0
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in
         dict(pos=pos, vel=vel, px=pos[:, 0], py=pos[:, 1], pz=pos[:, 2], m=pos[:, 3], vx=vel[:, 0], vy=vel[:, 1],
              vz=vel[:, 2]).items()}
    return pos, vel, t


def _run_ktt_nbody(cfg, t, n, new_pos, new_vel):
    ref_kernels.run_nbody_tuned(cfg, 0.001, t["pos"], t["px"], t["py"], t["pz"], t["m"], new_pos, t["vel"], t["vx"],
                                t["vy"], t["vz"], new_vel, 0.5, 0.01, n)


def test_ktt_nbody_kernels_match_this_library(ctx):
    """KTT's N-body reference kernel and 24 seeded configurations of its tuned kernel on 8,192 bodies,
    against this library's step (positions and velocities within 1e-5 of their magnitude)."""
    import torch
    n = 8192
    pos, vel, t = _nbody_inputs(n)
    ours_p, ours_v = ktt_b200.nbody_step(ctx, t["pos"], t["vel"], 0.001, 0.5, 0.01)
    torch.cuda.synchronize()
    sp, sv = float(ours_p.abs().max()), float(ours_v.abs().max())
    new_p, new_v = torch.empty_like(t["pos"]), torch.empty_like(t["vel"])
    ref_kernels.run_nbody_reference(0.001, t["pos"], new_p, t["vel"], new_v, 0.5, 0.01, n)
    torch.cuda.synchronize()
    assert float((new_p - ours_p).abs().max()) <= 1e-5 * sp
    assert float((new_v - ours_v).abs().max()) <= 1e-5 * sv
    configs = ref_kernels.nbody_configs()
    rng = np.random.default_rng(7)
    bad = []
    for k in rng.choice(len(configs), 24, replace=False):
        cfg = configs[int(k)]
        new_p.zero_()
        new_v.zero_()
        try:
            _run_ktt_nbody(cfg, t, n, new_p, new_v)
        except ref_kernels.DeviceLimitsExceeded:
            continue
        torch.cuda.synchronize()
        dp = float((new_p - ours_p).abs().max()) / sp
        dv = float((new_v[:, :3] - ours_v[:, :3]).abs().max()) / sv
        if dp > 1e-5 or dv > 1e-5:
            bad.append((cfg, dp, dv))
    assert not bad, bad[:3]


@pytest.mark.skipif(not os.environ.get("KTT_REF_NBODY_SWEEP_OUT"), reason="timing sweep is opt-in")
def test_time_ktt_nbody_space():
    """Device time of the compiled sample of KTT's tuned N-body kernel space and of its reference
    kernel on the example's 131,072 bodies (one warm-up, best of two timed launches each)."""
    import torch
    n = 128 * 1024
    _, _, t = _nbody_inputs(n)
    new_p, new_v = torch.empty_like(t["pos"]), torch.empty_like(t["vel"])

    def timed(fn):
        times = []
        for rep in range(3):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            b.synchronize()
            if rep:
                times.append(a.elapsed_time(b))
        return min(times)

    rows, limited = [], []
    for cfg in ref_kernels.nbody_configs():
        plain = {k: v for k, v in cfg.items() if k != "function"}
        try:
            ms = timed(lambda: _run_ktt_nbody(cfg, t, n, new_p, new_v))
        except ref_kernels.DeviceLimitsExceeded:
            limited.append(plain)
            continue
        rows.append({**plain, "ms": ms, "ginteractions_per_s": n * n / (ms * 1e-3) / 1e9})
    ref_ms = timed(lambda: ref_kernels.run_nbody_reference(0.001, t["pos"], new_p, t["vel"], new_v, 0.5, 0.01, n))
    with open(os.environ["KTT_REF_NBODY_SWEEP_OUT"], "w") as f:
        json.dump({"n": n, "configurations": rows, "best": min(rows, key=lambda r: r["ms"]),
                   "device_limits_exceeded": limited, "reference_kernel_ms": ref_ms}, f, indent=1)
