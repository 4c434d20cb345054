"""The autotuner on top of the ktt:: searchers (ktt_b200/autotune.py).

CPU: both tile spaces build through the tuner (parameters, KTT's thread modifiers, the block-size
constraint and the compiled-variant constraint) and every configuration the space keeps is one the
library accepts.  GPU: a short MCMC / random search on small workloads with the FP64 oracle registered
as the tuner's reference computation (Tuner::SetReferenceComputation) validates every configuration
against it and returns a configuration whose map is then checked against the oracle again; the
library's FP64 reference kernel (the default reference computation) agrees with the oracle.  Opt-in
(KTT_AUTOTUNE_OUT=path): the full 256^3 x 65,536 search validated against the oracle, written to path.
"""
import itertools
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import ktt_b200
from ktt_b200 import autotune


def _kept(space, supported, precisions=(0,)):
    space = dict(space, PRECISION=list(precisions))
    names = list(space)
    kept = 0
    for values in itertools.product(*space.values()):
        v = dict(zip(names, values))
        if 32 <= v["WORK_GROUP_SIZE_X"] * v["WORK_GROUP_SIZE_Y"] <= 256 and supported(autotune._tune_from(values, names)):
            kept += 1
    return kept


def test_map3d_space_is_the_compiled_variants():
    n = autotune.tune_map3d(grid=64, atoms=64, dry_run=True)["configurations"]
    assert n == _kept(autotune.MAP3D_SPACE, ktt_b200.tune_supported)
    assert n >= 100
    # the precise forms' space (compensated and FP64 merge)
    n = autotune.tune_map3d(grid=64, atoms=64, dry_run=True, precisions=(1, 2))["configurations"]
    assert n == _kept(autotune.MAP3D_SPACE, ktt_b200.tune_supported, (1, 2))
    assert n >= 100


def test_batch_space_is_the_compiled_variants():
    n = autotune.tune_batch(molecules=2, dry_run=True)["configurations"]
    assert n == _kept(autotune.BATCH_SPACE, ktt_b200.batch_tune_supported)
    assert n >= 20


def test_stored_configurations_are_in_the_spaces():
    # the configurations bench.py and ktt_b200.Batch read are ones the library still compiles
    assert ktt_b200.tune_supported(ktt_b200.tuned("b200_map3d"))
    assert ktt_b200.batch_tune_supported(ktt_b200.tuned("b200_batch", "batched"))


def test_cli_dry_run():
    out = subprocess.run([sys.executable, "-m", "ktt_b200.autotune", "batch", "--dry-run", "--molecules", "2"],
                         capture_output=True, text=True, timeout=300, check=True).stdout
    assert json.loads(out.strip().splitlines()[-1])["configurations"] > 0


class _Spy:
    """The oracle as a reference computation, counting its calls."""

    def __init__(self):
        import oracle
        self.fn = oracle.grid3d
        self.calls = 0

    def __call__(self, atoms, spacing, dims, origin):
        self.calls += 1
        return self.fn(atoms, spacing, dims, origin)


@pytest.mark.gpu
def test_map3d_search_short():
    import torch

    import oracle
    from ktt_b200 import workloads
    spy = _Spy()
    result = autotune.tune_map3d(grid=64, atoms=2048, searcher="mcmc", budget=8, reference=spy,
                                 reference_name="FP64 oracle (oracle/coulomb_oracle.c)")
    assert spy.calls == 1 and result["reference"] == "FP64 oracle (oracle/coulomb_oracle.c)"
    valid = [t for t in result["trials"] if t["gpairs_per_s"] is not None]
    assert len(result["trials"]) == 8 and len(valid) == 8
    tune = ktt_b200.Tune(**result["tune"])
    assert ktt_b200.tune_supported(tune)
    w = workloads.uniform_map(n_atoms=2048, n=64, box=32.0)
    ref = oracle.grid3d(w.atoms, w.spacing, w.dims)
    ctx = ktt_b200.CoulombContext(0)
    try:
        v = ctx.forward_3d(torch.from_numpy(w.atoms).cuda(), w.dims, w.spacing, tune=tune).cpu().numpy()
    finally:
        ctx.close()
    assert np.linalg.norm(v - ref) / np.linalg.norm(ref) <= 1e-5


@pytest.mark.gpu
def test_batch_search_short():
    spy = _Spy()
    result = autotune.tune_batch(molecules=12, seed=7, searcher="random", budget=6, reference=spy)
    assert spy.calls == 12
    assert len(result["trials"]) == 6
    assert all(t["status"] == "Ok" for t in result["trials"]), result["trials"]
    assert ktt_b200.batch_tune_supported(ktt_b200.Tune(**result["batched"]))


@pytest.mark.gpu
def test_precise_forms_searched_and_validated():
    """PRECISION as a searched parameter: the map search over both FP64-merge forms and the batch
    search over the shared-sum form validate every configuration they try against the reference."""
    spy = _Spy()
    result = autotune.tune_map3d(grid=64, atoms=2048, searcher="random", budget=6, reference=spy,
                                 precisions=(ktt_b200.PREC_FP64_MERGE, ktt_b200.PREC_FP64_MERGE_SHARED))
    assert all(t["status"] == "Ok" for t in result["trials"]), result["trials"]
    assert result["tune"]["precision"] in (ktt_b200.PREC_FP64_MERGE, ktt_b200.PREC_FP64_MERGE_SHARED)
    batch = autotune.tune_batch(molecules=10, seed=8, searcher="random", budget=5, reference=_Spy(),
                                precisions=(ktt_b200.PREC_FP64_MERGE_SHARED,))
    assert all(t["status"] == "Ok" for t in batch["trials"]), batch["trials"]
    assert batch["batched"]["precision"] == ktt_b200.PREC_FP64_MERGE_SHARED and batch["precisions"] == [4]


@pytest.mark.gpu
def test_fp64_reference_kernel_matches_the_oracle():
    import torch

    import oracle
    from ktt_b200 import workloads
    w = workloads.uniform_map(n_atoms=1500, n=40, box=20.0)
    dims = (40, 36, 28)
    origin = (-1.5, 0.25, 2.0)
    ref = oracle.grid3d(w.atoms, w.spacing, dims, origin)
    ctx = ktt_b200.CoulombContext(0)
    try:
        got = ctx.forward_3d_reference_fp64(torch.from_numpy(w.atoms).cuda(), dims, w.spacing, origin).cpu().numpy()
    finally:
        ctx.close()
    assert got.shape == ref.shape
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))
    # the default reference computation of the autotuner is this kernel
    maps = autotune._fp64_maps([(w.atoms, dims, w.spacing, origin)], None)
    assert np.max(np.abs(maps[0] - ref)) <= 1e-12 * np.max(np.abs(ref))


@pytest.mark.gpu
@pytest.mark.skipif(not os.environ.get("KTT_AUTOTUNE_OUT"), reason="the full search is opt-in")
def test_full_map3d_search_validated_against_the_oracle():
    """The search behind ktt_b200/tuned/b200_map3d.json: 256^3 x 65,536 atoms, MCMC, every configuration
    validated against the FP64 oracle's full map (about 100 s on 16 host cores, once)."""
    precisions = tuple(int(p) for p in os.environ.get("KTT_AUTOTUNE_PRECISIONS", "1,2").split(","))
    result = autotune.tune_map3d(grid=256, atoms=65536, searcher="mcmc",
                                 budget=int(os.environ.get("KTT_AUTOTUNE_BUDGET", "150")), reference=_Spy(),
                                 reference_name="FP64 oracle (oracle/coulomb_oracle.c), full map",
                                 precisions=precisions)
    with open(os.environ["KTT_AUTOTUNE_OUT"], "w") as f:
        json.dump(result, f, indent=1)
        f.write("\n")
    assert ktt_b200.tune_supported(ktt_b200.Tune(**result["tune"]))
