"""The autotuner on top of the ktt:: searchers (ktt_b200/autotune.py).

CPU: both tile spaces build through the tuner (parameters, KTT's thread modifiers, the block-size
constraint and the compiled-variant constraint) and every configuration the space keeps is one the
library accepts.  GPU: a short MCMC / random search on small workloads validates every configuration
against the FP64-merge map and returns a configuration whose map is then checked against the oracle.
"""
import itertools
import json
import subprocess
import sys

import numpy as np
import pytest

import ktt_b200
from ktt_b200 import autotune


def _kept(space, supported):
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


@pytest.mark.gpu
def test_map3d_search_short():
    import torch

    import oracle
    from ktt_b200 import workloads
    result = autotune.tune_map3d(grid=64, atoms=2048, searcher="mcmc", budget=8)
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
    result = autotune.tune_batch(molecules=12, seed=7, searcher="random", budget=6)
    assert len(result["trials"]) == 6
    assert all(t["status"] == "Ok" for t in result["trials"]), result["trials"]
    assert ktt_b200.batch_tune_supported(ktt_b200.Tune(**result["batched"]))
