"""KTT's own known-answer tuning script (Examples/JSON/CoulombSum3d.json, committed unchanged in
content under tests/golden/ktt_scripts) run on the B200 through ktt_tuning_launcher, the
counterpart of KTT's TuningLauncher: 10 random configurations of KTT's 210-configuration space,
atoms from the script's generator, the map validated by the tuner against Coulomb3d.bin (KTT's
SideBySide criterion, 0.01).  Coulomb3d.bin is written by the oracle's FP32 restatement of KTT's
generate-coulomb-output.c, which reproduces that program's output bit for bit.  Every configuration
the searcher picks must pass the script's constraints and the tuner's validation."""
import os
import shutil
import subprocess
import xml.etree.ElementTree as ET

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SCRIPTS = os.path.join(REPO, "tests", "golden", "ktt_scripts")
LAUNCHER = os.path.join(REPO, "ktt_b200", "ktt_tuning_launcher")


def test_known_answer_script_on_b200(tmp_path):
    assert os.path.exists(LAUNCHER), "build ktt_b200 first (python -m ktt_b200.build)"
    shutil.copy(os.path.join(SCRIPTS, "CoulombSum3d.json"), tmp_path)
    atoms = oracle.kat_atoms(64)
    oracle.kat_fp32(atoms, 0.49, 256).astype(np.float32).tofile(tmp_path / "Coulomb3d.bin")
    r = subprocess.run([LAUNCHER, "CoulombSum3d.json"], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    root = ET.parse(tmp_path / "CoulombSumTuningOutput.xml").getroot()
    results = root.findall(".//Result")
    assert len(results) == 10, r.stderr[-2000:]
    for res in results:
        assert res.get("Status") == "Ok", ET.tostring(res)[:500]
        params = {c.get("Name"): int(c.get("Value")) for c in res.iter("Pair")}
        assert params["INNER_UNROLL_FACTOR"] < params["Z_ITERATIONS"]
        assert params["WORK_GROUP_SIZE_X"] * params["WORK_GROUP_SIZE_Y"] >= 64
