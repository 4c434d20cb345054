"""CPU tests of the script evaluator and the JSON tuning-script loader of the ktt:: surface.

* The Python expression subset of KTT's scripts, evaluated natively, against Python itself: a
  hand-written list of the semantics that differ between languages (floored division and modulo,
  true division, power, chained comparisons, and/or returning operands, conditional expressions,
  comprehensions, built-ins) and 400 seeded random expressions.
* The generator of KTT's known-answer script, evaluated natively, against Python bit for bit, and
  against the known-answer generator's own atoms.
* A configuration space built from parameter, constraint and modifier scripts: KTT's 210.
* KTT's CUDA tuning script for this path (tests/golden/ktt_scripts, from the KTT tree) run through
  the loader in simulated-tuning mode over the recorded 2080 Ti results: all 210 configurations,
  the recorded best, a KTT-format result file; "$NAME" parameters; malformed scripts rejected.
The driver tests/cpp/loader_cpu_tests.cpp is compiled here against the built library."""
import json
import os
import random
import shutil
import subprocess

import numpy as np
import pytest

import oracle

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")
SCRIPTS = os.path.join(GOLDEN, "ktt_scripts")
KAT_GENERATOR = "1+(i//4)*(0.1 + 0.05*(i%4)) if i%4 < 3 else ((i//4)%10)*0.1"


@pytest.fixture(scope="session")
def driver(tmp_path_factory):
    from ktt_b200 import build as kb
    kb.build()
    out = tmp_path_factory.mktemp("loader") / "loader_cpu_tests"
    lib = os.path.join(REPO, "ktt_b200")
    subprocess.run([shutil.which("g++") or "g++", "-std=c++17", "-O1", "-Wall", "-I", os.path.join(REPO, "include"),
                    "-I", os.path.join(REPO, "ktt_b200", "csrc"), os.path.join(REPO, "tests", "cpp", "loader_cpu_tests.cpp"),
                    "-o", str(out), "-L", lib, "-lktt_b200", "-lcoulktt", f"-Wl,-rpath,{lib}"], check=True)
    return str(out)


def _parse(text):
    kind, _, rest = text.partition(" ")
    if kind == "int":
        return int(rest)
    if kind == "bool":
        return bool(int(rest))
    if kind == "float":
        return float(rest)
    if kind == "list":
        inner = rest[1:-1]
        items, depth, cur = [], 0, ""
        for c in inner:
            if c == "," and depth == 0:
                items.append(cur.strip())
                cur = ""
                continue
            depth += c == "["
            depth -= c == "]"
            cur += c
        if cur.strip():
            items.append(cur.strip())
        return [_parse(i) for i in items]
    if kind == "error":
        return Exception(rest)
    raise ValueError(text)


def _evaluate(driver, expressions):
    r = subprocess.run([driver, "eval"], input="\n".join(expressions) + "\n", capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.splitlines()
    assert len(lines) == len(expressions)
    return [_parse(line) for line in lines]


def _same(native, expected):
    if isinstance(expected, Exception):
        return isinstance(native, Exception)
    if isinstance(native, Exception):
        return False
    if isinstance(expected, list):
        return isinstance(native, list) and len(native) == len(expected) and all(
            _same(a, b) for a, b in zip(native, expected))
    if type(expected) is bool or type(native) is bool:
        return type(expected) is type(native) and expected == native
    if isinstance(expected, float) or isinstance(native, float):
        if not (isinstance(expected, float) and isinstance(native, float)):
            return False
        return native == expected or abs(native - expected) <= 1e-12 * max(abs(expected), 1e-300)
    return native == expected


def _python(expression):
    try:
        return eval(expression, {"__builtins__": {}}, {"a": 7, "b": -3, "x": 2.5, "min": min, "max": max, "abs": abs,
                                                        "int": int, "float": float, "bool": bool, "round": round,
                                                        "len": len, "range": lambda *r: list(range(*r)), "list": list,
                                                        "pow": pow})
    except Exception as e:  # noqa: BLE001 -- any Python error must be an error natively too
        return e


HAND = [
    "7 // 2", "-7 // 2", "7 // -2", "-7 % 3", "7 % -3", "7.5 // 2", "-7.5 % 2", "7 / 2", "6 / 3", "2 ** 10",
    "-2 ** 2", "2 ** -1", "(-2) ** 3", "2 ** 3 ** 2", "1 if a < b else 5", "a if a > b else b", "1 < 2 < 3",
    "3 > 2 > 2", "1 == 1.0", "0 or 5", "3 and 0", "not 0", "not []", "[] or [1]", "True + 1", "-True",
    "[y * 2 for y in range(4) if y != 2]",
    "min([3, 1, 2])", "max(1, 2.5)", "min(a, b, x)", "abs(b)", "abs(-x)", "round(2.5)", "round(3.5)", "round(-0.5)",
    "round(x, 0)", "int(-2.7)", "float(a)", "bool(0.0)", "len(range(5))", "list(range(2, 9, 3))", "pow(2, 5)",
    "[1, 2] + [3]", "[1, 2] == [1, 2]", "x // 1", "-x % 2", "1e3", "1.5e-2 * 2", ".5 + 1", "1_000 + 1",
    "1 / 0", "1 // 0", "1 % 0.0", "foo", "import os", "1 +", "a.b", "range(0, 5, 0)", "WORK_GROUP_SIZE_X * 2",
    KAT_GENERATOR.replace("i", "a"),
]
# valid Python outside the subset: rejected with an error, never evaluated differently
OUTSIDE = ["'str'", "[1, 2][0]", "[[i, j] for i in range(2) for j in range(2)]", "lambda: 1", "{1: 2}"]


def test_expressions_match_python(driver):
    native = _evaluate(driver, HAND)
    bad = [(e, n, _python(e)) for e, n in zip(HAND, native) if not _same(n, _python(e))]
    assert not bad, bad
    assert all(isinstance(n, Exception) for n in _evaluate(driver, OUTSIDE))


def _random_expression(rng, depth=0):
    if depth > 3 or rng.random() < 0.25:
        return rng.choice([str(rng.randint(-9, 99)), f"{rng.uniform(-50, 50):.3f}", "a", "b", "x", "True", "False"])
    kind = rng.random()
    l, r = _random_expression(rng, depth + 1), _random_expression(rng, depth + 1)
    if kind < 0.45:
        return f"({l} {rng.choice(['+', '-', '*', '/', '//', '%'])} {r})"
    if kind < 0.55:
        return f"({rng.randint(-5, 9)} ** {rng.randint(0, 3)})"
    if kind < 0.7:
        return f"({l} {rng.choice(['<', '<=', '>', '>=', '==', '!='])} {r})"
    if kind < 0.8:
        return f"({l} {rng.choice(['and', 'or'])} {r})"
    if kind < 0.85:
        return f"(not {l})"
    if kind < 0.95:
        return f"({l} if {_random_expression(rng, depth + 1)} else {r})"
    return f"{rng.choice(['min', 'max'])}({l}, {r})"


def test_random_expressions_match_python(driver):
    rng = random.Random(20261203)
    exprs = [_random_expression(rng) for _ in range(400)]
    native = _evaluate(driver, exprs)
    bad = [(e, n, _python(e)) for e, n in zip(exprs, native) if not _same(n, _python(e))]
    assert not bad, bad[:5]


def test_kat_generator(driver, tmp_path):
    out = tmp_path / "atoms.bin"
    subprocess.run([driver, "generator", KAT_GENERATOR, "256", str(out)], check=True, timeout=60)
    native = np.fromfile(out, dtype=np.float32)
    python = np.array([eval(KAT_GENERATOR, {}, {"i": i}) for i in range(256)], dtype=np.float32)
    assert np.array_equal(native.view(np.uint32), python.view(np.uint32))
    # KTT's script describes the known-answer generator's atoms, formed there in FP32 arithmetic
    np.testing.assert_allclose(native, oracle.kat_atoms(64).reshape(-1), rtol=2e-7, atol=1e-6)


def test_space_from_scripts(driver):
    r = subprocess.run([driver, "space"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "configurations 210" in r.stdout


def _recorded_results(path):
    g = json.load(open(os.path.join(GOLDEN, "coulomb3d_2080_space.json")))
    results = []
    for r in g["Results"]:
        results.append({
            "ComputationResults": [{"CompilationData": {}, "Duration": r["Duration"],
                                    "GlobalSize": dict(zip("XYZ", r["GlobalSize"])), "KernelFunction": "directCoulombSum",
                                    "LocalSize": dict(zip("XYZ", r["LocalSize"])), "Overhead": 0.0}],
            "Configuration": [{"Name": n, "Value": v, "ValueType": "UnsignedInt"} for n, v in r["Configuration"]],
            "DataMovementOverhead": 0.0, "ExtraDuration": 0.0, "KernelName": "CoulombSum", "SearcherOverhead": 0.0,
            "Status": r["Status"], "TotalDuration": r["TotalDuration"], "TotalOverhead": 0.0, "ValidationOverhead": 0.0})
    with open(path, "w") as f:
        json.dump({"Metadata": dict(g["Metadata"]), "Results": results}, f)
    return g


def _best_recorded(g):
    best = min((r for r in g["Results"] if r["Status"] == "Ok"), key=lambda r: r["TotalDuration"])
    return {n: v for n, v in best["Configuration"]}


def _run_script(driver, workdir, script, *params):
    return subprocess.run([driver, "script", script, *params], capture_output=True, text=True, timeout=300,
                          cwd=workdir)


def test_ktt_cuda_script_simulated(driver, tmp_path):
    shutil.copy(os.path.join(SCRIPTS, "CoulombSum3dCudaScript.json"), tmp_path)
    g = _recorded_results(tmp_path / "coulomb_2080_full_search_space.json")
    r = _run_script(driver, tmp_path, "CoulombSum3dCudaScript.json")
    assert r.returncode == 0, r.stdout + r.stderr
    # the profile-based searcher is not available: the loader says so and the default searcher replays all
    assert "profile-based searcher" in r.stderr
    head, best = r.stdout.strip().split(" best ")
    assert head == "results 210 configurations 210"
    assert dict(p.split("=") for p in best.split(",")) == {k: str(v) for k, v in _best_recorded(g).items()}
    out = json.load(open(tmp_path / "CoulombSumTuningOutput.json"))
    assert len(out["Results"]) == 210 and out["Metadata"]["TimeUnit"] == "Microseconds"


def test_script_parameters_and_budget(driver, tmp_path):
    doc = json.load(open(os.path.join(SCRIPTS, "CoulombSum3dCudaScript.json")))
    doc["Search"] = {"Name": "Random"}
    doc["Budget"] = [{"Type": "ConfigurationCount", "BudgetValue": "$COUNT"}]
    text = json.dumps(doc).replace('"$COUNT"', "$COUNT")
    (tmp_path / "script.json").write_text(text)
    _recorded_results(tmp_path / "coulomb_2080_full_search_space.json")
    r = _run_script(driver, tmp_path, "script.json", "COUNT=17")
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("results 17 configurations 210")


@pytest.mark.parametrize("change, message", [
    (lambda d: d.pop("KernelSpecification"), "KernelSpecification"),
    (lambda d: d["KernelSpecification"].update(Language="OpenCL"), "OpenCL"),
    (lambda d: d.update(Search={"Name": "Annealing"}), "searcher"),
    (lambda d: d["ConfigurationSpace"]["Conditions"][0].update(Expression="Z_ITERATIONS <"), "syntax"),
    (lambda d: d["KernelSpecification"]["Arguments"][0].update(FillType="Script"), "fill type"),
])
def test_malformed_scripts_rejected(driver, tmp_path, change, message):
    doc = json.load(open(os.path.join(SCRIPTS, "CoulombSum3dCudaScript.json")))
    change(doc)
    (tmp_path / "bad.json").write_text(json.dumps(doc))
    _recorded_results(tmp_path / "coulomb_2080_full_search_space.json")
    r = _run_script(driver, tmp_path, "bad.json")
    assert r.returncode != 0 or "results 0" in r.stdout or message in r.stderr, r.stdout + r.stderr
    assert message in r.stdout + r.stderr
