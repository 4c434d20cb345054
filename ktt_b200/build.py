"""Build recipe for the native libraries of ktt_b200.

    python -m ktt_b200.build            # libcoulktt.so (CUDA kernels + C ABI) and libktt_b200.so (C++ tuner)

Every CUDA translation unit is compiled ahead of time for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``), in parallel, into
``ktt_b200/_build/``; the shared libraries are written into the package
directory so they travel with the source tree.  Objects are rebuilt when the
source or any header under ``ktt_b200/csrc`` or ``include`` is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(REPO, "include")
BUILD = os.path.join(HERE, "_build")
LIB_CUDA = os.path.join(HERE, "libcoulktt.so")
LIB_TUNER = os.path.join(HERE, "libktt_b200.so")
LAUNCHER = os.path.join(HERE, "ktt_tuning_launcher")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler",
                     "-fPIC,-fvisibility=hidden", "-I", INCLUDE, "-I", CSRC]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-Wextra", "-I", INCLUDE, "-I", CSRC]


def _nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    p = os.path.join(cuda, "bin", "nvcc")
    return p if os.path.exists(p) else (shutil.which("nvcc") or "nvcc")


def _cxx() -> str:
    # The system g++ (an inherited $CXX may point at a toolchain without the C++ runtime headers).
    return shutil.which("g++") or "g++"


def _newest_header() -> float:
    heads = glob.glob(os.path.join(CSRC, "**", "*.h"), recursive=True)
    heads += glob.glob(os.path.join(CSRC, "**", "*.cuh"), recursive=True)
    heads += glob.glob(os.path.join(INCLUDE, "**", "*.h"), recursive=True)
    return max((os.path.getmtime(h) for h in heads), default=0.0)


def _stale(obj: str, src: str, newest_header: float) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return t < os.path.getmtime(src) or t < newest_header


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: " + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def _compile_all(jobs: list[tuple[list[str], str]], workers: int) -> None:
    if not jobs:
        return
    with cf.ThreadPoolExecutor(max_workers=workers) as ex:
        futs = {ex.submit(_run, cmd): out for cmd, out in jobs}
        for f in cf.as_completed(futs):
            f.result()


def build(verbose: bool = False, workers: int | None = None) -> list[str]:
    """Compile (incrementally) and link both libraries; returns their paths."""
    os.makedirs(BUILD, exist_ok=True)
    workers = workers or max(1, os.cpu_count() or 1)
    newest = _newest_header()
    nvcc, cxx = _nvcc(), _cxx()

    cu_sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    cu_objs, jobs = [], []
    for src in cu_sources:
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        cu_objs.append(obj)
        if _stale(obj, src, newest):
            jobs.append(([nvcc] + NVCC_FLAGS + ["-c", src, "-o", obj], obj))
    if verbose:
        print(f"[ktt_b200.build] compiling {len(jobs)} CUDA units", file=sys.stderr)
    _compile_all(jobs, workers)
    if jobs or not os.path.exists(LIB_CUDA) or any(os.path.getmtime(o) > os.path.getmtime(LIB_CUDA) for o in cu_objs):
        _run([nvcc] + ARCH + ["-shared", "-o", LIB_CUDA] + cu_objs + ["-Xlinker", "-z,defs"])

    cpp_sources = sorted(glob.glob(os.path.join(CSRC, "ktt", "*.cpp")))
    out = [LIB_CUDA]
    if cpp_sources:
        cpp_objs, jobs = [], []
        for src in cpp_sources:
            obj = os.path.join(BUILD, "ktt_" + os.path.basename(src) + ".o")
            cpp_objs.append(obj)
            if _stale(obj, src, newest):
                jobs.append(([cxx] + CXX_FLAGS + ["-c", src, "-o", obj], obj))
        if verbose:
            print(f"[ktt_b200.build] compiling {len(jobs)} C++ units", file=sys.stderr)
        _compile_all(jobs, workers)
        if (jobs or not os.path.exists(LIB_TUNER) or os.path.getmtime(LIB_CUDA) > os.path.getmtime(LIB_TUNER)
                or any(os.path.getmtime(o) > os.path.getmtime(LIB_TUNER) for o in cpp_objs)):
            _run([cxx, "-shared", "-o", LIB_TUNER] + cpp_objs +
                 ["-L", HERE, "-lcoulktt", "-Wl,-rpath,$ORIGIN", "-pthread"])
        out.append(LIB_TUNER)
        # KTT's TuningLauncher counterpart: runs a JSON tuning script
        launcher_src = os.path.join(CSRC, "launcher", "ktt_tuning_launcher.cpp")
        if (not os.path.exists(LAUNCHER) or os.path.getmtime(LIB_TUNER) > os.path.getmtime(LAUNCHER)
                or _stale(LAUNCHER, launcher_src, newest)):
            _run([cxx] + CXX_FLAGS + [launcher_src, "-o", LAUNCHER, "-L", HERE, "-lktt_b200", "-lcoulktt",
                                      "-Wl,-rpath,$ORIGIN", "-pthread"])
        out.append(LAUNCHER)
        # the Python module of the ktt:: surface, under KTT's module name (pyktt)
        try:
            import sysconfig

            import pybind11
            pyktt = os.path.join(HERE, "pyktt" + sysconfig.get_config_var("EXT_SUFFIX"))
            pyktt_src = os.path.join(CSRC, "python", "pyktt.cpp")
            if (not os.path.exists(pyktt) or os.path.getmtime(LIB_TUNER) > os.path.getmtime(pyktt)
                    or _stale(pyktt, pyktt_src, newest)):
                if verbose:
                    print("[ktt_b200.build] compiling the pyktt module", file=sys.stderr)
                _run([cxx] + CXX_FLAGS + ["-shared", "-fvisibility=hidden", "-I", sysconfig.get_paths()["include"],
                                          "-I", pybind11.get_include(), pyktt_src, "-o", pyktt, "-L", HERE,
                                          "-lktt_b200", "-lcoulktt", "-Wl,-rpath,$ORIGIN"])
            out.append(pyktt)
        except ImportError:
            if verbose:
                print("[ktt_b200.build] pybind11 not importable: pyktt module not built", file=sys.stderr)
    return out


if __name__ == "__main__":
    for p in build(verbose=True):
        print(p)
