"""Compile KTT's own CUDA Coulomb kernels the way KTT does, for the GPU parity tests (test
infrastructure; nothing in the library loads these).

KTT's CUDA engine compiles a kernel with NVRTC after prepending the configuration as one
"#define NAME VALUE" line per parameter in the order the parameters were added
(Source/Api/Configuration/KernelConfiguration.cpp:25-34), with the user's compiler options followed by
"--gpu-architecture=compute_<major><minor>" (Source/ComputeEngine/Cuda/CudaEngine.cpp:740-755,
921-932) and CoulombSum3d's "-use_fast_math" (Examples/CoulombSum3d/CoulombSum3d.cpp:121).  This
script does the same from the sources where they lie in the KTT tree, except that NVRTC also
finishes the compile for sm_100 (KTT leaves that step to the driver at module load), and writes one
cubin per (Z_ITERATIONS, INNER_UNROLL_FACTOR, USE_SOA) of KTT's CUDA space for CoulombSum3d
(Examples/CoulombSum3d/CoulombSum3d.cpp:137-212: the work-group sizes only change the launch) plus
the reference kernel, into oracle/_ref/kernels/.

    python oracle/build_ref_kernels.py [--ktt-root DIR] [--out DIR]
"""
from __future__ import annotations

import argparse
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# parameter order of CoulombSum3d.cpp's AddParameter calls (CUDA build, non-dense space)
PARAM_ORDER = ("WORK_GROUP_SIZE_X", "WORK_GROUP_SIZE_Y", "WORK_GROUP_SIZE_Z", "Z_ITERATIONS",
               "INNER_UNROLL_FACTOR", "USE_CONSTANT_MEMORY", "USE_SOA", "VECTOR_SIZE")
OPTIONS = ("-use_fast_math", "--gpu-architecture=sm_100")


def space():
    """(Z_ITERATIONS, INNER_UNROLL_FACTOR, USE_SOA) of the CUDA space (INNER_UNROLL_FACTOR < Z)."""
    for z in (1, 2, 4, 8, 16, 32):
        for u in (0, 1, 2, 4, 8, 16, 32):
            if u < z:
                for s in (0, 1):
                    yield z, u, s


def nbody_space():
    """A sample of the CUDA space of Examples/Nbody/Nbody.cpp:140-209, in its parameter order:
    WORK_GROUP_SIZE_X {64..512} x WORK_GROUP_SIZE_Y {1, 2, 4} x OUTER_UNROLL_FACTOR {1, 2, 4, 8} x
    (USE_SOA, VECTOR_TYPE) {(0, 1), (1, 1), (1, 4)} x LOCAL_MEM {0, 1}, INNER_UNROLL_FACTOR1/2 = 0,
    under the example's constraints (64 <= WGX * WGY <= 1024, vector types only with SoA)."""
    for wx in (64, 128, 256, 512):
        for wy in (1, 2, 4):
            if not 64 <= wx * wy <= 1024:
                continue
            for ouf in (1, 2, 4, 8):
                for soa, vt in ((0, 1), (1, 1), (1, 4)):
                    for local in (0, 1):
                        yield {"WORK_GROUP_SIZE_X": wx, "WORK_GROUP_SIZE_Y": wy, "OUTER_UNROLL_FACTOR": ouf,
                               "INNER_UNROLL_FACTOR1": 0, "INNER_UNROLL_FACTOR2": 0, "USE_SOA": soa,
                               "LOCAL_MEM": local, "USE_CONSTANT_MEMORY": 0, "VECTOR_TYPE": vt}


def lowered_name(source: str, name: str, defines: dict | None, kernel: str) -> str:
    """The mangled name of a kernel that is not declared extern "C" (KTT registers the kernel name as
    an NVRTC name expression and looks up its lowered name, Source/ComputeEngine/Cuda/CudaProgram.cpp)."""
    from cuda.bindings import nvrtc
    prefix = "".join(f"#define {k} {v}\n" for k, v in (defines or {}).items())
    err, prog = nvrtc.nvrtcCreateProgram((prefix + source).encode(), name.encode(), 0, [], [])
    try:
        nvrtc.nvrtcAddNameExpression(prog, kernel.encode())
        opts = [o.encode() for o in OPTIONS]
        err, = nvrtc.nvrtcCompileProgram(prog, len(opts), opts)
        if err != nvrtc.nvrtcResult.NVRTC_SUCCESS:
            raise RuntimeError(f"nvrtcCompileProgram {name}: {err}")
        err, lowered = nvrtc.nvrtcGetLoweredName(prog, kernel.encode())
        if err != nvrtc.nvrtcResult.NVRTC_SUCCESS:
            raise RuntimeError(f"nvrtcGetLoweredName {kernel}: {err}")
        return lowered.decode() if isinstance(lowered, bytes) else str(lowered)
    finally:
        nvrtc.nvrtcDestroyProgram(prog)


def compile_cubin(source: str, name: str, defines: dict | None) -> bytes:
    from cuda.bindings import nvrtc
    prefix = "".join(f"#define {k} {v}\n" for k, v in (defines or {}).items())
    err, prog = nvrtc.nvrtcCreateProgram((prefix + source).encode(), name.encode(), 0, [], [])
    if err != nvrtc.nvrtcResult.NVRTC_SUCCESS:
        raise RuntimeError(f"nvrtcCreateProgram: {err}")
    try:
        opts = [o.encode() for o in OPTIONS]
        err, = nvrtc.nvrtcCompileProgram(prog, len(opts), opts)
        if err != nvrtc.nvrtcResult.NVRTC_SUCCESS:
            _, n = nvrtc.nvrtcGetProgramLogSize(prog)
            log = b" " * n
            nvrtc.nvrtcGetProgramLog(prog, log)
            raise RuntimeError(f"nvrtcCompileProgram {name} {defines}: {log.decode(errors='replace')}")
        _, n = nvrtc.nvrtcGetCUBINSize(prog)
        cubin = b" " * n
        err, = nvrtc.nvrtcGetCUBIN(prog, cubin)
        if err != nvrtc.nvrtcResult.NVRTC_SUCCESS:
            raise RuntimeError(f"nvrtcGetCUBIN: {err}")
        return cubin
    finally:
        nvrtc.nvrtcDestroyProgram(prog)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ktt-root", default=os.environ.get("KTT_ROOT"), required="KTT_ROOT" not in os.environ,
                    help="KTT source tree (default: $KTT_ROOT)")
    ap.add_argument("--out", default=os.path.join(HERE, "_ref", "kernels"))
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    tuned = os.path.join(args.ktt_root, "Examples", "CoulombSum3d", "CoulombSum3d.cu")
    ref = os.path.join(args.ktt_root, "Examples", "CoulombSum3d", "CoulombSum3dReference.cu")
    with open(tuned) as f:
        tuned_src = f.read()
    with open(ref) as f:
        ref_src = f.read()
    manifest = {"options": list(OPTIONS), "kernels": {}}
    for z, u, s in space():
        values = {"WORK_GROUP_SIZE_X": 32, "WORK_GROUP_SIZE_Y": 4, "WORK_GROUP_SIZE_Z": 1, "Z_ITERATIONS": z,
                  "INNER_UNROLL_FACTOR": u, "USE_CONSTANT_MEMORY": 0, "USE_SOA": s, "VECTOR_SIZE": 1}
        fname = f"coulomb3d_z{z}_u{u}_soa{s}.cubin"
        with open(os.path.join(args.out, fname), "wb") as f:
            f.write(compile_cubin(tuned_src, "CoulombSum3d.cu", {k: values[k] for k in PARAM_ORDER}))
        manifest["kernels"][fname] = {"Z_ITERATIONS": z, "INNER_UNROLL_FACTOR": u, "USE_SOA": s}
    with open(os.path.join(args.out, "coulomb3d_reference.cubin"), "wb") as f:
        f.write(compile_cubin(ref_src, "CoulombSum3dReference.cu", None))
    manifest["kernels"]["coulomb3d_reference.cubin"] = {"reference": True}

    # KTT's N-body example: the reference kernel and a sample of the tuned kernel's CUDA space
    nbody_dir = os.path.join(args.ktt_root, "Examples", "Nbody")
    with open(os.path.join(nbody_dir, "Nbody.cu")) as f:
        nbody_src = f.read()
    with open(os.path.join(nbody_dir, "NbodyReference.cu")) as f:
        nbody_ref_src = f.read()
    with open(os.path.join(args.out, "nbody_reference.cubin"), "wb") as f:
        f.write(compile_cubin(nbody_ref_src, "NbodyReference.cu", None))
    manifest["kernels"]["nbody_reference.cubin"] = {"reference": True}
    # neither N-body kernel is extern "C": record the names to look up in the cubins (the tuned kernel's
    # name depends on VECTOR_TYPE, which sets the type of its array parameters)
    manifest["kernels"]["nbody_reference.cubin"]["function"] = lowered_name(
        nbody_ref_src, "NbodyReference.cu", None, "nbody_kernel_reference")
    names = {}
    for values in nbody_space():
        if values["VECTOR_TYPE"] not in names:
            names[values["VECTOR_TYPE"]] = lowered_name(nbody_src, "Nbody.cu", values, "nbody_kernel")
    failed = []
    for values in nbody_space():
        fname = "nbody_" + "_".join(f"{v}" for v in values.values()) + ".cubin"
        try:
            cubin = compile_cubin(nbody_src, "Nbody.cu", values)
        except RuntimeError:
            failed.append(values)  # e.g. static shared memory beyond 48 KB: KTT reports CompilationFailed
            continue
        with open(os.path.join(args.out, fname), "wb") as f:
            f.write(cubin)
        manifest["kernels"][fname] = dict(values, function=names[values["VECTOR_TYPE"]])
    manifest["nbody_compilation_failed"] = failed
    with open(os.path.join(args.out, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1)
    print(f"{len(manifest['kernels'])} cubins in {args.out}")


if __name__ == "__main__":
    main()
