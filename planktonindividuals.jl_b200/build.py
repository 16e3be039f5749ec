"""Builds libpib200.so (sm_100a) in-tree next to the Python package.

    python planktonindividuals.jl_b200/build.py

Each translation unit has its own floating-point flags:
  pib200.cu  (FP64 form)  -fmad=false keeps every multiply and add separately rounded so the
                          Float64 path produces the same bits as the CPU oracle, which is compiled
                          with -ffp-contract=off;
  fp32.cu    (FP32 form)  default contraction and -prec-div=false: fused multiply-adds and the
                          approximate (2 ulp) division are faster, and the FP32 form is compared
                          with the oracle within a tolerance.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "PlanktonIndividuals", "libpib200.so")
SOURCES = {"pib200.cu": ["-fmad=false", "-Xcompiler", "-ffp-contract=off"],
           "fp32.cu": ["-prec-div=false"]}
DEPS = ["pib200.cu", "kernels_fp64.cuh", "kernels_abiotic.cuh", "kernels_iron.cuh", "pib200_internal.h", "noalloc.cu", "host_common.h",
        "fp32.cu", "kernels_fp32.cuh", "fp32_internal.h", "kernels_tracer.cuh"]
BUILD_DIR = os.path.join(HERE, "_build")


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def host_compiler():
    # the default $CXX wrapper of this image lacks some runtime spec files; prefer the system g++
    for c in ("/usr/bin/g++", shutil.which("g++")):
        if c and os.path.exists(c):
            return c
    return None


def needs_build():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, d) for d in DEPS]
    deps += [os.path.join(HERE, "..", "include", h) for h in ("pib200.h", "pi_numerics.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    if not force and not needs_build():
        return OUT
    os.makedirs(BUILD_DIR, exist_ok=True)
    base = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
            "-Xcompiler", "-fPIC"]
    hc = host_compiler()
    if hc:
        base[1:1] = ["-ccbin", hc]
    objs = []
    for src, flags in SOURCES.items():
        obj = os.path.join(BUILD_DIR, src.replace(".cu", ".o"))
        cmd = base + flags + ["-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.append("-Xptxas=-v")
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(obj)
    subprocess.run(base + ["-shared", "-o", OUT] + objs, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
