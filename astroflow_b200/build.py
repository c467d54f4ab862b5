"""Build libastroflow_dd.so (the C-ABI dedispersion library) in-tree for sm_100a.

Usage: python -m astroflow_b200.build [--force]

Compile units:
  csrc/dd_fastmath.cu  device flags of the reference build (--use_fast_math ...), because
                       its kernels must reproduce the reference's fast-math delay tables
                       and zero-DM arithmetic bit for bit;
  csrc/dd_rfi.cu, csrc/dd_dedisp.cu  plain -O3 (IEEE arithmetic, explicit roundings);
  csrc/dd_api.cpp      host code, -ffp-contract=off, no fast-math;
  csrc/dd_hosttable.cpp  the reference CPU path's host flags (-Ofast, FMA, AVX2), because
                       the brute-force delay table must equal the reference build's.
The CUDA runtime is linked statically so the library does not depend on which
libcudart the host process (e.g. torch) has already loaded.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libastroflow_dd.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
          "--expt-relaxed-constexpr", "-I", os.path.join(HERE, "..", "include")]
FASTMATH = ["--use_fast_math", "--ftz=true", "--prec-div=false", "--prec-sqrt=false",
            "--fmad=true"]

UNITS = [
    ("dd_fastmath.cu", FASTMATH),
    ("dd_rfi.cu", []),
    ("dd_dedisp.cu", []),
    ("dd_probe.cu", []),
    ("dd_sumsmem.cu", []),
    ("dd_noalloc.cu", []),
    ("dd_single.cu", ["-Xcompiler", "-fno-fast-math"]),
    ("dd_image.cu", ["-Xcompiler", "-fno-fast-math"]),
    ("dd_ingest.cu", []),
]
HOST = ["dd_api.cpp"]
# The brute-force delay table in the reference's host arithmetic: its CPU path's
# flags (CMakeLists.txt:116-118; -march=native pinned to x86-64-v3, as the
# parity build of the reference does, so the library runs on any AVX2 host).
HOST_REFMATH = [("dd_hosttable.cpp", ["-std=gnu++17", "-Ofast", "-march=x86-64-v3", "-mtune=native",
                                      "-fno-math-errno", "-ffast-math", "-funroll-loops",
                                      "-fomit-frame-pointer", "-mfma", "-mavx2", "-msse4.2",
                                      "-DNDEBUG", "-fPIC"])]
HEADERS = ["dd_internal.h", os.path.join("..", "..", "include", "astroflow_dd.h")]


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:4])} ...")


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS]
    objs = []
    for src, extra in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or not _newer(o, [s, *headers, __file__]):
            cmd = [NVCC, *ARCH, *COMMON, *extra, "-c", s, "-o", o]
            if verbose:
                cmd += ["-Xptxas", "-v"]
            _run(cmd)
    for src in HOST:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or not _newer(o, [s, *headers, __file__]):
            _run(["g++", "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math",
                  "-Wall", "-I", os.path.join(CUDA, "include"), "-c", s, "-o", o])
    for src, flags in HOST_REFMATH:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or not _newer(o, [s, __file__]):
            _run(["g++", *flags, "-c", s, "-o", o])
    if force or not _newer(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-cudart", "static"])
    return LIB


if __name__ == "__main__":
    path = build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(path)
