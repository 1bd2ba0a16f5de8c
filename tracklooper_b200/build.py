"""Builds the in-tree native libraries of the package.

  _lst_b200.so  CUDA kernels + host runtime + C ABI (include/lst_b200.h),
                compiled for sm_100a with IEEE single-precision arithmetic
                (no FMA contraction, IEEE division and square root), which the
                bit-exact parity with the reference CPU backend relies on.
  _lstgen.so    seeded synthetic event generator (host only).

Usage: python -m tracklooper_b200.build [--force]
"""
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")

LIB = os.path.join(PKG, "_lst_b200.so")
GEN_LIB = os.path.join(PKG, "_lstgen.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC,-O2,-ffp-contract=off,-fno-fast-math",
    "-shared",
]

LIB_SOURCES = ["lst_event.cu", "lst_dnn.cu", "es.cc", "es_device.cu"]
LIB_DEPS = ["lst_core.h", "lst_md.h", "lst_ls.h", "lst_t3.h", "lst_t5.h", "lst_pixel.h", "lst_device.h",
            "lst_kernels.cuh", "lst_fields.h", "lst_seed.h", "es.h"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _stale(target, inputs):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(p) > t for p in inputs)


def build_lib(force=False, extra_flags=()):
    srcs = [os.path.join(CSRC, s) for s in LIB_SOURCES]
    deps = srcs + [os.path.join(CSRC, d) for d in LIB_DEPS] + [os.path.join(INCLUDE, "lst_b200.h")]
    if not force and not _stale(LIB, deps):
        return LIB
    cmd = [_nvcc()] + NVCC_FLAGS + list(extra_flags) + ["-I", INCLUDE, "-I", CSRC, "-o", LIB + ".tmp"] + srcs
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


def build_gen(force=False):
    src = os.path.join(CSRC, "gen", "lstgen.cc")
    if not force and not _stale(GEN_LIB, [src]):
        return GEN_LIB
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-o", GEN_LIB + ".tmp", src]
    subprocess.run(cmd, check=True)
    os.replace(GEN_LIB + ".tmp", GEN_LIB)
    return GEN_LIB


def build_all(force=False):
    build_gen(force)
    build_lib(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
