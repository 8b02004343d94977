"""Builds the engine library libperft_b200.so in-tree with nvcc (sm_100a).

Usage: python -m perft_gpu_b200.build [--verbose]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libperft_b200.so")
PROBE_LIB = os.path.join(HERE, "libperft_probe.so")
CLI = os.path.join(HERE, "perft_gpu")

SOURCES = ["engine.cu", "tables.cpp", "host.cpp"]
HEADERS = ["movegen.cuh", "serve.cuh", os.path.join("..", "..", "include", "perft_b200.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "-shared",
]


def nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def up_to_date(lib, sources):
    if not os.path.exists(lib):
        return False
    t = os.path.getmtime(lib)
    deps = [os.path.join(CSRC, s) for s in sources] + [__file__]
    return all(os.path.getmtime(d) <= t for d in deps)


def _nvcc(lib, sources, verbose, defines=()):
    cmd = [nvcc()] + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose else []) + [f"-D{d}" for d in defines] + [
        "-I", os.path.join(ROOT, "include"),
        "-o", lib,
    ] + [os.path.join(CSRC, s) for s in sources] + ["-lcudart"]
    subprocess.run(cmd, check=True)


def build_variant(out, defines, verbose=False):
    """Compiles the engine with extra -D definitions into `out` (tuning builds)."""
    _nvcc(out, SOURCES, verbose, defines)
    return out


def _cli():
    """The perft_gpu command-line program, linked against the engine library."""
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", CLI, os.path.join(CSRC, "cli.cpp"),
                    "-L", HERE, "-lperft_b200", "-Wl,-rpath,$ORIGIN"], check=True)


def build(verbose=False, force=False):
    """Compiles the engine and the integer-peak probe libraries (sm_100a) and
    the perft_gpu program."""
    if force or not up_to_date(LIB, SOURCES + HEADERS):
        _nvcc(LIB, SOURCES, verbose)
    if force or not up_to_date(PROBE_LIB, ["int_peak.cu"]):
        _nvcc(PROBE_LIB, ["int_peak.cu"], verbose)
    if force or not up_to_date(CLI, ["cli.cpp", os.path.join("..", "..", "include", "perft_b200.h")]) \
            or os.path.getmtime(CLI) < os.path.getmtime(LIB):
        _cli()
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force=True)
    print(LIB)
