"""Builds libmpf.so in-tree for sm_100a (nvcc) and the CPU oracle (make).

Usage: python -m mapol_b200.build [--verbose]
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmpf.so")

SOURCES = ["engine.cu", "symbolic.cpp", "synth.cpp"]
HEADERS = ["internal.h", "kernels.cuh"]

NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-Xcompiler", "-fPIC,-O3",
    "-shared",
]


def nvcc_path():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_lib(force=False, verbose=False):
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "mpf.h")]
    if not force and not _stale(LIB, deps):
        return LIB
    cmd = [nvcc_path()] + NVCC_FLAGS + [
        "-I" + os.path.join(ROOT, "include"),
        "-I" + CSRC,
        *[os.path.join(CSRC, s) for s in SOURCES],
        "-o", LIB + ".tmp",
    ]
    if verbose:
        print(" ".join(cmd))
    env = dict(os.environ)
    env.pop("CXX", None)
    env.pop("CC", None)
    subprocess.run(cmd, check=True, env=env)
    os.replace(LIB + ".tmp", LIB)
    return LIB


def build_oracle(verbose=False):
    env = dict(os.environ)
    env.pop("CXX", None)
    env.pop("CC", None)
    out = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], env=env,
                         capture_output=not verbose, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + (out.stderr or ""))


def build(force=False, verbose=False):
    build_lib(force=force, verbose=verbose)
    build_oracle(verbose=verbose)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv)
