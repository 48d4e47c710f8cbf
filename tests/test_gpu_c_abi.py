"""A plain C program drives the engine through include/mpf.h (no ctypes, no Python
in the call path): tests/native/c_abi_smoke.c is compiled with gcc, linked against
mapol_b200/libmpf.so, run, and its results (30-bus grid, base case + 10 N-1 outages,
NR in FP64 and mixed precision) are checked against the CPU oracle."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import mapol_b200 as m
from mapol_b200 import _types as T
from oracle import oracle

from .parity import compare

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NB, NBR, NC, NOUT = 30, 41, 11, 10


def test_c_program_solves_through_the_c_abi(gpu, tmp_path):
    if not shutil.which("gcc"):
        pytest.skip("gcc not available")
    libdir = os.path.join(ROOT, "mapol_b200")
    exe = tmp_path / "c_abi_smoke"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "native", "c_abi_smoke.c"), "-L", libdir, "-lmpf",
                    "-Wl,-rpath," + libdir, "-o", str(exe)], check=True)
    out = tmp_path / "results.bin"
    r = subprocess.run([str(exe), str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    raw = out.read_bytes()
    o = 0

    def take(dtype, count):
        nonlocal o
        a = np.frombuffer(raw, dtype=dtype, count=count, offset=o)
        o += a.nbytes
        return a

    buses = take(T.BUS_DTYPE, NB)
    branches = take(T.BRANCH_DTYPE, NBR)
    offs = take(np.int32, NC + 1)
    flat = take(np.int32, NOUT)
    cases = [flat[offs[c]:offs[c + 1]].tolist() for c in range(NC)]
    # the C caller built the same workload the Python side names cfg0_30bus
    b0, br0, c0 = m.workload("cfg0_30bus")
    assert buses.tobytes() == b0.tobytes() and branches.tobytes() == br0.tobytes() and cases == c0
    ref = oracle.runpf(buses, branches, cases, alg=m.NR)
    for prec in (m.FP64, m.MIXED):
        st = take(np.uint8, NC)
        it = take(np.int32, NC)
        mis = take(np.float64, NC)
        v = take(np.float64, NC * NB * 2).reshape(NC, NB, 2)
        res = m.Results(v[..., 0] + 1j * v[..., 1], it.copy(), st.copy(), mis.copy())
        conv = compare(res, ref, max_extra_iter=0 if prec == m.FP64 else 1)
        assert conv.all()
    assert o == len(raw)
