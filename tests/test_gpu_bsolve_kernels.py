"""Every backward-substitution kernel gives the same voltages.

The autotuner picks one backward-solve kernel per elimination level by timing, so a
run may use any of them.  MPF_BSOLVE_LANES forces one kernel on every level: the
one-case-per-thread kernel (0), k_mf_bsolve_chunk<G> (G) or k_mf_bsolve_staged<G>
(-G).  Each must converge to the oracle's voltages (1e-8 p.u., as the parity tests)
with the oracle's iteration counts, and the staged kernel, which sums in another
order, must agree with the chunk kernel to round-off.  MPF_BSOLVE_TOP forces the
near-root levels into one k_mf_bsolve_top launch, which does the chunk kernel's
arithmetic: with the other levels on the chunk kernel of the same lane count, the
results must be the same bit for bit.
"""
import os

import numpy as np
import pytest

import mapol_b200 as m
from oracle import oracle

pytestmark = pytest.mark.gpu


def _solve(buses, branches, cases, prec, lanes, top=None):
    os.environ["MPF_BSOLVE_LANES"] = str(lanes)
    if top:
        os.environ["MPF_BSOLVE_TOP"] = str(top)
    try:
        with m.PowerFlow(buses, branches) as pf:
            pf.set_cases(cases)
            pf.solve(m.NR, prec)
            return pf.results()
    finally:
        del os.environ["MPF_BSOLVE_LANES"]
        os.environ.pop("MPF_BSOLVE_TOP", None)


@pytest.mark.parametrize("prec", [m.MIXED, m.FP64])
def test_staged_matches_chunk(gpu, prec):
    buses, branches, cases = m.workload("cfg2_1354bus")
    cases = cases[:64]
    for g in (8, 4, 2, 1):
        a = _solve(buses, branches, cases, prec, g)
        b = _solve(buses, branches, cases, prec, -g)
        assert np.array_equal(a.status, b.status)
        assert np.array_equal(a.iterations, b.iterations)
        conv = a.status == m.runpf.CONVERGED
        assert conv.all()
        # both converged to max |F| < 1e-8: plain FP64 agrees to round-off; mixed
        # precision (inexact Newton steps from an FP32 LU) to the parity tolerance
        tol = 1e-10 if prec == m.FP64 else 1e-8
        assert np.abs(a.v - b.v).max() < tol, g


def test_forced_kernels_match_oracle(gpu):
    buses, branches, cases = m.workload("cfg1_300bus")
    cases = cases[:40]
    ref = oracle.runpf(buses, branches, cases, alg=m.NR)
    for lanes in (0, 16, 8, 4, 2, 1, -8, -4, -2, -1):
        res = _solve(buses, branches, cases, m.FP64, lanes)
        conv = res.status == m.runpf.CONVERGED
        assert np.array_equal(conv, ref["converged"])
        assert np.array_equal(res.iterations[conv], ref["iterations"][conv]), lanes
        assert np.abs(res.v[conv] - ref["v"][conv]).max() < 1e-8, lanes


@pytest.mark.parametrize("prec", [m.MIXED, m.FP64])
def test_fused_near_root_levels_equal_chunk_kernel(gpu, prec):
    buses, branches, cases = m.workload("cfg3_9241bus")
    cases = cases[:96]
    ref = oracle.runpf(buses, branches, cases[:16], alg=m.NR)
    for g in (8, 4, 2, 1):
        a = _solve(buses, branches, cases, prec, g)
        b = _solve(buses, branches, cases, prec, g, top=g)
        assert np.array_equal(a.status, b.status) and np.array_equal(a.iterations, b.iterations)
        assert np.array_equal(a.v, b.v), g
        conv = b.status[:16] == m.runpf.CONVERGED
        assert np.array_equal(conv, ref["converged"])
        if prec == m.FP64:  # (mixed precision: the parity tests' rules, bitwise equality here)
            assert np.abs(b.v[:16][conv] - ref["v"][conv]).max() < 1e-8
