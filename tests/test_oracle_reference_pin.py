"""Pins the oracle to the reference's own CPU power-flow code.

oracle/_ref/librefpf.so is the reference's src/powerflow/runpf.h (mkl_init / mkl_runpf
with makeYbus.h, newtonpf.h, makeB.h, fdpf.h) compiled unmodified from its sources by
oracle/Makefile, with in-project stand-ins for the MKL routines it calls
(oracle/refshim/mkl.h).  The oracle must reproduce it: the same Ybus, and for
Newton-Raphson (the reference's Eigen SparseLU option) and fast-decoupled XB / BX (its
DSS path) the same converged flags, the same iteration counts and the same voltages to
rounding, on the reference's own bundled MATPOWER cases with N-1 outages and on the
synthetic workloads.  Skipped where the reference tree was not available to build it.
"""
import os

import numpy as np
import pytest

import mapol_b200 as m
from oracle import oracle, refpf

pytestmark = pytest.mark.skipif(not refpf.available(), reason="oracle/_ref/librefpf.so not built (no reference tree)")

HERE = os.path.dirname(os.path.abspath(__file__))
V_TOL = 1e-11  # measured: <= 1.5e-13 (case300), <= 1.2e-14 below


def _mp(name):
    g = np.load(os.path.join(HERE, "golden", "matpower_cases.npz"))
    return g[name + "_buses"], g[name + "_branches"]


def _n1(buses, branches, k=20, seed=3):
    nnb = int((~m.find_bridges(branches, len(buses))).sum())
    return m.n1_cases(branches, len(buses), min(k, nnb), seed, with_base=True)


def _check(r, o, v_tol=V_TOL):
    assert np.array_equal(r["converged"], o["converged"]), (r["converged"], o["converged"])
    assert np.array_equal(r["iterations"], o["iterations"]), (r["iterations"], o["iterations"])
    both = r["converged"] & o["converged"]
    assert both.any()
    assert np.abs(r["v"][both] - o["v"][both]).max() < v_tol


@pytest.mark.parametrize("name", ["case14", "case30", "case118"])
def test_ybus_matches_reference(built, name):
    buses, branches = _mp(name)
    for outages in ([], [3], [1, 7]):
        Y, nnz = refpf.ybus(buses, branches, outages)
        p, c, val = oracle.ybus(buses, branches, outages)
        O = np.zeros_like(Y)
        for i in range(len(buses)):
            O[i, c[p[i]:p[i + 1]]] += val[p[i]:p[i + 1]]
        assert nnz == len(c)  # same superset pattern (an outaged branch keeps its entries)
        assert np.abs(Y - O).max() <= 1e-13 * np.abs(Y).max()


@pytest.mark.parametrize("alg", [m.NR, m.FDXB, m.FDBX])
@pytest.mark.parametrize("name", ["case14", "case30", "case118", "case300"])
def test_bundled_cases_n1_match_reference(built, name, alg):
    buses, branches = _mp(name)
    cases = _n1(buses, branches)
    solver = refpf.SOLVER_EIGEN if alg == m.NR else refpf.SOLVER_DSS
    r = refpf.runpf(buses, branches, cases, alg=alg, solver=solver)
    for angle_mode in (1, 0):  # 1: the reference's atan(y/x); 0: atan2 (equal below 90 degrees)
        _check(r, oracle.runpf(buses, branches, cases, alg=alg, angle_mode=angle_mode))


@pytest.mark.parametrize("alg", [m.NR, m.FDXB, m.FDBX])
def test_synthetic_30_bus_matches_reference(built, alg):
    buses, branches, cases = m.workload("cfg0_30bus")
    solver = refpf.SOLVER_EIGEN if alg == m.NR else refpf.SOLVER_DSS
    _check(refpf.runpf(buses, branches, cases, alg=alg, solver=solver), oracle.runpf(buses, branches, cases, alg=alg))


def test_load_scenarios_match_reference(built):
    buses, branches = _mp("case118")
    cases = _n1(buses, branches, 8)
    sbus = m.load_scenarios(buses, len(cases), 0.05, 5)
    _check(refpf.runpf(buses, branches, cases, sbus=sbus), oracle.runpf(buses, branches, cases, sbus=sbus))


def test_angle_quirk_reproduced_on_300_bus_workload(built):
    """The reference computes voltage angles as atan(y/x) (cuCangle,
    util/complexUtils.h:21-23), which loses the quadrant beyond 90 degrees; on the
    300-bus synthetic workload its Newton iterates pass there and none of its cases
    converge.  The oracle's angle_mode 1 reproduces exactly that (flags and iteration
    counts); with atan2 (the default, angle_mode 0) every case converges."""
    buses, branches, cases = m.workload("cfg1_300bus")
    cases = cases[:6]
    r = refpf.runpf(buses, branches, cases)
    o1 = oracle.runpf(buses, branches, cases, angle_mode=1)
    assert not r["converged"].any()
    assert np.array_equal(r["converged"], o1["converged"])
    assert np.array_equal(r["iterations"], o1["iterations"])
    assert oracle.runpf(buses, branches, cases)["converged"].all()


def test_stepper_reproduces_runpf_bitwise(built):
    """bench.py's reference arm steps the reference's Newton one iteration at a time;
    the sequence must be mkl_runpf's own, bit for bit."""
    buses, branches = _mp("case118")
    cases = _n1(buses, branches, 6)
    r = refpf.runpf(buses, branches, cases)
    st = refpf.Stepper(buses, branches)
    try:
        vv = np.zeros((len(buses), 2))
        for c, outages in enumerate(cases):
            res = None
            while res is None:
                res = st.step(outages, vv)
            assert res == (bool(r["converged"][c]), int(r["iterations"][c]))
            assert np.array_equal(vv[:, 0] + 1j * vv[:, 1], r["v"][c])
    finally:
        st.close()
