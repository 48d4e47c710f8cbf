"""The CUDA path against outputs of the reference's OWN CPU code (not the oracle):
tests/golden/reference_outputs.npz holds what the reference's mkl_runpf computed
(oracle/_ref/librefpf.so, built from its sources; tests/golden/make_reference_fixtures.py)
on its bundled MATPOWER cases with N-1 outages and on the synthetic 30/300-bus
workloads, for Newton-Raphson and fast-decoupled XB / BX.

Plain FP64: identical converged flags and iteration counts, |V - V_ref| < 1e-8 p.u.
Mixed precision: identical flags, at most one more iteration, the same voltage bar (a
case that took the extra iteration against the oracle run to 1e-11: it stopped
further past the criterion than the reference did).  The reference takes voltage
angles as atan(y/x) (util/complexUtils.h:21-23); the engine's angle_mode 1 reproduces
that, including the 300-bus workload where it makes every reference case fail.
"""
import os

import numpy as np
import pytest

import mapol_b200 as m
from oracle import oracle

from .parity import TIGHT_TOL, compare

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ALGS = {"nr": m.NR, "fdxb": m.FDXB, "fdbx": m.FDBX}


def _fixture():
    return np.load(os.path.join(HERE, "golden", "reference_outputs.npz"))


def _ref(g, name, tag):
    return dict(v=g[f"{name}_{tag}_v"], iterations=g[f"{name}_{tag}_iterations"],
                converged=g[f"{name}_{tag}_converged"])


def _grid(g, name):
    cases = [[int(o)] if o >= 0 else [] for o in g[f"{name}_outage"]]
    return g[f"{name}_buses"], g[f"{name}_branches"], cases


@pytest.mark.parametrize("tag", ["nr", "fdxb", "fdbx"])
@pytest.mark.parametrize("name", ["case14", "case30", "case118", "case300", "cfg0_30bus"])
def test_engine_matches_reference_outputs(gpu, name, tag):
    g = _fixture()
    buses, branches, cases = _grid(g, name)
    ref = _ref(g, name, tag)
    alg = ALGS[tag]
    precisions = (m.FP64, m.MIXED) if alg == m.NR else (m.FP64,)
    for angle_mode in (0, 1):
        with m.PowerFlow(buses, branches, angle_mode=angle_mode) as pf:
            pf.set_cases(cases)
            for prec in precisions:
                pf.solve(alg, prec)
                res = pf.results()

                def tight(idx):
                    return oracle.runpf(buses, branches, [cases[i] for i in idx], alg=alg, tol=TIGHT_TOL)

                conv = compare(res, ref, max_extra_iter=0 if prec == m.FP64 else 1, v_tol=1e-8, tight=tight)
                assert conv.any()


def test_reference_angle_quirk_reproduced(gpu):
    """300-bus workload: the reference's own Newton fails every case (atan(y/x) loses
    the quadrant as iterates pass 90 degrees); the engine with angle_mode 1 fails the
    same cases after the same number of iterations, and with atan2 solves them all."""
    g = _fixture()
    buses, branches, cases = _grid(g, "cfg1_300bus")
    ref = _ref(g, "cfg1_300bus", "nr")
    assert not ref["converged"].any()
    with m.PowerFlow(buses, branches, angle_mode=1) as pf:
        pf.set_cases(cases)
        pf.solve(m.NR, m.FP64)
        res = pf.results()
    assert np.array_equal(res.status == m.runpf.CONVERGED, ref["converged"])
    assert np.array_equal(res.iterations, ref["iterations"])
    with m.PowerFlow(buses, branches) as pf:
        pf.set_cases(cases)
        pf.solve(m.NR, m.FP64)
        assert (pf.results().status == m.runpf.CONVERGED).all()
