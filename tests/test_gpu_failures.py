"""Per-case failure statuses, injected from the host through the public API (no GPU
fault): each failing case must retire with its documented status while the cases in
the same 32-lane group carry on and finish exactly as they would without it.

  MAX_ITER  iteration limit reached (options.max_it_nr = 1), as the reference's loop
            stops at MAX_IT_NR (newtonpf.h:398)
  DIVERGED  non-finite mismatch: an AVR set-point of 1e200 p.u. makes S = V conj(Y V)
            overflow at the start point
  SINGULAR  outages that cut buses off from the slack (a bridge, or two branches that
            isolate a bus): mpf_set_cases finds them, the case is not iterated
The reference has no per-case status: a non-converged case just gets fitness
DBL_MAX (runpf.h:782-789) and its zero pivots are ignored (newtonpf.h:952-956).
"""
import numpy as np
import pytest

import mapol_b200 as m
from mapol_b200 import _types as T
from oracle import oracle

pytestmark = pytest.mark.gpu


def test_iteration_limit_gives_max_iter(gpu):
    buses, branches, cases = m.workload("cfg1_300bus")
    cases = cases[:64]
    ref = oracle.runpf(buses, branches, cases, alg=m.NR, max_it=1)
    assert not ref["converged"].any()
    for prec in (m.FP64, m.MIXED):
        with m.PowerFlow(buses, branches, max_it_nr=1) as pf:
            pf.set_cases(cases)
            pf.solve(m.NR, prec)
            res = pf.results()
        assert (res.status == T.CASE_MAX_ITER).all()
        assert (res.iterations == 1).all()
        dv = np.abs(res.v - ref["v"]).max()
        # one step from the flat start; the mixed form solves it with FP32 factors
        # (measured 1.8e-4 on a step of order 0.1)
        assert dv < (1e-10 if prec == m.FP64 else 1e-3), dv


@pytest.mark.parametrize("alg", [m.NR, m.FDXB])
def test_overflowing_case_diverges_alone(gpu, alg):
    buses, branches, cases = m.workload("cfg1_300bus")
    cases = cases[:64]
    pv = int(np.where(buses["type"] == 2)[0][0])
    controls = [(m.CTRL_AVR, pv)]
    good = np.full((64, 1), buses["vm"][pv])
    bad = good.copy()
    bad[5, 0] = 1e200
    out = []
    for vals in (good, bad):
        with m.PowerFlow(buses, branches) as pf:
            pf.set_cases(cases)
            pf.set_controls(controls, vals)
            pf.solve(alg, m.FP64)
            out.append(pf.results())
    a, b = out
    assert b.status[5] == T.CASE_DIVERGED and b.iterations[5] == 0
    keep = np.arange(64) != 5
    assert (a.status == T.CASE_CONVERGED).all()
    assert np.array_equal(a.status[keep], b.status[keep])
    assert np.array_equal(a.iterations[keep], b.iterations[keep])
    assert np.array_equal(a.v[keep], b.v[keep])  # bit for bit: lanes are independent


def _islanding_cases(buses, branches):
    """Single bridge outages, and pairs of non-bridge branches that isolate a bus of
    degree two."""
    nb = len(buses)
    bridges = np.where(m.find_bridges(branches, nb))[0]
    single = [[int(k)] for k in bridges[:6]]
    inc = [[] for _ in range(nb)]
    for k, (f, t) in enumerate(zip(branches["from"], branches["to"])):
        inc[f].append(k)
        inc[t].append(k)
    isb = m.find_bridges(branches, nb)
    pairs = [inc[i] for i in range(nb) if len(inc[i]) == 2 and not isb[inc[i]].any() and buses["type"][i] != 3]
    return single, [list(map(int, p)) for p in pairs[:4]]


@pytest.mark.parametrize("alg", [m.NR, m.FDXB])
def test_islanding_outages_are_singular(gpu, alg):
    buses, branches = m.synth_grid(300, 411, 69, 0.1, seed=1)
    single, pairs = _islanding_cases(buses, branches)
    assert single and pairs
    normal = m.n1_cases(branches, 300, 20, 5)
    cases = single + normal[:10] + pairs + normal[10:]
    cut = np.array([1] * len(single) + [0] * 10 + [1] * len(pairs) + [0] * 10, bool)
    ref = oracle.runpf(buses, branches, cases, alg=alg)
    assert not ref["converged"][cut].any()
    for prec in (m.FP64, m.MIXED):
        with m.PowerFlow(buses, branches) as pf:
            pf.set_cases(cases)
            pf.solve(alg, prec)
            res = pf.results()
        assert (res.status[cut] == T.CASE_SINGULAR).all(), res.status
        assert (res.iterations[cut] == 0).all()
        v0 = buses["vm"] * np.exp(1j * buses["va"])  # the start point (runpf.h:211-226)
        assert np.abs(res.v[cut] - v0[None]).max() < 1e-14
        assert (res.status[~cut] == T.CASE_CONVERGED).all()
        if prec == m.FP64:
            assert np.abs(res.v[~cut] - ref["v"][~cut]).max() < 1e-8
    # the same islanding cases, each alone in a batch, give the same answer
    with m.PowerFlow(buses, branches) as pf:
        pf.set_cases(pairs[:1])
        pf.solve(alg, m.FP64)
        assert pf.results().status[0] == T.CASE_SINGULAR
