"""Reactive limits of PV buses (mpf_set_q_limits): PV -> PQ switching in rounds, against
the oracle's restatement (oracle.runpf_qlim, MATPOWER's runpf with ENFORCE_Q_LIMS = 1).
Bar: identical converged flags and identical switched buses per case, |dV| < 1e-8 on
converged cases.  Iteration counts are not compared: the engine continues each round
from the case's voltages, the oracle restarts from the start point."""
import os

import numpy as np
import pytest

import mapol_b200 as m
from oracle import oracle

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _compare(res, types, ref, buses):
    conv = res.status == m.runpf.CONVERGED
    assert np.array_equal(conv, ref["converged"]), np.where(conv != ref["converged"])
    sw = (types == 1) & (buses["type"] == 2)[None, :]
    assert np.array_equal(sw[conv], ref["switched"][conv]), np.where(sw != ref["switched"])
    assert (res.max_mis[conv] < 1e-8).all()
    assert np.abs(res.v[conv] - ref["v"][conv]).max() < 1e-8


def _q_at(buses, branches, v, outages=()):
    ptr, col, val = oracle.ybus(buses, branches, outages)
    ib = np.array([np.dot(val[ptr[i]:ptr[i + 1]], v[col[ptr[i]:ptr[i + 1]]]) for i in range(len(buses))])
    return (v * np.conj(ib)).imag


@pytest.mark.parametrize("name", ["case118", "case300"])
def test_real_grid_generator_limits_match_oracle(gpu, name):
    g = np.load(os.path.join(HERE, "golden", "matpower_cases.npz"))
    buses, branches = g[name + "_buses"], g[name + "_branches"]
    qmin, qmax = g[name + "_qmin"], g[name + "_qmax"]
    cases = m.n1_cases(branches, len(buses), 24, 5, with_base=True)
    ref = oracle.runpf_qlim(buses, branches, cases, qmin, qmax)
    assert ref["switched"].any()
    with m.PowerFlow(buses, branches) as pf:
        pf.set_q_limits(qmin, qmax)
        pf.set_cases(cases)
        for prec in (m.FP64, m.MIXED):
            pf.solve(m.NR, prec)
            _compare(pf.results(), pf.bus_types(), ref, buses)


def test_tight_limits_switch_in_several_rounds(gpu):
    """Synthetic 300-bus grid with limits just inside the base case's reactive output of
    a third of its PV buses: many cases switch, some in more than one round."""
    buses, branches, cases = m.workload("cfg1_300bus")
    cases = [[]] + cases[:60]
    base = oracle.runpf(buses, branches, [[]])
    q = _q_at(buses, branches, base["v"][0])
    pv = np.where(buses["type"] == 2)[0]
    rng = np.random.default_rng(3)
    pick = rng.choice(pv, len(pv) // 3, replace=False)
    qmin = np.full(len(buses), -np.inf)
    qmax = np.full(len(buses), np.inf)
    qmax[pick] = q[pick] - 0.01
    qmin[pick] = q[pick] - 2.0
    ref = oracle.runpf_qlim(buses, branches, cases, qmin, qmax)
    assert ref["switched"].sum() >= len(cases) and (ref["rounds"] >= 2).any()
    with m.PowerFlow(buses, branches) as pf:
        pf.set_q_limits(qmin, qmax)
        pf.set_cases(cases)
        for prec in (m.FP64, m.MIXED):
            pf.solve(m.NR, prec)
            res = pf.results()
            types = pf.bus_types()
            _compare(res, types, ref, buses)
            # a switched bus holds its limit
            c = int(np.argmax(ref["switched"].sum(1)))
            k = np.where(ref["switched"][c])[0]
            bb = buses.copy()
            bb["type"][k] = 1
            bb["q"][k] = qmax[k]
            assert np.abs(_q_at(bb, branches, res.v[c], cases[c])[k] - qmax[k]).max() < 1e-7


def test_limits_that_never_bind_change_nothing(gpu):
    """Wide limits: the superset system (a Vm variable per limited PV bus, inactive)
    gives the same voltages and iteration counts as no limits."""
    buses, branches, cases = m.workload("cfg1_300bus")
    cases = cases[:50]
    nb = len(buses)
    with m.PowerFlow(buses, branches) as pf:
        pf.set_cases(cases)
        pf.solve(m.NR, m.FP64)
        a = pf.results()
        pf.set_q_limits(np.full(nb, -50.0), np.full(nb, 50.0))
        pf.set_cases(cases)
        pf.solve(m.NR, m.FP64)
        b = pf.results()
        assert (pf.bus_types() == buses["type"][None, :]).all()
        pf.set_q_limits(None, None)
        pf.set_cases(cases)
        pf.solve(m.NR, m.FP64)
        c = pf.results()
    assert np.array_equal(a.status, b.status) and np.array_equal(a.iterations, b.iterations)
    conv = a.converged
    assert np.abs(a.v[conv] - b.v[conv]).max() < 1e-12
    assert np.array_equal(a.v, c.v)


def test_limit_inputs_are_checked(gpu):
    buses, branches, cases = m.workload("cfg0_30bus")
    nb = len(buses)
    with m.PowerFlow(buses, branches) as pf:
        with pytest.raises(m.MpfError):
            pf.set_q_limits(np.zeros(nb), np.full(nb, -1.0))  # qmin > qmax
        pf.set_q_limits(np.full(nb, -5.0), np.full(nb, 5.0))
        with pytest.raises(m.MpfError):
            pf.solve(m.NR, m.FP64)  # the batch must be set again
        pf.set_cases(cases)
        with pytest.raises(m.MpfError):
            pf.solve(m.FDXB, m.FP64)  # Newton-Raphson only
        pf.solve(m.NR, m.FP64)
        assert pf.results().converged.all()
