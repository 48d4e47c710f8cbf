"""Per-case control overrides (mpf_set_controls) and the optimiser shim
(mapol_b200.pso) on the GPU, against the oracle run on each case's own grid: the
base grid with that case's AVR set-points written into bus.vm, taps into
branch.tap and shunt susceptances into bus.bsh, which is what the reference's
hybrid_computeVoltage / hybrid_computeYfYt do with a particle (runpf.h:524-541,
makeYbus.h:313-332).  Same bar as the outage parity tests: identical flags, at
most one extra iteration for mixed precision, |dV| < 1e-8 on converged cases (a case
that took the extra iteration against the oracle run to the tighter tolerance, see
tests/parity.py)."""
import os

import numpy as np
import pytest

import mapol_b200 as m
from mapol_b200 import pso
from oracle import oracle

from .parity import TIGHT_TOL, compare

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
V_TOL = 1e-8


def _grid(name):
    g = np.load(os.path.join(HERE, "golden", "matpower_cases.npz"))
    return g[name + "_buses"], g[name + "_branches"]


def _apply(buses, branches, controls, vals):
    b, br = buses.copy(), branches.copy()
    for (kind, idx), v in zip(controls, vals):
        if kind == m.CTRL_AVR:
            b["vm"][idx] = v
        elif kind == m.CTRL_SHC:
            b["bsh"][idx] = v
        else:
            br["tap"][idx] = v
    return b, br


def _oracle(buses, branches, cases, controls, values, alg, tol=1e-8):
    outs = [oracle.runpf(*_apply(buses, branches, controls, values[c]), [cases[c]], alg=alg, tol=tol)
            for c in range(len(cases))]
    return {k: np.concatenate([o[k] for o in outs]) for k in outs[0]}


def _compare(res, ref, max_extra_iter=0, tight=None):
    return compare(res, ref, max_extra_iter, V_TOL, tight)


def _particles(est, n, seed):
    """Particle 0 at the defaults, the rest uniform in each structure's range."""
    rng = np.random.default_rng(seed)
    lo = np.array([e.min for e in est])
    hi = np.array([e.max for e in est])
    X = lo + (hi - lo) * rng.random((n, len(est)))
    X[0] = [e.default for e in est]
    return X


def _controls(buses, branches, n, seed):
    est, bie, rie = pso.estruturas(buses, branches)
    controls, cols = pso.bind(est, bie, rie, branches)
    return est, bie, rie, controls, _particles(est, n, seed)[:, cols]


@pytest.mark.parametrize("name", ["case118", "case300"])
@pytest.mark.parametrize("alg", [m.NR, m.FDXB, m.FDBX])
def test_controls_match_oracle_on_each_case_grid(gpu, name, alg):
    buses, branches = _grid(name)
    *_, controls, vals = _controls(buses, branches, 40, 5)
    kinds = {k for k, _ in controls}
    assert kinds == {m.CTRL_AVR, m.CTRL_OLTC, m.CTRL_SHC}
    cases = [[] for _ in range(len(vals))]
    ref = _oracle(buses, branches, cases, controls, vals, alg)
    assert ref["converged"].sum() >= 20
    with m.PowerFlow(buses, branches) as pf:
        pf.set_cases(cases)
        pf.set_controls(controls, vals)
        for prec in (m.FP64, m.MIXED):
            pf.solve(alg, prec)
            tight = lambda idx: _oracle(buses, branches, [cases[i] for i in idx], controls, vals[idx], alg,
                                        TIGHT_TOL)
            _compare(pf.results(), ref, 0 if prec == m.FP64 else 1, tight)


def test_controls_at_base_values_change_nothing(gpu):
    buses, branches = _grid("case300")
    est, bie, rie, controls, vals = _controls(buses, branches, 1, 0)
    cases = [[]] + [[int(b)] for b in m.select_outages(branches, len(buses), 20, 1)]
    base = np.repeat(vals[:1], len(cases), 0)
    with m.PowerFlow(buses, branches) as pf:
        pf.set_cases(cases)
        pf.solve(m.NR, m.FP64)
        a = pf.results()
        pf.set_controls(controls, base)
        pf.solve(m.NR, m.FP64)
        b = pf.results()
        pf.set_controls([], None)
        pf.solve(m.NR, m.FP64)
        c = pf.results()
    assert np.array_equal(a.status, b.status) and np.array_equal(a.iterations, b.iterations)
    conv = a.converged
    assert conv.sum() >= 15
    assert np.abs(a.v[conv] - b.v[conv]).max() < 1e-11
    assert np.array_equal(a.v, c.v)


def test_controls_combine_with_outages_and_injections(gpu):
    """N-1 cases with controls and per-case loads; an outaged controlled tap has no
    effect (the oracle removes the modified branch)."""
    buses, branches = _grid("case118")
    *_, controls, vals = _controls(buses, branches, 24, 7)
    bridge = m.find_bridges(branches, len(buses)).astype(bool)
    taps = [idx for kind, idx in controls if kind == m.CTRL_OLTC and not bridge[idx]]
    assert taps
    outs = [int(b) for b in m.select_outages(branches, len(buses), 30, 2)]
    cases = [[taps[(c // 3) % len(taps)]] if c % 3 == 0 else [outs[c]] if c % 3 == 1 else [] for c in range(24)]
    sbus = m.load_scenarios(buses, 24, 0.03, 11)
    refs = []
    for c in range(24):
        b, br = _apply(buses, branches, controls, vals[c])
        refs.append(oracle.runpf(b, br, [cases[c]], alg=m.NR, sbus=sbus[c:c + 1]))
    ref = {k: np.concatenate([o[k] for o in refs]) for k in refs[0]}
    with m.PowerFlow(buses, branches) as pf:
        pf.set_cases(cases, sbus=sbus)
        pf.set_controls(controls, vals)
        pf.solve(m.NR, m.FP64)
        _compare(pf.results(), ref)


def test_pso_shim_fitness_is_oracle_loss_or_dbl_max(gpu):
    buses, branches = _grid("case118")
    est, bie, rie = pso.estruturas(buses, branches)
    X = _particles(est, 32, 3)
    enxame = [pso.Particula(x) for x in X]
    eng = pso.hybrid_init(buses, branches, len(enxame), 1, est, m.NR, bie, rie)
    try:
        fit = pso.hybrid_runpf(eng, est, enxame)
    finally:
        pso.hybrid_free(eng)
    controls, cols = pso.bind(est, bie, rie, branches)
    for c, p in enumerate(enxame):
        b, br = _apply(buses, branches, controls, X[c, cols])
        r = oracle.runpf(b, br, [[]], alg=m.NR)
        assert p.fitness == fit[c]
        if r["converged"][0]:
            assert abs(p.fitness - oracle.loss(b, br, r["v"][0])) < 1e-9
        else:
            assert p.fitness == pso.DBL_MAX
    assert (fit < pso.DBL_MAX).sum() >= 16


def test_flows_and_adjoint_use_the_case_taps(gpu):
    """Branch-admittance gradients of a controlled tap branch at a non-default tap
    against central differences (step 1e-4 |y|) of the overload loss."""
    buses, branches = _grid("case118")
    est, bie, rie, controls, vals = _controls(buses, branches, 6, 9)
    cases = [[] for _ in range(len(vals))]
    tol = 1e-12

    def run(br, rating=None):
        with m.PowerFlow(buses, br, tol=tol) as pf:
            pf.set_cases(cases)
            pf.set_controls(controls, vals)
            pf.solve(m.NR, m.FP64)
            res = pf.results()
            assert res.converged.all()
            if rating is None:
                return res, pf.branch_flows(flows=True)
            pf.set_ratings(rating)
            return pf.branch_flows()["overload"], pf.adjoint(m.FP64)

    res, fl = run(branches)
    for c in range(len(cases)):
        b, br = _apply(buses, branches, controls, vals[c])
        assert abs(fl["ploss"][c] - oracle.loss(b, br, res.v[c])) < 1e-10
    rating = 0.95 * np.abs(fl["sf"]).max(0)
    L, g = run(branches, rating)
    assert (L > 0).all()
    taps = [idx for kind, idx in controls if kind == m.CTRL_OLTC]
    sf = np.abs(fl["sf"])
    ks = sorted(taps, key=lambda k: -sf[:, k].max())[:2]
    adjs, fds = [], []
    for k in ks:
        ys = 1.0 / (branches["r"][k] + 1j * branches["x"][k])
        hk = 1e-4 * abs(ys)
        for comp, d in ((0, hk), (1, 1j * hk)):
            Ls = []
            for sgn in (1, -1):
                br = branches.copy()
                z = 1.0 / (ys + sgn * d)
                br["r"][k], br["x"][k] = z.real, z.imag
                Ls.append(run(br, rating)[0])
            fds.append((Ls[0] - Ls[1]) / (2 * hk))
            adjs.append((g["grad_g"] if comp == 0 else g["grad_b"])[:, k])
    adj, fd = np.concatenate(adjs), np.concatenate(fds)
    assert np.abs(fd).max() > 0
    assert np.linalg.norm(adj - fd) <= 1e-5 * np.linalg.norm(fd), (adj, fd)


def test_bad_controls_raise(gpu):
    buses, branches = _grid("case118")
    pq = int(np.where(buses["type"] == 1)[0][0])
    pv = int(np.where(buses["type"] == 2)[0][0])
    untapped = int(np.where(branches["tap"] == 0)[0][0])
    tapped = int(np.where(branches["tap"] != 0)[0][0])
    with m.PowerFlow(buses, branches) as pf:
        with pytest.raises(m.MpfError):
            pf.set_controls([(m.CTRL_AVR, pv)], np.ones((0, 1)))  # before set_cases
        pf.set_cases([[], []])
        bad = [
            ([(m.CTRL_AVR, pq)], [[1.0], [1.0]]),
            ([(m.CTRL_OLTC, untapped)], [[1.0], [1.0]]),
            ([(m.CTRL_OLTC, tapped)], [[0.0], [1.0]]),
            ([(m.CTRL_AVR, pv), (m.CTRL_AVR, pv)], [[1.0, 1.0], [1.0, 1.0]]),
            ([(m.CTRL_SHC, len(buses))], [[0.1], [0.1]]),
            ([(7, 0)], [[1.0], [1.0]]),
            ([(m.CTRL_SHC, 3)], [[np.nan], [0.1]]),
        ]
        for ctl, vals in bad:
            with pytest.raises(m.MpfError):
                pf.set_controls(ctl, np.array(vals))
        pf.set_controls([(m.CTRL_AVR, pv)], np.array([[1.02], [0.98]]))
        pf.solve(m.NR, m.FP64)
        r = pf.results()
        assert r.converged.all()
        assert abs(abs(r.v[0, pv]) - 1.02) < 1e-12 and abs(abs(r.v[1, pv]) - 0.98) < 1e-12


@pytest.mark.parametrize("use_graph", [1, 0])
def test_case_buffer_changes_between_solves(gpu, use_graph):
    """Captured iterations hold the device pointers of the cases they were captured
    with: solves after set_cases / set_controls swap those buffers must match fresh
    handles."""
    buses, branches = _grid("case118")
    *_, controls, vals = _controls(buses, branches, 40, 4)
    cases = [[] for _ in range(40)]
    sbus = m.load_scenarios(buses, 40, 0.03, 5)
    seq = [dict(sbus=sbus, ctl=None), dict(sbus=None, ctl=None), dict(sbus=None, ctl=vals),
           dict(sbus=sbus, ctl=vals[::-1].copy()), dict(sbus=None, ctl=None)]
    with m.PowerFlow(buses, branches, use_graph=use_graph) as pf:
        got = []
        for s in seq:
            pf.set_cases(cases, sbus=s["sbus"])
            if s["ctl"] is not None:
                pf.set_controls(controls, s["ctl"])
            pf.solve(m.NR, m.MIXED)
            got.append(pf.results())
    for s, r in zip(seq, got):
        with m.PowerFlow(buses, branches, use_graph=0) as pf:
            pf.set_cases(cases, sbus=s["sbus"])
            if s["ctl"] is not None:
                pf.set_controls(controls, s["ctl"])
            pf.solve(m.NR, m.MIXED)
            f = pf.results()
        assert np.array_equal(r.status, f.status) and np.array_equal(r.iterations, f.iterations)
        assert np.array_equal(r.v, f.v)
