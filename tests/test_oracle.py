"""CPU tests of the oracle itself (the checker): pinned against an independent
numpy/scipy Newton, a hand-solvable 2-bus case, the reference's Eigen SparseLU
option, and the committed golden fixtures."""
import os

import numpy as np
import pytest

import mapol_b200 as m
from oracle import oracle

from .np_newton import newton

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module", autouse=True)
def _built(built):
    return built


def two_bus(p_load, q_load, x, r=0.0, v1=1.0):
    buses = np.zeros(2, m.BUS_DTYPE)
    buses["type"] = [3, 1]
    buses["vm"] = [v1, 1.0]
    buses["p"] = [0.0, -p_load]
    buses["q"] = [0.0, -q_load]
    br = np.zeros(1, m.BRANCH_DTYPE)
    br[0]["from"], br[0]["to"], br[0]["status"] = 0, 1, 1
    br[0]["r"], br[0]["x"] = r, x
    return buses, br


def test_two_bus_lossless_closed_form():
    # load P + jQ behind reactance x from a stiff source v1: with a = |V2|^2,
    # a^2 + (2 Q x - v1^2) a + x^2 (P^2 + Q^2) = 0 (high-voltage root), sin(d) = -P x / (v1 |V2|)
    P, Q, x, v1 = 0.6, 0.2, 0.3, 1.02
    buses, br = two_bus(P, Q, x, v1=v1)
    r = oracle.runpf(buses, br, [[]], alg=m.NR)
    assert r["converged"][0]
    b = 2 * Q * x - v1 ** 2
    a = (-b + np.sqrt(b * b - 4 * x * x * (P * P + Q * Q))) / 2
    v2 = np.sqrt(a)
    d = np.arcsin(-P * x / (v1 * v2))
    assert abs(abs(r["v"][0, 1]) - v2) < 1e-10
    assert abs(np.angle(r["v"][0, 1]) - d) < 1e-10


@pytest.mark.parametrize("name", ["cfg0_30bus", "cfg1_300bus"])
def test_oracle_matches_independent_numpy_newton(name):
    buses, branches, cases = m.workload(name)
    sel = cases[:12]
    r = oracle.runpf(buses, branches, sel, alg=m.NR)
    for k, c in enumerate(sel):
        v, it, ok = newton(buses, branches, c)
        assert ok == bool(r["converged"][k])
        assert it == r["iterations"][k]
        assert np.abs(v - r["v"][k]).max() < 1e-9


def test_fd_variants_reach_the_newton_solution():
    buses, branches, cases = m.workload("cfg1_300bus")
    sel = cases[:10]
    ref = oracle.runpf(buses, branches, sel, alg=m.NR, tol=1e-11)
    for alg in (m.FDXB, m.FDBX):
        r = oracle.runpf(buses, branches, sel, alg=alg, tol=1e-11)
        assert r["converged"].all()
        assert np.abs(r["v"] - ref["v"]).max() < 1e-9


@pytest.mark.skipif(not oracle.has_eigen(), reason="oracle/_ref (reference Eigen build) not built")
@pytest.mark.parametrize("alg", [m.NR, m.FDXB])
def test_own_lu_matches_reference_eigen_sparselu(alg):
    buses, branches, cases = m.workload("cfg1_300bus")
    sel = cases[:16]
    a = oracle.runpf(buses, branches, sel, alg=alg, solver=oracle.SOLVER_GP)
    b = oracle.runpf(buses, branches, sel, alg=alg, solver=oracle.SOLVER_EIGEN)
    assert np.array_equal(a["iterations"], b["iterations"])
    assert np.array_equal(a["converged"], b["converged"])
    assert np.abs(a["v"] - b["v"]).max() < 1e-11


def test_angle_quirk_is_identical_below_90_degrees():
    buses, branches, cases = m.workload("cfg0_30bus")
    a = oracle.runpf(buses, branches, cases, alg=m.NR, angle_mode=0)
    b = oracle.runpf(buses, branches, cases, alg=m.NR, angle_mode=1)
    assert np.abs(np.angle(a["v"])).max() < np.pi / 2
    assert np.array_equal(a["iterations"], b["iterations"])
    assert np.abs(a["v"] - b["v"]).max() < 1e-12


def test_losses_equal_net_injection():
    buses, branches, cases = m.workload("cfg0_30bus")
    r = oracle.runpf(buses, branches, cases[:3], alg=m.NR, tol=1e-12)
    for k in range(3):
        v = r["v"][k]
        p, c, val = oracle.ybus(buses, branches, cases[k])
        import scipy.sparse as sp

        Y = sp.csr_matrix((val, c, p), shape=(len(buses), len(buses)))
        s_inj = v * np.conj(Y @ v)
        assert abs(oracle.loss(buses, branches, v, cases[k]) - s_inj.real.sum()) < 1e-10


def test_golden_fixtures_reproduced():
    path = os.path.join(HERE, "golden", "oracle_cfg0_cfg1.npz")
    g = np.load(path)
    for name in ("cfg0_30bus", "cfg1_300bus"):
        buses, branches, cases = m.workload(name)
        assert np.array_equal(buses.view(np.uint8), g[f"{name}_buses"].view(np.uint8))
        assert np.array_equal(branches.view(np.uint8), g[f"{name}_branches"].view(np.uint8))
        n = len(g[f"{name}_nr_iterations"])
        for alg, tag in ((m.NR, "nr"), (m.FDXB, "fdxb"), (m.FDBX, "fdbx")):
            r = oracle.runpf(buses, branches, cases[:n], alg=alg)
            assert np.array_equal(r["iterations"], g[f"{name}_{tag}_iterations"])
            assert np.array_equal(r["converged"], g[f"{name}_{tag}_converged"])
            assert np.abs(r["v"] - g[f"{name}_{tag}_v"]).max() < 1e-12


def test_qlim_oracle_switches_and_holds_the_limit():
    """runpf_qlim on the IEEE 14-bus case: limits that never bind change nothing; a
    limit just below a PV bus's solved Q switches it to PQ, where its Q then equals
    the limit and its |V| leaves the set-point."""
    import os

    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "matpower_cases.npz"))
    b, br = g["case14_buses"], g["case14_branches"]
    nb = len(b)
    base = oracle.runpf(b, br, [[]], alg=0)
    wide = oracle.runpf_qlim(b, br, [[]], np.full(nb, -np.inf), np.full(nb, np.inf))
    assert not wide["switched"].any() and np.array_equal(wide["v"], base["v"])
    v = base["v"][0]
    ptr, col, val = oracle.ybus(b, br)
    ib = np.array([np.dot(val[ptr[i]:ptr[i + 1]], v[col[ptr[i]:ptr[i + 1]]]) for i in range(nb)])
    q = (v * np.conj(ib)).imag
    pv = np.where(b["type"] == 2)[0]
    k = pv[np.argmax(q[pv])]
    qmax = np.full(nb, np.inf)
    qmax[k] = q[k] - 0.05
    r = oracle.runpf_qlim(b, br, [[]], np.full(nb, -np.inf), qmax)
    assert r["converged"][0] and r["switched"][0, k] and r["switched"][0].sum() == 1
    v2 = r["v"][0]
    bb = b.copy()
    bb["type"][k] = 1
    bb["q"][k] = qmax[k]
    ptr, col, val = oracle.ybus(bb, br)
    ib2 = np.array([np.dot(val[ptr[i]:ptr[i + 1]], v2[col[ptr[i]:ptr[i + 1]]]) for i in range(nb)])
    assert abs((v2[k] * np.conj(ib2[k])).imag - qmax[k]) < 1e-9
    assert abs(abs(v2[k]) - b["vm"][k]) > 1e-4
