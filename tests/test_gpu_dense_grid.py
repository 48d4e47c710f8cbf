"""A densely meshed grid: the uniform-random topology of the synthetic generator
(extra branches between random bus pairs, not nearest neighbours) at 1354 buses, whose
Newton system has fronts of up to 352 rows (37 supernodes above the 167 rows a dense
front of one FP64 lane can hold in shared memory; B' and B'' have such fronts too).  Those fronts run k_mf_factor_big (panel
in shared memory, trailing block in global memory); the results must meet the same
bar as every other grid against the CPU oracle: identical flags, identical FP64
iteration counts (mixed at most one more), |dV| < 1e-8 p.u.  The same split is checked
bit for bit against the dense loop on the CPU by tests/native/mf_emulate.cpp."""
import numpy as np
import pytest

import mapol_b200 as m
from oracle import oracle

from .parity import TIGHT_TOL, compare

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dense_grid(gpu):
    buses, branches = m.synth_grid(1354, 1991, 260, tap_fraction=0.05, seed=5, topology=1)
    cases = [[]] + m.n1_cases(branches, len(buses), 63, 3)
    return buses, branches, cases


def test_dense_grid_nr_both_precisions_match_oracle(dense_grid):
    buses, branches, cases = dense_grid
    ref = oracle.runpf(buses, branches, cases, alg=m.NR)
    assert ref["converged"].all()

    def tight(idx):
        return oracle.runpf(buses, branches, [cases[i] for i in idx], alg=m.NR, tol=TIGHT_TOL)

    with m.PowerFlow(buses, branches) as pf:
        pf.set_cases(cases)
        for prec, extra in ((m.FP64, 0), (m.MIXED, 1)):
            pf.solve(m.NR, prec)
            res = pf.results()
            conv = compare(res, ref, extra, 1e-8, tight if extra else None)
            assert conv.all()


@pytest.mark.parametrize("alg", [m.FDXB, m.FDBX])
def test_dense_grid_fast_decoupled_matches_oracle(dense_grid, alg):
    """B' and B'' of the dense grid have large fronts too; their factors feed the
    forward substitution kernel with stored factors."""
    buses, branches, cases = dense_grid
    ref = oracle.runpf(buses, branches, cases, alg=alg)
    with m.PowerFlow(buses, branches) as pf:
        pf.set_cases(cases)
        pf.solve(alg, m.FP64)
        compare(pf.results(), ref)


def test_dense_grid_kernels_agree_bit_for_bit(dense_grid):
    """Graph replay and direct launches, and a second handle, give the same bits."""
    buses, branches, cases = dense_grid
    out = []
    for use_graph in (1, 0):
        with m.PowerFlow(buses, branches, use_graph=use_graph) as pf:
            pf.set_cases(cases)
            pf.solve(m.NR, m.MIXED)
            out.append(pf.results().v)
    assert np.array_equal(out[0], out[1])


def test_dense_grid_adjoint_matches_finite_differences(gpu):
    """The adjoint on the dense grid: its transposed substitutions run on the large
    fronts' factors with fewer warps per block (a warp's slice of x of a 352-row front
    takes 86 KB in FP64).  Injection gradients against central FP64 differences (step
    1e-6, the tolerance of tests/test_gpu_adjoint.py), and the refined FP32-factor
    adjoint against the FP64 one."""
    tol, h = 1e-12, 1e-6
    buses, branches = m.synth_grid(1354, 1991, 260, tap_fraction=0.05, seed=5, topology=1)
    cases = [[]] + m.n1_cases(branches, len(buses), 7, 3)

    def loss(rating, sbus=None):
        with m.PowerFlow(buses, branches, tol=tol) as pf:
            pf.set_cases(cases, sbus=sbus)
            pf.solve(m.NR, m.FP64)
            assert (pf.results().status == m.runpf.CONVERGED).all()
            pf.set_ratings(rating)
            return pf.branch_flows()["overload"]

    with m.PowerFlow(buses, branches, tol=tol) as pf:
        pf.set_cases(cases)
        pf.solve(m.NR, m.FP64)
        rating = 1.2 * np.abs(pf.branch_flows(flows=True)["sf"][0])
        pf.set_ratings(rating)
        L = pf.branch_flows()["overload"]
        g64 = pf.adjoint(m.FP64)
        g32 = pf.adjoint(m.MIXED)
    assert (L > 0).any()
    s0 = np.stack([np.tile(buses["p"], (len(cases), 1)), np.tile(buses["q"], (len(cases), 1))], -1)
    # PQ buses with gradients well above the differences' noise floor (~5e-10): three of
    # the twenty largest in P and in Q
    pq = np.where(buses["type"] == 1)[0]
    rng = np.random.default_rng(4)
    coords = []
    for comp, key in ((0, "grad_p"), (1, "grad_q")):
        top = pq[np.argsort(-np.abs(g64[key][:, pq]).max(0))[:20]]
        coords += [(int(i), comp) for i in rng.choice(top, 3, replace=False)]
    adjs, fds = [], []
    for i, comp in coords:
        sp, sm = s0.copy(), s0.copy()
        sp[:, i, comp] += h
        sm[:, i, comp] -= h
        fds.append((loss(rating, sp) - loss(rating, sm)) / (2 * h))
        adjs.append((g64["grad_p"] if comp == 0 else g64["grad_q"])[:, i])
    adj, fd = np.concatenate(adjs), np.concatenate(fds)
    assert np.linalg.norm(adj - fd) <= 1e-6 * np.linalg.norm(fd), (np.linalg.norm(adj - fd), np.linalg.norm(fd))
    assert (np.abs(adj - fd) <= 1e-5 * np.abs(fd) + 2e-9).all()
    for key in ("grad_p", "grad_q", "grad_g", "grad_b"):
        a, b = g64[key], g32[key]
        assert np.abs(a - b).max() <= 1e-9 * np.abs(a).max() + 1e-15, (key, np.abs(a - b).max())
