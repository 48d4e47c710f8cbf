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
