"""The reference's bundled PEGASE grids (src/datasets/case1354pegase.m,
case2869pegase.m, case9241pegase.m, converted by mapol_b200.matpower with the
reference loader's semantics, loadMatpowerFormat.h:14-209) as real-grid inputs:
base case + N-1 outages of non-bridge branches, Newton-Raphson in plain FP64 and in
mixed precision, against the oracle (flags identical, FP64 iterations identical, mixed
at most one more, |V - V_oracle| < 1e-8 p.u.)."""
import os

import numpy as np
import pytest

import mapol_b200 as m
from oracle import oracle

from .parity import TIGHT_TOL, compare

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("name,n_out", [("case1354pegase", 200), ("case2869pegase", 200), ("case9241pegase", 160)])
def test_pegase_n1_matches_oracle(gpu, name, n_out):
    g = np.load(os.path.join(HERE, "golden", "matpower_cases.npz"))
    buses, branches = g[name + "_buses"], g[name + "_branches"]
    cases = m.n1_cases(branches, len(buses), n_out, 7, with_base=True)
    ref = oracle.runpf(buses, branches, cases, alg=m.NR)
    assert ref["converged"][0]  # the base case solves
    with m.PowerFlow(buses, branches) as pf:
        pf.set_cases(cases)
        pf.solve(m.NR, m.FP64)
        res = pf.results()
        pf.solve(m.NR, m.MIXED)
        res32 = pf.results()

    def tight(idx):
        return oracle.runpf(buses, branches, [cases[i] for i in idx], alg=m.NR, tol=TIGHT_TOL)

    conv = compare(res, ref)
    compare(res32, ref, max_extra_iter=1, tight=tight)
    assert conv.mean() > 0.9
