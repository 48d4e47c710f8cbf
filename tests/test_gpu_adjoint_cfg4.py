"""Adjoint gradients at the size the benchmark fixes for them: the 1354-bus synthetic
grid with 4096 load scenarios (each load x (1 + N(0, 0.05^2)), fixed power factor),
overload loss L = sum relu(|Sf| - 0.9 rating)^2 with rating = 1.2 x the base case's
|Sf|, central FP64 differences (step 1e-6) on 64 random injection coordinates.  Each
coordinate is perturbed in every scenario at once (two batched solves per
coordinate), so the check covers 64 x 4096 gradient entries.  Tolerance: 1e-6
relative in the 2-norm, as the 118-bus adjoint tests, and every entry within 1e-6 of
the largest gradient.  No tighter per-entry bound: among 4096 scenarios some branch
flows lie within the +-1e-6 stencil of an overload threshold, where the loss has a
kink and a central difference is not a derivative, and the smallest entries sit at
the differences' noise floor."""
import numpy as np
import pytest

import mapol_b200 as m

pytestmark = pytest.mark.gpu

H = 1e-6
TOL = 1e-12
N_SCEN = 4096


def test_config4_scenario_gradients_match_finite_differences(gpu):
    buses, branches, _ = m.workload("cfg4_1354bus")
    sb = m.load_scenarios(buses, N_SCEN, 0.05, 11)
    with m.PowerFlow(buses, branches, tol=TOL) as pf:
        pf.set_cases([[]])
        pf.solve(m.NR, m.FP64)
        assert pf.results().converged.all()
        rating = 1.2 * np.abs(pf.branch_flows(flows=True)["sf"][0])
        pf.set_ratings(rating)

        def loss(s):
            pf.set_cases([[]] * N_SCEN, sbus=s)
            pf.solve(m.NR, m.FP64)
            assert pf.results().converged.all()
            return pf.branch_flows()["overload"]

        L = loss(sb)
        g = pf.adjoint(m.FP64)
        assert (L > 0).sum() > N_SCEN // 4
        pq = np.where(buses["type"] == 1)[0]
        pv = np.where(buses["type"] == 2)[0]
        rng = np.random.default_rng(5)
        coords = ([(int(i), 0) for i in rng.choice(pq, 24, replace=False)] +
                  [(int(i), 0) for i in rng.choice(pv, 16, replace=False)] +
                  [(int(i), 1) for i in rng.choice(pq, 24, replace=False)])
        adjs, fds = [], []
        for i, comp in coords:
            sp, sm = sb.copy(), sb.copy()
            sp[:, i, comp] += H
            sm[:, i, comp] -= H
            fds.append((loss(sp) - loss(sm)) / (2 * H))
            adjs.append((g["grad_p"] if comp == 0 else g["grad_q"])[:, i])
    adj, fd = np.concatenate(adjs), np.concatenate(fds)
    assert np.abs(fd).max() > 0
    assert np.linalg.norm(adj - fd) <= 1e-6 * np.linalg.norm(fd), (np.linalg.norm(adj - fd), np.linalg.norm(fd))
    err = np.abs(adj - fd)
    assert err.max() <= 1e-6 * np.abs(fd).max(), (err.max(), np.abs(fd).max())
