"""Adjoint gradients at the size the benchmark fixes for them: the 1354-bus synthetic
grid with 4096 load scenarios (each load x (1 + N(0, 0.05^2)), fixed power factor),
overload loss L = sum relu(|Sf| - 0.9 rating)^2 with rating = 1.2 x the base case's
|Sf|, central FP64 differences (step 1e-6) on 64 random injection coordinates.  Each
coordinate is perturbed in every scenario at once (two batched solves per
coordinate), so the check covers 64 x 4096 gradient entries.

Both forms are checked against the same differences: FP64 (solve and adjoint in
FP64) and the mixed form the configuration names (mixed-precision Newton, adjoint on
FP32 factors refined with FP64 residuals).  Tolerance: 1e-6 relative in the 2-norm,
as the 118-bus adjoint tests, and every entry within 1e-6 of the largest gradient.
No tighter per-entry bound: among 4096 scenarios some branch flows lie within the
+-1e-6 stencil of an overload threshold, where the loss has a kink and a central
difference is not a derivative, and the smallest entries sit at the differences'
noise floor.

The dense implicit-function check repeats the 118-bus one at this size: for a few
scenarios, lambda = J^-T dL/dx with the oracle's Jacobian at the oracle's solution
(dense FP64 solve, n = 2447) and dL/dx by central differences of the explicit loss."""
import numpy as np
import pytest

import mapol_b200 as m

from .test_gpu_adjoint import _explicit_loss

pytestmark = pytest.mark.gpu

H = 1e-6
TOL = 1e-12
N_SCEN = 4096


@pytest.fixture(scope="module")
def cfg4(gpu):
    buses, branches, _ = m.workload("cfg4_1354bus")
    sb = m.load_scenarios(buses, N_SCEN, 0.05, 11)
    with m.PowerFlow(buses, branches, tol=TOL) as pf:
        pf.set_cases([[]])
        pf.solve(m.NR, m.FP64)
        assert pf.results().converged.all()
        rating = 1.2 * np.abs(pf.branch_flows(flows=True)["sf"][0])
        pf.set_ratings(rating)

        def loss(s, prec=m.FP64):
            pf.set_cases([[]] * N_SCEN, sbus=s)
            pf.solve(m.NR, prec)
            assert pf.results().converged.all()
            return pf.branch_flows()["overload"]

        L = loss(sb)
        g64 = pf.adjoint(m.FP64)
        L32 = loss(sb, m.MIXED)
        v32 = pf.results().v
        g32 = pf.adjoint(m.MIXED)
        assert (L > 0).sum() > N_SCEN // 4
        np.testing.assert_allclose(L32, L, rtol=1e-8, atol=1e-14)
        pq = np.where(buses["type"] == 1)[0]
        pv = np.where(buses["type"] == 2)[0]
        rng = np.random.default_rng(5)
        coords = ([(int(i), 0) for i in rng.choice(pq, 24, replace=False)] +
                  [(int(i), 0) for i in rng.choice(pv, 16, replace=False)] +
                  [(int(i), 1) for i in rng.choice(pq, 24, replace=False)])
        fds = []
        for i, comp in coords:
            sp, sm = sb.copy(), sb.copy()
            sp[:, i, comp] += H
            sm[:, i, comp] -= H
            fds.append((loss(sp) - loss(sm)) / (2 * H))
    return dict(buses=buses, branches=branches, sb=sb, rating=rating, L=L, g64=g64, g32=g32, v32=v32,
                coords=coords, fd=np.concatenate(fds))


@pytest.mark.parametrize("form", ["g64", "g32"])
def test_config4_scenario_gradients_match_finite_differences(cfg4, form):
    g = cfg4[form]
    adj = np.concatenate([(g["grad_p"] if comp == 0 else g["grad_q"])[:, i] for i, comp in cfg4["coords"]])
    fd = cfg4["fd"]
    assert np.abs(fd).max() > 0
    assert np.linalg.norm(adj - fd) <= 1e-6 * np.linalg.norm(fd), (np.linalg.norm(adj - fd), np.linalg.norm(fd))
    err = np.abs(adj - fd)
    assert err.max() <= 1e-6 * np.abs(fd).max(), (err.max(), np.abs(fd).max())


def test_config4_dense_implicit_function_gradient(cfg4):
    from oracle import oracle

    buses, branches, sb, rating, L = cfg4["buses"], cfg4["branches"], cfg4["sb"], cfg4["rating"], cfg4["L"]
    pv = np.where(buses["type"] == 2)[0]
    pq = np.where(buses["type"] == 1)[0]
    npv, npq = len(pv), len(pq)
    n = npv + 2 * npq
    va_bus = np.concatenate([pv, pq])
    scen = [int(c) for c in np.where(L > 0)[0][:3]]
    checked = 0
    for c in scen:
        b = buses.copy()
        b["p"], b["q"] = sb[c, :, 0], sb[c, :, 1]
        v = oracle.runpf(b, branches, [[]], alg=0, tol=1e-12)["v"][0]
        _, (jp, jc, jv), _ = oracle.nr_system(b, branches, v)
        J = np.zeros((n, n))
        for r in range(n):
            J[r, jc[jp[r]:jp[r + 1]]] = jv[jp[r]:jp[r + 1]]
        dldx = np.zeros(n)
        h = 1e-7
        for k in range(n):
            vp, vm_ = v.copy(), v.copy()
            if k < npv + npq:
                i = va_bus[k]
                vp[i] *= np.exp(1j * h)
                vm_[i] *= np.exp(-1j * h)
            else:
                i = pq[k - npv - npq]
                vp[i] *= (abs(v[i]) + h) / abs(v[i])
                vm_[i] *= (abs(v[i]) - h) / abs(v[i])
            dldx[k] = (_explicit_loss(b, branches, vp, rating, ()) - _explicit_loss(b, branches, vm_, rating, ())) / (2 * h)
        lam = np.linalg.solve(J.T, dldx)
        gp = np.zeros(len(buses))
        gq = np.zeros(len(buses))
        gp[va_bus] = lam[:npv + npq]
        gq[pq] = lam[npv + npq:]
        d = np.concatenate([gp, gq])
        for form in ("g64", "g32"):
            g = cfg4[form]
            a = np.concatenate([g["grad_p"][c], g["grad_q"][c]])
            assert np.linalg.norm(a - d) <= 1e-6 * np.linalg.norm(d), (form, c, np.linalg.norm(a - d), np.linalg.norm(d))
        checked += 1
    assert checked == 3
