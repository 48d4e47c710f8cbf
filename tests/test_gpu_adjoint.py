"""Adjoint gradients of the overload loss L = sum relu(|Sf| - 0.9 rating)^2 against
central FP64 finite differences (step 1e-6) of the same loss computed through full
power-flow solves, on P/Q injections and branch series admittances.

Tolerance (FP64 adjoint): the checked gradient entries (all coordinates x all cases)
agree with the finite differences to 1e-6 relative in the 2-norm, and each entry to
1e-5 relative plus 2e-9 absolute: a loss evaluated to ~1e-15 absolute gives central
differences at step 1e-6 a noise floor of ~5e-10, so entries of ~1e-4 cannot be
resolved past ~5e-6 relative.  Branch admittances are stepped by 1e-4 x |y_k|: their
gradients are small next to L, and with steps of 1e-6 and 1e-5 x |y_k| the differences
still sit at that noise floor while they converge to the adjoint values as the step
grows (the nearest branch is 2.8e-4 relative away from its overload threshold, so
the larger step stays on one side of the kink).  The FP32-factor adjoint (mixed
precision, refined twice with FP64 residuals) must agree with the FP64 one to 1e-9
relative.
"""
import numpy as np
import pytest

import mapol_b200 as m

pytestmark = pytest.mark.gpu

H = 1e-6
TOL = 1e-12


def _setup():
    buses, branches = m.synth_grid(118, 179, 53, 0.1, seed=2)
    out = m.select_outages(branches, 118, 7, 3)
    cases = [[]] + [[int(o)] for o in out]
    return buses, branches, cases


def _loss(buses, branches, cases, rating, sbus=None):
    with m.PowerFlow(buses, branches, tol=TOL) as pf:
        pf.set_cases(cases, sbus=sbus)
        pf.solve(m.NR, m.FP64)
        res = pf.results()
        assert (res.status == m.runpf.CONVERGED).all()
        pf.set_ratings(rating)
        return pf.branch_flows()["overload"]


def _check(adj, fd):
    adj, fd = np.concatenate(adj), np.concatenate(fd)
    assert np.linalg.norm(adj - fd) <= 1e-6 * np.linalg.norm(fd), (np.linalg.norm(adj - fd), np.linalg.norm(fd))
    err = np.abs(adj - fd)
    assert (err <= 1e-5 * np.abs(fd) + 2e-9).all(), err.max()


@pytest.fixture(scope="module")
def base(gpu):
    buses, branches, cases = _setup()
    with m.PowerFlow(buses, branches, tol=TOL) as pf:
        pf.set_cases(cases)
        pf.solve(m.NR, m.FP64)
        rating = 1.2 * np.abs(pf.branch_flows(flows=True)["sf"][0])
        pf.set_ratings(rating)
        L = pf.branch_flows()["overload"]
        g64 = pf.adjoint(m.FP64)
        g32 = pf.adjoint(m.MIXED)
    assert L[0] == 0.0 and (L[1:] > 0).sum() >= 3
    return buses, branches, cases, rating, L, g64, g32


def test_injection_gradients_match_finite_differences(base):
    buses, branches, cases, rating, L, g, _ = base
    nb = len(buses)
    s0 = np.stack([np.tile(buses["p"], (len(cases), 1)), np.tile(buses["q"], (len(cases), 1))], -1)
    pq = np.where(buses["type"] == 1)[0]
    pv = np.where(buses["type"] == 2)[0]
    rng = np.random.default_rng(0)
    coords = [(i, 0) for i in rng.choice(pq, 6, replace=False)] + [(i, 0) for i in rng.choice(pv, 4, replace=False)]
    coords += [(i, 1) for i in rng.choice(pq, 6, replace=False)]
    adjs, fds = [], []
    for i, comp in coords:
        sp, sm = s0.copy(), s0.copy()
        sp[:, i, comp] += H
        sm[:, i, comp] -= H
        fds.append((_loss(buses, branches, cases, rating, sp) - _loss(buses, branches, cases, rating, sm)) / (2 * H))
        adjs.append((g["grad_p"] if comp == 0 else g["grad_q"])[:, i])
    _check(adjs, fds)
    slack = np.where(buses["type"] == 3)[0][0]
    assert (g["grad_p"][:, slack] == 0).all() and (g["grad_q"][:, pv] == 0).all()
    assert nb == 118


def test_branch_admittance_gradients_match_finite_differences(base):
    buses, branches, cases, rating, L, g, _ = base
    rng = np.random.default_rng(1)
    outaged = {c[0] for c in cases if c}
    ks = [k for k in rng.permutation(len(branches)) if k not in outaged][:5] + [cases[1][0]]
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
                Ls.append(_loss(buses, br, cases, rating))
            fd = (Ls[0] - Ls[1]) / (2 * hk)
            adj = (g["grad_g"] if comp == 0 else g["grad_b"])[:, k]
            # an outaged branch has no effect in the cases that remove it
            fd[[i for i, c in enumerate(cases) if c and c[0] == k]] = 0.0
            adjs.append(adj)
            fds.append(fd)
    _check(adjs, fds)


def test_fp32_factor_adjoint_close_to_fp64(base):
    *_, g64, g32 = base
    for key in ("grad_p", "grad_q", "grad_g", "grad_b"):
        a, b = g64[key], g32[key]
        assert np.abs(a - b).max() <= 1e-9 * np.abs(a).max() + 1e-15, (key, np.abs(a - b).max(), np.abs(a).max())


def test_autograd_function_backward_is_the_adjoint(base):
    import torch

    from mapol_b200.autograd import PowerFlowLoss

    buses, branches, cases, rating, L, g, _ = base
    n = len(cases)
    p = torch.tensor(np.tile(buses["p"], (n, 1)), dtype=torch.float64, requires_grad=True)
    q = torch.tensor(np.tile(buses["q"], (n, 1)), dtype=torch.float64, requires_grad=True)
    with m.PowerFlow(buses, branches, tol=TOL) as pf:
        pf.set_ratings(rating)
        out = PowerFlowLoss.apply(p, q, pf, cases, m.FP64)
        np.testing.assert_allclose(out.detach().numpy(), L, rtol=1e-9, atol=1e-14)
        w = torch.arange(1, n + 1, dtype=torch.float64)
        (out * w).sum().backward()
    np.testing.assert_allclose(p.grad.numpy(), g["grad_p"] * w.numpy()[:, None], rtol=1e-9, atol=1e-14)
    np.testing.assert_allclose(q.grad.numpy(), g["grad_q"] * w.numpy()[:, None], rtol=1e-9, atol=1e-14)


def _explicit_loss(buses, branches, v, rating, outages):
    """sum relu(|Sf| - 0.9 rating)^2 at complex voltages v (pi model, numpy)."""
    br = branches
    ys = np.where(br["status"] == 1, 1.0 / (br["r"] + 1j * br["x"]), 0.0)
    bc = np.where(br["status"] == 1, br["b"], 0.0)
    tap = np.where(br["tap"] != 0, br["tap"], 1.0) * np.exp(1j * np.pi / 180 * br["shift"])
    yff = (ys + 0.5j * bc) / np.abs(tap) ** 2
    yft = -ys / np.conj(tap)
    vf, vt = v[br["from"]], v[br["to"]]
    sf = vf * np.conj(yff * vf + yft * vt)
    ex = np.abs(sf) - 0.9 * rating
    on = np.ones(len(br), bool)
    on[list(outages)] = False
    return float(np.sum(np.where(on & (ex > 0), ex * ex, 0.0)))


def test_adjoint_matches_dense_implicit_function_gradient(base):
    """lambda = J^-T dL/dx with the oracle's Jacobian at the oracle's solution (dense
    FP64 solve), dL/dx by central differences (step 1e-7) of the explicit loss: the
    P/Q gradients agree with the adjoint to 1e-6 relative (2-norm over each case)."""
    from oracle import oracle

    buses, branches, cases, rating, L, g, _ = base
    ref = oracle.runpf(buses, branches, cases, alg=0, tol=1e-12)
    pv = np.where(buses["type"] == 2)[0]
    pq = np.where(buses["type"] == 1)[0]
    npv, npq = len(pv), len(pq)
    checked = 0
    for c, out in enumerate(cases):
        if L[c] == 0.0:
            continue
        v = ref["v"][c]
        _, (jp, jc, jv), _ = oracle.nr_system(buses, branches, v, outages=out)
        n = npv + 2 * npq
        J = np.zeros((n, n))
        for r in range(n):
            J[r, jc[jp[r]:jp[r + 1]]] = jv[jp[r]:jp[r + 1]]
        # x = [Va (PV, PQ), Vm (PQ)], bus-index order within each group
        va_bus = np.concatenate([pv, pq])
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
            dldx[k] = (_explicit_loss(buses, branches, vp, rating, out)
                       - _explicit_loss(buses, branches, vm_, rating, out)) / (2 * h)
        lam = np.linalg.solve(J.T, dldx)
        gp = np.zeros(len(buses))
        gq = np.zeros(len(buses))
        gp[va_bus] = lam[:npv + npq]
        gq[pq] = lam[npv + npq:]
        a = np.concatenate([g["grad_p"][c], g["grad_q"][c]])
        d = np.concatenate([gp, gq])
        assert np.linalg.norm(a - d) <= 1e-6 * np.linalg.norm(d), (c, np.linalg.norm(a - d), np.linalg.norm(d))
        checked += 1
    assert checked >= 3
