"""Comparison of GPU results with the oracle, shared by the GPU parity tests.

The bar: identical convergence flags; every converged case at max |F| < 1e-8 p.u.
(the reference's criterion, newtonpf.h:394,518); iteration counts equal to the
oracle's, or up to max_extra_iter more (mixed precision solves each Newton step in
FP32, so it may take one more); voltages within v_tol of the oracle's.

A case that took more iterations than the oracle stopped further past the 1e-8
criterion than the oracle did (its last step squared an already small error), so on
an ill-conditioned case its voltages can sit closer to the exact solution than the
oracle's own, by more than v_tol.  Such cases are compared with `tight(idx)`: the
oracle run on those cases to max |F| < 1e-11, i.e. to the same side of the criterion.
"""
import numpy as np

import mapol_b200 as m

TIGHT_TOL = 1e-11


def compare(res, ref, max_extra_iter=0, v_tol=1e-8, tight=None):
    conv = res.status == m.runpf.CONVERGED
    assert np.array_equal(conv, ref["converged"]), (np.where(conv != ref["converged"]), res.status)
    assert (res.max_mis[conv] < 1e-8).all()
    d_it = res.iterations - ref["iterations"]
    assert (d_it[conv] >= 0).all() and (d_it[conv] <= max_extra_iter).all(), (res.iterations, ref["iterations"])
    same = conv & (d_it == 0)
    extra = conv & (d_it > 0)
    if same.any():
        dv = np.abs(res.v[same] - ref["v"][same]).max()
        assert dv < v_tol, dv
    if extra.any():
        idx = np.where(extra)[0]
        v_ref = ref["v"][idx]
        if tight is not None:
            t = tight(idx)
            ok = t["converged"]
            v_ref = np.where(ok[:, None], t["v"], v_ref)
        dv = np.abs(res.v[idx] - v_ref).max()
        assert dv < v_tol, dv
    return conv
