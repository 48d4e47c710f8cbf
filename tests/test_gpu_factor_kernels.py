"""Every factorisation kernel computes the same factors, bit for bit.

The autotuner picks one kernel per factorisation launch by timing, so a run may use
any of them: warp teams (kind 0), 256-thread teams with the partial LU in shared
memory (1), the register-tile LU (2), 512- and 1024-thread teams (3), two pivots per
barrier (5), at every lane-chunk width.  All apply the same operations to every entry
of a front in the same order (the extend-add in child order, then the right-looking
updates pivot by pivot), so the factors, and with them every Newton iterate, are
identical.  MPF_FACTOR_KIND=k forces kind k on every launch that has such a
candidate (the others keep the tuned kernel); the converged voltages, statuses and
iteration counts must equal those of the tuned run exactly, in both precisions.
"""
import os

import numpy as np
import pytest

import mapol_b200 as m

pytestmark = pytest.mark.gpu


def _solve(buses, branches, cases, prec, kind=None):
    if kind is not None:
        os.environ["MPF_FACTOR_KIND"] = str(kind)
    try:
        with m.PowerFlow(buses, branches) as pf:
            pf.set_cases(cases)
            pf.solve(m.NR, prec)
            return pf.results()
    finally:
        os.environ.pop("MPF_FACTOR_KIND", None)


@pytest.mark.parametrize("prec", [m.MIXED, m.FP64])
def test_every_factor_kernel_gives_identical_results(gpu, prec):
    buses, branches, cases = m.workload("cfg3_9241bus")
    cases = cases[:64]
    ref = _solve(buses, branches, cases, prec)
    assert (ref.status == m.runpf.CONVERGED).all()
    for kind in (0, 1, 2, 3, 5):
        res = _solve(buses, branches, cases, prec, kind)
        assert np.array_equal(res.status, ref.status), kind
        assert np.array_equal(res.iterations, ref.iterations), kind
        assert np.array_equal(res.v, ref.v), kind
