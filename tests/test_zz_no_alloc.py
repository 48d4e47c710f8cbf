"""mpf_mismatch_noalloc: the mismatch evaluation for callers that cannot allocate
device memory when they call it (inside stream capture, real-time loops, or when
another framework's pool owns the GPU).  It must give mpf_mismatch's result, call
after call, from its fixed built-in scratch, and refuse batches larger than that
scratch.  Collected last on purpose (file name) so a failure here cannot hide
another test's result.
"""
import numpy as np
import pytest

import mapol_b200 as m

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(np.stack([a.real, a.imag], -1))).cuda()


def test_noalloc_matches_mismatch_two_calls_in_a_row(gpu):
    import torch

    from mapol_b200._lib import lib

    buses, branches, cases = m.workload("cfg1_300bus")
    cases = cases[:70]
    with m.PowerFlow(buses, branches) as pf:
        pf.set_cases(cases)
        pf.solve(m.NR, m.FP64)
        res = pf.results()
        flat = np.zeros((len(cases), len(buses)), complex)
        flat[:] = buses["vm"] * np.exp(1j * buses["va"])
        ref = torch.zeros(len(cases), dtype=torch.float64, device="cuda")
        got = torch.zeros(len(cases), dtype=torch.float64, device="cuda")
        # large mismatches first, then small ones: leftovers in the scratch would show
        for volts in (flat, res.v, res.v):
            v = _dev(volts)
            assert lib().mpf_mismatch(pf._h, v.data_ptr(), ref.data_ptr(), None) == 0
            assert lib().mpf_mismatch_noalloc(pf._h, v.data_ptr(), got.data_ptr(), None) == 0
            torch.cuda.synchronize()
            np.testing.assert_allclose(got.cpu().numpy(), ref.cpu().numpy(), rtol=1e-12, atol=0.0)
        assert (got.cpu().numpy() < 1e-8).all()


def test_noalloc_rejects_batches_beyond_its_scratch(gpu):
    import torch

    from mapol_b200._lib import lib

    buses, branches = m.synth_grid(30, 41, 5)
    with m.PowerFlow(buses, branches) as pf:
        pf.set_cases([[]] * 65537)
        v = torch.zeros((65537, 30, 2), dtype=torch.float64, device="cuda")
        out = torch.zeros(65537, dtype=torch.float64, device="cuda")
        rc = lib().mpf_mismatch_noalloc(pf._h, v.data_ptr(), out.data_ptr(), None)
        assert rc == 1  # MPF_ERR_BAD_INPUT
        assert b"65536" in lib().mpf_last_error(pf._h)
