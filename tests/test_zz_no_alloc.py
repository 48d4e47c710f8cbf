"""mpf_mismatch_noalloc: the mismatch evaluation for callers that cannot allocate
device memory when they call it (real-time loops that may not enter an allocator, or
processes where another framework's caching pool owns the GPU's memory).  It must give mpf_mismatch's result, call
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


def test_noalloc_at_its_documented_limit(gpu):
    """Exactly 65536 cases (the documented maximum) launch and equal mpf_mismatch."""
    import torch

    from mapol_b200._lib import lib

    buses, branches = m.synth_grid(30, 41, 5)
    n = 65536
    rng = np.random.default_rng(3)
    with m.PowerFlow(buses, branches) as pf:
        pf.set_cases([[]] * n)
        v0 = buses["vm"] * np.exp(1j * buses["va"])
        volts = v0[None] * (1.0 + 0.01 * rng.standard_normal((n, len(buses))))
        v = _dev(volts)
        ref = torch.zeros(n, dtype=torch.float64, device="cuda")
        got = torch.full((n,), -1.0, dtype=torch.float64, device="cuda")
        assert lib().mpf_mismatch(pf._h, v.data_ptr(), ref.data_ptr(), None) == 0
        for _ in range(2):
            got.fill_(-1.0)
            assert lib().mpf_mismatch_noalloc(pf._h, v.data_ptr(), got.data_ptr(), None) == 0
            torch.cuda.synchronize()
            np.testing.assert_allclose(got.cpu().numpy(), ref.cpu().numpy(), rtol=1e-12, atol=0.0)
        assert (ref.cpu().numpy() > 0).all()


def test_noalloc_on_a_user_stream_then_new_cases(gpu):
    """A call on the caller's stream, followed at once by mpf_set_cases: the new
    cases must not be written while the call still reads the old ones."""
    import torch

    from mapol_b200._lib import lib

    buses, branches, cases = m.workload("cfg1_300bus")
    with m.PowerFlow(buses, branches) as pf:
        pf.set_cases(cases[:64])
        flat = np.zeros((64, len(buses)), complex)
        flat[:] = buses["vm"] * np.exp(1j * buses["va"])
        v = _dev(flat)
        ref = torch.zeros(64, dtype=torch.float64, device="cuda")
        assert lib().mpf_mismatch(pf._h, v.data_ptr(), ref.data_ptr(), None) == 0
        torch.cuda.synchronize()
        s = torch.cuda.Stream()
        got = torch.zeros(64, dtype=torch.float64, device="cuda")
        with torch.cuda.stream(s):
            torch.cuda._sleep(2_000_000)  # keep the stream busy so the call is still queued
        assert lib().mpf_mismatch_noalloc(pf._h, v.data_ptr(), got.data_ptr(), s.cuda_stream) == 0
        pf.set_cases(cases[64:128])
        torch.cuda.synchronize()
        np.testing.assert_allclose(got.cpu().numpy(), ref.cpu().numpy(), rtol=1e-12, atol=0.0)
