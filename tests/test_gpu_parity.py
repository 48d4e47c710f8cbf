"""Parity of the CUDA path (through the C-ABI) with the CPU oracle.

Tolerances: converged cases must satisfy the reference's own criterion
max |F| < 1e-8 p.u. (newtonpf.h:394,518); flags must match exactly; plain FP64
Newton iteration counts must match exactly and mixed precision may take at most
one more; voltages must agree with the oracle to 1e-8 p.u. (both are converged
to < 1e-8 mismatch, so agreement is bounded by the conditioning of J).
"""
import numpy as np
import pytest

import mapol_b200 as m
from oracle import oracle

from .parity import TIGHT_TOL, compare

pytestmark = pytest.mark.gpu

V_TOL = 1e-8


def _oracle(buses, branches, cases, alg, sbus=None, tol=1e-8):
    return oracle.runpf(buses, branches, cases, alg=alg, sbus=sbus, tol=tol)


def _tight(buses, branches, cases, alg, sbus=None):
    """The oracle on a subset of the cases, to max |F| < TIGHT_TOL."""
    def run(idx):
        sub = None if sbus is None else sbus[idx]
        return _oracle(buses, branches, [cases[i] for i in idx], alg, sub, tol=TIGHT_TOL)
    return run


def _compare(res, ref, max_extra_iter=0, v_tol=V_TOL, tight=None):
    return compare(res, ref, max_extra_iter, v_tol, tight)


@pytest.mark.parametrize("name", ["cfg0_30bus", "cfg1_300bus"])
def test_nr_fp64_matches_oracle(gpu, name):
    buses, branches, cases = m.workload(name)
    ref = _oracle(buses, branches, cases, m.NR)
    with m.PowerFlow(buses, branches) as pf:
        pf.set_cases(cases)
        pf.solve(m.NR, m.FP64)
        res = pf.results()
    conv = _compare(res, ref)
    assert conv.mean() > 0.9


@pytest.mark.parametrize("alg", [m.FDXB, m.FDBX])
@pytest.mark.parametrize("name", ["cfg0_30bus", "cfg1_300bus"])
def test_fd_fp64_matches_oracle(gpu, name, alg):
    buses, branches, cases = m.workload(name)
    ref = _oracle(buses, branches, cases, alg)
    with m.PowerFlow(buses, branches) as pf:
        pf.set_cases(cases)
        pf.solve(alg, m.FP64)
        res = pf.results()
    _compare(res, ref)  # measured: |V - V_oracle| <= 2.4e-13 on these workloads


@pytest.mark.parametrize("name", ["cfg0_30bus", "cfg1_300bus"])
def test_nr_mixed_at_most_one_extra_iteration(gpu, name):
    buses, branches, cases = m.workload(name)
    ref = _oracle(buses, branches, cases, m.NR)
    with m.PowerFlow(buses, branches) as pf:
        pf.set_cases(cases)
        pf.solve(m.NR, m.MIXED)
        res = pf.results()
    _compare(res, ref, max_extra_iter=1, tight=_tight(buses, branches, cases, m.NR))


def test_runpf_host_end_to_end(gpu):
    buses, branches, cases = m.workload("cfg1_300bus")
    ref = _oracle(buses, branches, cases, m.NR)
    pf = m.hybrid_init(buses, branches, len(cases), m.NR)
    res = m.hybrid_runpf(pf, cases)
    m.hybrid_free(pf)
    _compare(res, ref)


def test_runpf_host_device_loop_equals_host_loop(gpu):
    """mpf_runpf_host (case lists in from host memory, results out to host memory)
    through the device-side Newton loop (use_graph = 2), as the bench's end-to-end figure
    runs it, equals the host-read loop bit for bit, in both precisions."""
    from mapol_b200._lib import lib, ptr
    from mapol_b200.grid import cases_to_offsets

    buses, branches, cases = m.workload("cfg1_300bus")
    offs, flat = cases_to_offsets(cases)
    n, nb = len(cases), len(buses)
    out = {}
    for use_graph in (1, 2):
        with m.PowerFlow(buses, branches, use_graph=use_graph) as pf:
            for prec in (m.MIXED, m.FP64):
                v = np.zeros((n, nb, 2))
                it = np.zeros(n, np.int32)
                st = np.zeros(n, np.uint8)
                mm = np.zeros(n)
                assert lib().mpf_runpf_host(pf._h, m.NR, prec, n, ptr(offs), ptr(flat), None, ptr(v), ptr(it),
                                            ptr(st), ptr(mm)) == 0
                out[use_graph, prec] = (v, it, st, mm)
    for prec in (m.MIXED, m.FP64):
        assert (out[2, prec][2] == m.runpf.CONVERGED).sum() > 0.9 * n
        for a, b in zip(out[1, prec], out[2, prec]):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("n_bus,n_branch,n_pv,n_out", [(118, 179, 53, 64), (1354, 1991, 259, 40)])
def test_uneven_sizes_match_oracle(gpu, n_bus, n_branch, n_pv, n_out):
    buses, branches = m.synth_grid(n_bus, n_branch, n_pv, 0.1, seed=2)
    cases = m.n1_cases(branches, n_bus, n_out, 5, with_base=True)
    ref = _oracle(buses, branches, cases, m.NR)
    with m.PowerFlow(buses, branches) as pf:
        pf.set_cases(cases)
        pf.solve(m.NR, m.FP64)
        _compare(pf.results(), ref)


def test_n2_outages_and_load_scenarios(gpu):
    buses, branches = m.synth_grid(300, 411, 69, 0.1, seed=4)
    out = m.select_outages(branches, 300, 40, 9)
    cases = [[int(out[2 * k]), int(out[2 * k + 1])] for k in range(20)] + [[]] * 4
    sbus = m.load_scenarios(buses, len(cases), 0.05, 3)
    ref = _oracle(buses, branches, cases, m.NR, sbus=sbus)
    with m.PowerFlow(buses, branches) as pf:
        pf.set_cases(cases, sbus=sbus)
        pf.solve(m.NR, m.FP64)
        _compare(pf.results(), ref)


def test_batch_not_multiple_of_32_and_repeated_solves(gpu):
    buses, branches, cases = m.workload("cfg1_300bus")
    cases = cases[:45]
    ref = _oracle(buses, branches, cases, m.NR)
    with m.PowerFlow(buses, branches) as pf:
        pf.set_cases(cases)
        for alg in (m.NR, m.FDXB, m.NR):
            pf.solve(alg, m.FP64)
        _compare(pf.results(), ref)


def test_bridge_outage_is_reported_not_converged(gpu):
    buses, branches = m.synth_grid(300, 411, 69, 0.1, seed=1)
    bridges = np.where(m.find_bridges(branches, 300))[0]
    cases = [[int(bridges[0])], []]
    ref = _oracle(buses, branches, cases, m.NR)
    with m.PowerFlow(buses, branches) as pf:
        pf.set_cases(cases)
        pf.solve(m.NR, m.FP64)
        res = pf.results()
    assert res.status[1] == m.runpf.CONVERGED
    assert res.status[0] != m.runpf.CONVERGED
    assert not ref["converged"][0]


def test_bad_inputs_raise_not_crash(gpu):
    buses, branches = m.synth_grid(30, 41, 5)
    with m.PowerFlow(buses, branches) as pf:
        with pytest.raises(m.MpfError):
            pf.solve(m.NR, m.FP64)  # before set_cases
        with pytest.raises(m.MpfError):
            pf.set_cases([[1000]])
        with pytest.raises(m.MpfError):
            pf.set_cases([[1, 1]])
        with pytest.raises(m.MpfError):
            pf.set_cases([[1, 2, 3, 4, 5]])
        pf.set_cases([[]])
        with pytest.raises(m.MpfError):
            pf.solve(7, m.FP64)
    bad = buses.copy()
    bad["type"][bad["type"] == 3] = 1
    with pytest.raises(m.MpfError):
        m.PowerFlow(bad, branches)


def test_full_size_9241_bus_all_cases_match_oracle(gpu):
    """The headline workload at full size: all 1000 N-1 cases of the 9241-bus grid,
    in both precisions, against the oracle on every case.  Flags identical, FP64
    iteration counts identical (mixed at most one more), |V - V_oracle| < 1e-8 p.u.
    (a mixed case that took the extra iteration against the oracle run to 1e-11)."""
    buses, branches, cases = m.workload("cfg3_9241bus")
    assert len(cases) == 1000
    with m.PowerFlow(buses, branches) as pf:
        pf.set_cases(cases)
        pf.solve(m.NR, m.FP64)
        res = pf.results()
        pf.solve(m.NR, m.MIXED)
        res_mixed = pf.results()
    ref = _oracle(buses, branches, cases, m.NR)
    conv = _compare(res, ref)
    _compare(res_mixed, ref, max_extra_iter=1, tight=_tight(buses, branches, cases, m.NR))
    assert conv.all()  # every case of this workload has a solution (non-bridge outages)


def test_mismatch_entry_point_matches_solve_and_oracle(gpu):
    """mpf_mismatch at the solved voltages reproduces the solve's own final max |F| (both
    round-off there, so to 1e-13 absolute: the solve's fused mismatch-Jacobian pass and
    this evaluation kernel order their operations differently) and, at an unconverged
    point, the oracle's mismatch to 1e-12 relative."""
    import torch

    from mapol_b200._lib import lib

    buses, branches, cases = m.workload("cfg1_300bus")
    cases = cases[:40]
    with m.PowerFlow(buses, branches) as pf:
        pf.set_cases(cases)
        pf.solve(m.NR, m.FP64)
        res = pf.results()
        v = torch.from_numpy(np.stack([res.v.real, res.v.imag], -1)).cuda()
        out = torch.zeros(len(cases), dtype=torch.float64, device="cuda")
        for _ in range(2):
            assert lib().mpf_mismatch(pf._h, v.data_ptr(), out.data_ptr(), None) == 0
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            np.testing.assert_allclose(got, res.max_mis, rtol=1e-6, atol=1e-13)
            assert (got < 1e-8).all()
        # an unconverged point: the flat start
        flat = np.zeros((len(cases), len(buses)), complex)
        flat[:] = buses["vm"] * np.exp(1j * buses["va"])
        vf = torch.from_numpy(np.stack([flat.real, flat.imag], -1)).cuda()
        assert lib().mpf_mismatch(pf._h, vf.data_ptr(), out.data_ptr(), None) == 0
        torch.cuda.synchronize()
        got = out.cpu().numpy()
    for k in (0, 7, 31):
        _, _, err = oracle.nr_system(buses, branches, flat[k], cases[k])
        assert abs(got[k] - err) <= 1e-12 * max(1.0, err)


def test_graph_and_direct_launches_agree(gpu):
    """The graph-captured iteration (default), the whole Newton loop as one graph with a
    device-side while node (use_graph = 2) and direct launches give identical results,
    and replays after set_cases with a different batch size rebuild the graphs."""
    buses, branches, cases = m.workload("cfg1_300bus")
    out = []
    for use_graph in (1, 0, 2):
        pf = m.PowerFlow(buses, branches)
        pf_opt = pf  # noqa: F841
        pf.close()
        from mapol_b200 import _types as T
        from mapol_b200._lib import lib, ptr
        import ctypes

        opt = T.Options()
        lib().mpf_default_options(ctypes.byref(opt))
        opt.use_graph = use_graph
        h = ctypes.c_void_p()
        assert lib().mpf_create(ptr(buses), len(buses), ptr(branches), len(branches), ctypes.byref(opt),
                                ctypes.byref(h)) == 0
        res = []
        for n in (200, 45, 200):
            from mapol_b200.grid import cases_to_offsets

            offs, flat = cases_to_offsets(cases[:n])
            assert lib().mpf_set_cases(h, n, ptr(offs), ptr(flat), None) == 0
            for prec in (m.FP64, m.MIXED):
                assert lib().mpf_solve(h, m.NR, prec, None) == 0
                v = np.zeros((n, len(buses), 2))
                it = np.zeros(n, np.int32)
                assert lib().mpf_get_results(h, ptr(v), ptr(it), None, None) == 0
                res.append((v.copy(), it.copy()))
        lib().mpf_destroy(h)
        out.append(res)
    for other in out[1:]:
        for (va, ia), (vb, ib) in zip(out[0], other):
            assert np.array_equal(ia, ib)
            assert np.array_equal(va, vb)


def test_device_loop_iteration_limit_and_q_limit_rounds(gpu):
    """The device-side Newton loop stops at max_it_nr like the host loop (MAX_ITER per
    case, same iteration counts) and runs again for each reactive-limit round."""
    buses, branches, cases = m.workload("cfg1_300bus")
    cases = [[]] + cases[:60]
    rng = np.random.default_rng(5)
    pv = np.where(buses["type"] == 2)[0]
    qmin = np.full(len(buses), -np.inf)
    qmax = np.full(len(buses), np.inf)
    qmax[rng.choice(pv, len(pv) // 4, replace=False)] = 0.0
    for max_it in (2, 10):
        got = []
        for use_graph in (1, 2):
            with m.PowerFlow(buses, branches, use_graph=use_graph, max_it_nr=max_it) as pf:
                if max_it == 10:
                    pf.set_q_limits(qmin, qmax)  # before the cases: limits reset them
                pf.set_cases(cases)
                r = []
                for prec in (m.FP64, m.MIXED):
                    pf.solve(m.NR, prec)
                    res = pf.results()
                    r.append((res.status.copy(), res.iterations.copy(), res.v.copy(), pf.bus_types().copy()
                              if max_it == 10 else None))
                got.append(r)
        for (sa, ia, va, ta), (sb, ib, vb, tb) in zip(*got):
            assert np.array_equal(sa, sb) and np.array_equal(ia, ib) and np.array_equal(va, vb)
            if ta is not None:
                assert np.array_equal(ta, tb)
        if max_it == 2:
            from mapol_b200 import _types as T

            assert (got[1][0][0] == T.CASE_MAX_ITER).any()
        else:
            # some cases switched PV buses to PQ (a second Newton run in the same solve)
            assert ((got[1][0][3] == 1).sum(axis=1) > (buses["type"] == 1).sum()).any()


def test_branch_flows_loss_and_overload_match_oracle(gpu):
    buses, branches, cases = m.workload("cfg1_300bus")
    cases = cases[:40] + [[]]
    with m.PowerFlow(buses, branches) as pf:
        pf.set_cases(cases)
        pf.solve(m.NR, m.FP64)
        res = pf.results()
        fl = pf.branch_flows(flows=True)
        rating = 1.2 * np.abs(fl["sf"][-1])  # base case flows
        pf.set_ratings(rating)
        fl2 = pf.branch_flows()
        fit = pf.fitness(res)
    np.testing.assert_allclose(fl["ploss"], fl2["ploss"], rtol=1e-12, atol=0)
    for k in (0, 5, 17, 40):
        ref = oracle.loss(buses, branches, res.v[k], cases[k])
        assert abs(fl["ploss"][k] - ref) <= 1e-10 * max(1.0, abs(ref))
    # overload from the flows themselves, and outaged branches carry nothing
    ex = np.maximum(np.abs(fl["sf"]) - 0.9 * rating, 0.0)
    np.testing.assert_allclose(fl2["overload"], (ex ** 2).sum(1), rtol=1e-10, atol=1e-14)
    for k in range(40):
        assert fl["sf"][k, cases[k][0]] == 0 and fl["st"][k, cases[k][0]] == 0
    assert (fl2["overload"][:40] > 0).any()
    # per-case sums are accumulated with atomics: equal up to summation order
    np.testing.assert_allclose(fit, fl["ploss"], rtol=1e-12, atol=0)


@pytest.mark.parametrize("name", ["case118", "case300"])
def test_real_matpower_grids_n1_match_oracle(gpu, name):
    """The reference's bundled IEEE 118 / 300-bus cases (fixture converted from its
    datasets), base + 40 N-1 outages, solved from the stored start point."""
    import os

    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "matpower_cases.npz"))
    buses, branches = g[name + "_buses"], g[name + "_branches"]
    cases = m.n1_cases(branches, len(buses), 40, 3, with_base=True)
    ref = _oracle(buses, branches, cases, m.NR)
    with m.PowerFlow(buses, branches) as pf:
        pf.set_cases(cases)
        pf.solve(m.NR, m.FP64)
        res = pf.results()
        pf.solve(m.NR, m.MIXED)
        res32 = pf.results()
    _compare(res, ref)
    _compare(res32, ref, max_extra_iter=1, tight=_tight(buses, branches, cases, m.NR))
