"""Grids of uneven size in one batch (mapol_b200.MultiGrid, mpf_set_cases_islands):
the grids become islands of one handle and every stage runs all of their cases in
the same launches.  Each grid's results must equal the oracle run on that grid
alone, with the bar of the single-grid parity tests (identical flags, identical FP64
iteration counts, at most one extra in mixed precision, |dV| < 1e-8)."""
import os

import numpy as np
import pytest

import mapol_b200 as m
from oracle import oracle

from .parity import TIGHT_TOL, compare

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
V_TOL = 1e-8


def _compare(res, ref, max_extra_iter=0, tight=None):
    return compare(res, ref, max_extra_iter, V_TOL, tight)


@pytest.fixture(scope="module")
def cfg2(gpu):
    """The config-2 grids (118 / 1354 / 2869 buses), a slice of each one's N-1 set."""
    grids, cases = m.grid.workload_set("cfg2")
    return grids, [cs[:n] for cs, n in zip(cases, (60, 90, 70))]


@pytest.mark.parametrize("alg", [m.NR, m.FDXB])
def test_three_grids_one_batch_match_oracle(cfg2, alg):
    grids, cases = cfg2
    refs = [oracle.runpf(b, br, cs, alg=alg) for (b, br), cs in zip(grids, cases)]
    with m.MultiGrid(grids) as mg:
        mg.set_cases(cases)
        for prec in (m.FP64, m.MIXED):
            mg.solve(alg, prec)
            for res, ref, (b, br), cs in zip(mg.results(), refs, grids, cases):
                tight = lambda idx, b=b, br=br, cs=cs: oracle.runpf(b, br, [cs[i] for i in idx], alg=alg,
                                                                    tol=TIGHT_TOL)
                _compare(res, ref, 0 if prec == m.FP64 else 1, tight)


def test_config2_full_size_matches_oracle(gpu):
    """Config 2 at its stated size: the 118-, 1354- and 2869-bus grids with 167 / 400 /
    400 N-1 cases in one batch (167 = every non-bridge branch of the 118-bus grid, of
    the 200 asked for), Newton-Raphson in both precisions, each grid against the oracle."""
    grids, cases = m.grid.workload_set("cfg2")
    assert [len(c) for c in cases] == [167, 400, 400]
    refs = [oracle.runpf(b, br, cs, alg=m.NR) for (b, br), cs in zip(grids, cases)]
    with m.MultiGrid(grids) as mg:
        mg.set_cases(cases)
        for prec in (m.FP64, m.MIXED):
            mg.solve(m.NR, prec)
            for res, ref, (b, br), cs in zip(mg.results(), refs, grids, cases):
                tight = lambda idx, b=b, br=br, cs=cs: oracle.runpf(b, br, [cs[i] for i in idx], alg=m.NR,
                                                                    tol=TIGHT_TOL)
                conv = _compare(res, ref, 0 if prec == m.FP64 else 1, tight)
                assert conv.all()


def test_one_batch_launches_like_its_largest_grid(cfg2):
    """The stages of all grids share launches: a three-grid solve launches about as
    many kernels as its largest grid alone, not the sum of the three.  The fixed
    kernel rule is used (no autotuning): the tuner may fold the backward solve's
    near-root levels into one launch for one batch and not for another, which changes
    launch counts without changing what this test is about."""
    grids, cases = cfg2
    launches = []
    for (b, br), cs in zip(grids, cases):
        with m.PowerFlow(b, br, autotune=0) as pf:
            pf.set_cases(cs)
            pf.solve(m.NR, m.MIXED)
            launches.append(pf.timing()["launches"])
    with m.MultiGrid(grids, autotune=0) as mg:
        mg.set_cases(cases)
        mg.solve(m.NR, m.MIXED)
        joint = mg.timing()["launches"]
    assert joint < sum(launches), (joint, launches)
    assert joint <= 1.15 * max(launches), (joint, launches)


def test_real_grids_with_base_cases_and_load_scenarios(gpu):
    """IEEE 118- and 300-bus grids in one batch: base cases (island given explicitly),
    N-1 cases and per-case loads of one grid; branch flows per case as the oracle's."""
    g = np.load(os.path.join(HERE, "golden", "matpower_cases.npz"))
    grids = [(g["case118_buses"], g["case118_branches"]), (g["case300_buses"], g["case300_branches"])]
    cases = [[[]] * 3 + m.n1_cases(grids[0][1], len(grids[0][0]), 25, 2),
             [[]] * 2 + m.n1_cases(grids[1][1], len(grids[1][0]), 30, 3)]
    sb0 = m.load_scenarios(grids[0][0], len(cases[0]), 0.02, 4)
    refs = [oracle.runpf(grids[0][0], grids[0][1], cases[0], alg=m.NR, sbus=sb0),
            oracle.runpf(grids[1][0], grids[1][1], cases[1], alg=m.NR)]
    with m.MultiGrid(grids) as mg:
        mg.set_cases(cases, sbus_per_grid=[sb0, None])
        mg.solve(m.NR, m.FP64)
        res = mg.results()
        for r, ref in zip(res, refs):
            _compare(r, ref)
        ploss = mg.pf.branch_flows()["ploss"]
    row = 0
    for k, ((b, br), cs) in enumerate(zip(grids, cases)):
        for c, out in enumerate(cs):
            if res[k].converged[c]:
                bb = b.copy()
                if k == 0:
                    bb["p"], bb["q"] = sb0[c, :, 0], sb0[c, :, 1]
                assert abs(ploss[row + c] - oracle.loss(bb, br, res[k].v[c], out)) < 1e-9
        row += len(cs)


def test_island_inputs_are_checked(gpu):
    g = np.load(os.path.join(HERE, "golden", "matpower_cases.npz"))
    b1, br1 = g["case14_buses"], g["case14_branches"]
    b2, br2 = g["case30_buses"], g["case30_branches"]
    with m.MultiGrid([(b1, br1), (b2, br2)]) as mg:
        pf = mg.pf
        with pytest.raises(m.MpfError):
            pf.set_cases([[]])                      # base case: island unknown
        with pytest.raises(m.MpfError):
            pf.set_cases([[]], islands=[2])         # no island 2
        with pytest.raises(m.MpfError):
            pf.set_cases([[len(br1)]], islands=[0])  # outage in the other island
        pf.set_cases([[len(br1) + 3], [5]])         # islands from the outages
        pf.solve(m.NR, m.FP64)
        assert pf.results().converged.all()
    # the engine rejects an island without a slack bus
    b3 = b2.copy()
    b3["type"][b3["type"] == 3] = 2
    br3 = br2.copy()
    br3["from"] += len(b1)
    br3["to"] += len(b1)
    with pytest.raises(m.MpfError):
        m.PowerFlow(np.concatenate([b1, b3]), np.concatenate([br1, br3]))


def test_device_loop_equals_host_loop(cfg2):
    """The whole Newton loop as one CUDA graph (use_graph = 2, as the config-2 bench runs
    it) gives each grid of the batch the host-read loop's results bit for bit."""
    grids, cases = cfg2
    out = []
    for use_graph in (1, 2):
        with m.MultiGrid(grids, use_graph=use_graph) as mg:
            mg.set_cases(cases)
            r = []
            for prec in (m.FP64, m.MIXED):
                mg.solve(m.NR, prec)
                r.append([(x.v.copy(), x.iterations.copy(), x.status.copy()) for x in mg.results()])
            out.append(r)
    for pa, pb in zip(*out):
        for ga, gb in zip(pa, pb):
            for a, b in zip(ga, gb):
                assert np.array_equal(a, b)
