"""Grids and case batches: seeded synthetic grids, bridges, N-1 outage selection,
load scenarios (all computed by libmpf.so so every machine gets the same inputs).
"""
import ctypes

import numpy as np

from . import _types as T
from ._lib import MpfError, lib, ptr


def synth_grid(n_bus, n_branch, n_pv, tap_fraction=0.0, seed=1, topology=0, **overrides):
    """Seeded synthetic grid (include/mpf.h mpf_synth_grid).  Returns (buses, branches)
    as numpy arrays of BUS_DTYPE / BRANCH_DTYPE.  overrides set other mpf_synth_params
    fields (r_lo, pload_hi, loading, ...)."""
    p = T.SynthParams()
    lib().mpf_synth_default(ctypes.byref(p))
    p.n_bus, p.n_branch, p.n_pv = n_bus, n_branch, n_pv
    p.tap_fraction, p.seed, p.topology = tap_fraction, seed, topology
    for k, v in overrides.items():
        setattr(p, k, v)
    buses = np.zeros(n_bus, T.BUS_DTYPE)
    branches = np.zeros(n_branch, T.BRANCH_DTYPE)
    rc = lib().mpf_synth_grid(ctypes.byref(p), ptr(buses), ptr(branches))
    if rc != 0:
        raise MpfError(rc, "mpf_synth_grid rejected the parameters")
    return buses, branches


def find_bridges(branches, n_bus):
    out = np.zeros(len(branches), np.uint8)
    rc = lib().mpf_find_bridges(ptr(branches), len(branches), n_bus, ptr(out))
    if rc != 0:
        raise MpfError(rc, "mpf_find_bridges failed")
    return out.astype(bool)


def select_outages(branches, n_bus, n_out, seed):
    out = np.zeros(n_out, np.int32)
    rc = lib().mpf_select_outages(ptr(branches), len(branches), n_bus, n_out, seed, ptr(out))
    if rc != 0:
        raise MpfError(rc, "not enough non-bridge branches for the requested outages")
    return out


def load_scenarios(buses, n_cases, sigma, seed):
    sbus = np.zeros((n_cases, len(buses), 2))
    rc = lib().mpf_synth_load_scenarios(ptr(buses), len(buses), n_cases, sigma, seed, ptr(sbus))
    if rc != 0:
        raise MpfError(rc, "mpf_synth_load_scenarios failed")
    return sbus


def cases_to_offsets(cases):
    """List of outage lists -> (offsets[n+1], branches[]) int32 arrays."""
    offs = np.zeros(len(cases) + 1, np.int32)
    flat = []
    for i, c in enumerate(cases):
        offs[i + 1] = offs[i] + len(c)
        flat.extend(int(b) for b in c)
    return offs, np.asarray(flat + [0], np.int32)


def n1_cases(branches, n_bus, n_out, seed, with_base=False):
    out = select_outages(branches, n_bus, n_out, seed)
    cases = [[int(b)] for b in out]
    return ([[]] if with_base else []) + cases


# The synthetic workloads (sizes of the reference's benchmark grids, README.md:3).
# loading = 0.2 everywhere (see mpf_synth_default).
WORKLOADS = {
    "cfg0_30bus": dict(n_bus=30, n_branch=41, n_pv=5, tap_fraction=0.0, n_out=10, with_base=True),
    "cfg1_300bus": dict(n_bus=300, n_branch=411, n_pv=69, tap_fraction=0.10, n_out=200, with_base=False),
    # 200 outages are asked for, but the 179-branch grid has 167 non-bridge branches:
    # its N-1 set is all of them
    "cfg2_118bus": dict(n_bus=118, n_branch=179, n_pv=53, tap_fraction=0.10, n_out=200, with_base=False),
    "cfg2_1354bus": dict(n_bus=1354, n_branch=1991, n_pv=259, tap_fraction=0.10, n_out=400, with_base=False),
    "cfg2_2869bus": dict(n_bus=2869, n_branch=4582, n_pv=509, tap_fraction=0.10, n_out=400, with_base=False),
    "cfg3_9241bus": dict(n_bus=9241, n_branch=16049, n_pv=1445, tap_fraction=0.15, n_out=1000, with_base=False),
    "cfg4_1354bus": dict(n_bus=1354, n_branch=1991, n_pv=259, tap_fraction=0.10, n_out=0, with_base=False),
    # stress row: the same sizes with uniform-random extra branches (topology 1), a
    # densely meshed grid whose fronts reach 337 rows (large-front kernel)
    "stress_uniform_1354bus": dict(n_bus=1354, n_branch=1991, n_pv=259, tap_fraction=0.10, n_out=1000,
                                   with_base=False, topology=1),
}


# Grids of uneven size solved as one batch (MultiGrid): config 2.
WORKLOAD_SETS = {"cfg2": ["cfg2_118bus", "cfg2_1354bus", "cfg2_2869bus"]}


def workload(name, seed=1, outage_seed=7):
    """(buses, branches, cases) of a named workload.  The N-1 set holds n_out
    non-bridge outages, or every non-bridge branch when the grid has fewer."""
    w = WORKLOADS[name]
    buses, branches = synth_grid(w["n_bus"], w["n_branch"], w["n_pv"], w["tap_fraction"], seed=seed,
                                 topology=w.get("topology", 0))
    n_out = w["n_out"]
    if n_out:
        n_out = min(n_out, int((find_bridges(branches, w["n_bus"]) == 0).sum()))
    cases = n1_cases(branches, w["n_bus"], n_out, outage_seed, w["with_base"]) if n_out else [[]]
    return buses, branches, cases


def workload_set(name, seed=1, outage_seed=7):
    """(grids, cases_per_grid) of a named set of grids solved as one batch."""
    grids, cases = [], []
    for wname in WORKLOAD_SETS[name]:
        b, br, cs = workload(wname, seed, outage_seed)
        grids.append((b, br))
        cases.append(cs)
    return grids, cases
