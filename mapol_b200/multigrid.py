"""Grids of uneven size in one batch.

The reference solves one grid per process (hybrid_init, runpf.h:795, keeps it in
globals).  Here several grids share one handle as the islands of a single
concatenated grid: their Jacobians form a block-diagonal system whose supernodes
each belong to one island, every case belongs to one grid, and each Newton or
fast-decoupled stage runs the cases of all grids in the same kernel launches
(rows, branches and supernodes of the other grids are skipped per case group).
"""
import numpy as np

from . import _types as T
from .runpf import FP64, NR, PowerFlow, Results


class MultiGrid:
    """grids: sequence of (buses, branches), each with exactly one slack bus."""

    def __init__(self, grids, **kw):
        bus_off, br_off = [0], [0]
        bs, brs = [], []
        for buses, branches in grids:
            b = np.array(buses, dtype=T.BUS_DTYPE)
            br = np.array(branches, dtype=T.BRANCH_DTYPE)
            if int((b["type"] == T.BUS_SLACK).sum()) != 1:
                raise ValueError("each grid needs exactly one slack bus")
            br["from"] += bus_off[-1]
            br["to"] += bus_off[-1]
            bs.append(b)
            brs.append(br)
            bus_off.append(bus_off[-1] + len(b))
            br_off.append(br_off[-1] + len(br))
        self.bus_off, self.br_off = bus_off, br_off
        self.n_grids = len(bs)
        self.pf = PowerFlow(np.concatenate(bs), np.concatenate(brs), **kw)

    def close(self):
        self.pf.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_cases(self, cases_per_grid, sbus_per_grid=None):
        """cases_per_grid[k]: outage lists of grid k in its own branch numbering;
        sbus_per_grid[k]: None or (n_cases_k, n_bus_k, 2) injections of grid k."""
        if len(cases_per_grid) != self.n_grids:
            raise ValueError(f"expected case lists for {self.n_grids} grids")
        cases, islands = [], []
        for k, cs in enumerate(cases_per_grid):
            cases += [[int(b) + self.br_off[k] for b in c] for c in cs]
            islands += [k] * len(cs)
        sbus = None
        if sbus_per_grid is not None and any(s is not None for s in sbus_per_grid):
            base = np.stack([self.pf.buses["p"], self.pf.buses["q"]], -1)
            sbus = np.repeat(base[None], len(cases), 0)
            row = 0
            for k, cs in enumerate(cases_per_grid):
                if sbus_per_grid[k] is not None:
                    sbus[row:row + len(cs), self.bus_off[k]:self.bus_off[k + 1]] = sbus_per_grid[k]
                row += len(cs)
        self.counts = [len(cs) for cs in cases_per_grid]
        self.pf.set_cases(cases, sbus=sbus, islands=islands)

    def solve(self, alg=NR, precision=FP64):
        self.pf.solve(alg, precision)

    def results(self):
        """One Results per grid, voltages over that grid's buses only."""
        r = self.pf.results()
        out, row = [], 0
        for k, n in enumerate(self.counts):
            s = slice(row, row + n)
            out.append(Results(r.v[s, self.bus_off[k]:self.bus_off[k + 1]], r.iterations[s], r.status[s],
                               r.max_mis[s]))
            row += n
        return out

    def timing(self):
        return self.pf.timing()
