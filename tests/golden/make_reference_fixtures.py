"""Writes tests/golden/reference_outputs.npz: outputs of the reference's OWN CPU
power-flow code (oracle/_ref/librefpf.so, built by `make -C oracle` from the reference's
sources) on its bundled MATPOWER cases (case14/30/118/300, base case + up to 20 N-1
outages each) and on the 30- and 300-bus synthetic workloads, for Newton-Raphson (its
Eigen SparseLU option) and fast-decoupled XB / BX (its DSS path).  The GPU tests compare
the engine with these where the reference tree is absent.  Run from the repository root
(needs the reference tree to build librefpf.so):
    python tests/golden/make_reference_fixtures.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import mapol_b200 as m  # noqa: E402
from oracle import refpf  # noqa: E402

ALGS = ((m.NR, "nr", refpf.SOLVER_EIGEN), (m.FDXB, "fdxb", refpf.SOLVER_DSS), (m.FDBX, "fdbx", refpf.SOLVER_DSS))


def grids():
    g = np.load(os.path.join(ROOT, "tests", "golden", "matpower_cases.npz"))
    for name in ("case14", "case30", "case118", "case300"):
        buses, branches = g[name + "_buses"], g[name + "_branches"]
        nnb = int((~m.find_bridges(branches, len(buses))).sum())
        yield name, buses, branches, m.n1_cases(branches, len(buses), min(20, nnb), 3, with_base=True), ALGS
    buses, branches, cases = m.workload("cfg0_30bus")
    yield "cfg0_30bus", buses, branches, cases, ALGS
    buses, branches, cases = m.workload("cfg1_300bus")
    yield "cfg1_300bus", buses, branches, cases[:32], ALGS[:1]  # NR: the reference's angle quirk


def main():
    out = {}
    for name, buses, branches, cases, algs in grids():
        out[f"{name}_buses"] = buses
        out[f"{name}_branches"] = branches
        out[f"{name}_outage"] = np.array([c[0] if c else -1 for c in cases], np.int32)
        for alg, tag, solver in algs:
            r = refpf.runpf(buses, branches, cases, alg=alg, solver=solver)
            out[f"{name}_{tag}_v"] = r["v"]
            out[f"{name}_{tag}_iterations"] = r["iterations"]
            out[f"{name}_{tag}_converged"] = r["converged"]
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "reference_outputs.npz"), **out)


if __name__ == "__main__":
    main()
