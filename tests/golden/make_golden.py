"""Generates tests/golden/oracle_cfg0_cfg1.npz: the synthetic grids of the two small
workloads (as generated by libmpf's seeded generator) and the oracle's NR / FDXB /
FDBX results on their first cases.  Run from the repository root:
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import mapol_b200 as m  # noqa: E402
from oracle import oracle  # noqa: E402


def main():
    out = {}
    for name, n in (("cfg0_30bus", 11), ("cfg1_300bus", 24)):
        buses, branches, cases = m.workload(name)
        out[f"{name}_buses"] = buses
        out[f"{name}_branches"] = branches
        out[f"{name}_cases"] = np.array([c[0] if c else -1 for c in cases[:n]], np.int32)
        for alg, tag in ((m.NR, "nr"), (m.FDXB, "fdxb"), (m.FDBX, "fdbx")):
            r = oracle.runpf(buses, branches, cases[:n], alg=alg)
            out[f"{name}_{tag}_v"] = r["v"]
            out[f"{name}_{tag}_iterations"] = r["iterations"]
            out[f"{name}_{tag}_converged"] = r["converged"]
            out[f"{name}_{tag}_max_mis"] = r["max_mis"]
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "oracle_cfg0_cfg1.npz"), **out)


if __name__ == "__main__":
    main()
