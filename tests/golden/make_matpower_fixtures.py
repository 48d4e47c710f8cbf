"""Converts the reference's bundled MATPOWER cases (src/datasets/case14, 30, 57, 118, 300,
case1354pegase, case2869pegase, case9241pegase)
with mapol_b200.matpower.load_matpower (and the generators' Q limits, q_limits) into
tests/golden/matpower_cases.npz, so the GPU tests can run real grids where the reference
tree is absent.  Run from the repository root:
python tests/golden/make_matpower_fixtures.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from mapol_b200.matpower import load_matpower, q_limits  # noqa: E402

SRC = "/root/reference/src/datasets"


def main():
    out = {}
    for name in ("case14", "case30", "case57", "case118", "case300", "case1354pegase", "case2869pegase", "case9241pegase"):
        buses, branches, rating = load_matpower(os.path.join(SRC, name + ".m"))
        out[name + "_buses"] = buses
        out[name + "_branches"] = branches
        out[name + "_rating"] = rating
        out[name + "_qmin"], out[name + "_qmax"] = q_limits(os.path.join(SRC, name + ".m"))
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "matpower_cases.npz"), **out)


if __name__ == "__main__":
    main()
