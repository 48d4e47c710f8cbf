"""Writes tests/golden/workload_cfg3_9241bus.npz: the 9241-bus synthetic grid and its
1000 N-1 outages exactly as libmpf's seeded generator makes them (mapol_b200.workload).
The CPU baseline arm of bench.py reads this file with numpy only, so that timing the
reference's CPU path never loads libmpf.so; tests/test_workload_fixture.py checks that
the generator still reproduces it byte for byte.  Run from the repository root:
    python tests/golden/make_workload_fixtures.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import mapol_b200 as m  # noqa: E402

NAMES = ("cfg3_9241bus",)


def path(name):
    return os.path.join(ROOT, "tests", "golden", f"workload_{name}.npz")


def main():
    for name in NAMES:
        buses, branches, cases = m.workload(name)
        assert all(len(c) == 1 for c in cases)
        np.savez_compressed(path(name), buses=buses, branches=branches,
                            outages=np.array([c[0] for c in cases], np.int32))


if __name__ == "__main__":
    main()
