"""The committed 9241-bus workload fixture (read by bench.py's CPU arms with numpy
only) is exactly what the seeded generator produces."""
import os

import numpy as np

import mapol_b200 as m

HERE = os.path.dirname(os.path.abspath(__file__))


def test_cfg3_fixture_matches_generator(built):
    g = np.load(os.path.join(HERE, "golden", "workload_cfg3_9241bus.npz"))
    buses, branches, cases = m.workload("cfg3_9241bus")
    assert g["buses"].tobytes() == buses.tobytes()
    assert g["branches"].tobytes() == branches.tobytes()
    assert g["outages"].tolist() == [c[0] for c in cases]
    assert len(cases) == 1000
