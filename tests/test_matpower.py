"""MATPOWER loader (mapol_b200.matpower) and an external pin of the oracle: from a
flat start it reproduces the solved state stored in the reference's bundled
case14.m (the IEEE 14-bus published solution) to the rounding of that file
(|V| to 3 decimals, angles to 2 decimals of a degree)."""
import os

import numpy as np
import pytest

from mapol_b200.matpower import load_matpower
from oracle import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "matpower_cases.npz")
REF = "/root/reference/src/datasets"


@pytest.fixture(scope="module", autouse=True)
def _built(built):
    return built


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference datasets not present")
@pytest.mark.parametrize("name", ["case14", "case30", "case118", "case300"])
def test_fixture_is_the_loader_output(name):
    g = np.load(FIX)
    b, br, rt = load_matpower(os.path.join(REF, name + ".m"))
    assert b.tobytes() == g[name + "_buses"].tobytes()
    assert br.tobytes() == g[name + "_branches"].tobytes()
    assert np.array_equal(rt, g[name + "_rating"])


def test_case14_flat_start_reproduces_published_solution():
    g = np.load(FIX)
    b = g["case14_buses"].copy()
    br = g["case14_branches"]
    stored_vm, stored_va = b["vm"].copy(), np.degrees(b["va"])
    b["va"] = 0.0
    b["vm"][b["type"] == 1] = 1.0
    r = oracle.runpf(b, br, [[]], alg=0)
    assert r["converged"][0] and r["iterations"][0] == 4
    v = r["v"][0]
    assert np.abs(np.abs(v) - stored_vm).max() < 1.5e-3
    assert np.abs(np.degrees(np.angle(v)) - stored_va).max() < 0.02


def test_loader_semantics():
    g = np.load(FIX)
    b = g["case14_buses"]
    br = g["case14_branches"]
    # bus 2 (index 1): Pd 21.7, Qd 12.7, generator Pg 40, Qg 42.4 on 100 MVA
    assert abs(b["p"][1] - (40 - 21.7) / 100) < 1e-12 and abs(b["q"][1] - (42.4 - 12.7) / 100) < 1e-12
    assert abs(b["bsh"][8] - 0.19) < 1e-12  # bus 9 Bs = 19 MVAr
    assert (b["type"] == 3).sum() == 1
    assert br["tap"][br["tap"] != 0].min() > 0.9
    assert len(br) == 20 and (br["status"] == 1).all()
