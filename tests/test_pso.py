"""The optimiser shim's host logic (no GPU): the structures main.cu:232-262 builds
from a grid and how bind() maps particle coordinates to engine controls, on the
reference's bundled IEEE 118-bus case."""
import os

import numpy as np

import mapol_b200 as m
from mapol_b200 import pso

HERE = os.path.dirname(os.path.abspath(__file__))


def _grid(name):
    g = np.load(os.path.join(HERE, "golden", "matpower_cases.npz"))
    return g[name + "_buses"], g[name + "_branches"]


def test_structures_follow_main():
    buses, branches = _grid("case118")
    est, bie, rie = pso.estruturas(buses, branches)
    pv = np.where(buses["type"] == m._types.BUS_PV)[0]
    shunt = np.where(buses["bsh"] > 0)[0]
    tapped = np.where(branches["tap"] > 0)[0]
    assert len(est) == len(pv) + len(shunt) + len(tapped)
    kinds = [e.tipo for e in est]
    assert kinds.count(pso.AVR) == len(pv) and kinds.count(pso.SHC) == len(shunt)
    assert kinds.count(pso.OLTC) == len(tapped)
    # buses first in bus order (AVR before SHC at one bus), then branches
    assert [e.id for e in est[:len(est) - len(tapped)]] == sorted(e.id for e in est[:len(est) - len(tapped)])
    for e in est:
        if e.tipo == pso.AVR:
            assert (e.min, e.max, e.qtd, e.default) == (0.9, 1.1, 0, buses["vm"][e.id])
        elif e.tipo == pso.SHC:
            assert (e.min, e.max, e.qtd, e.default) == (0.0, 0.18, 3, buses["bsh"][e.id])
        else:
            assert (e.min, e.max, e.qtd, e.default) == (0.9, 1.1, 20, branches["tap"][e.id])
    assert (rie[tapped] >= 0).all() and (rie[branches["tap"] == 0] == -1).all()


def test_bind_keeps_the_last_structure_of_a_bus():
    buses, branches = _grid("case118")
    est, bie, rie = pso.estruturas(buses, branches)
    both = [i for i in range(len(buses)) if buses["type"][i] == m._types.BUS_PV and buses["bsh"][i] > 0]
    controls, cols = pso.bind(est, bie, rie, branches)
    assert len(controls) == len(cols) == len(set(controls))
    for i in both:
        # main.cu binds the bus to its ShC structure, so its AVR coordinate is unused
        assert (m.CTRL_SHC, i) in controls and (m.CTRL_AVR, i) not in controls
    used = set(cols.tolist())
    unused = [k for k, e in enumerate(est) if k not in used]
    assert all(est[k].tipo == pso.AVR and est[k].id in both for k in unused)
    for (kind, idx), col in zip(controls, cols):
        assert est[col].id == idx and est[col].tipo == kind


def test_bind_on_a_synthetic_grid_without_shunts():
    buses, branches = m.synth_grid(300, 411, 69, 0.1, seed=1)
    est, bie, rie = pso.estruturas(buses, branches)
    controls, cols = pso.bind(est, bie, rie, branches)
    assert len(controls) == len(est)
    assert {k for k, _ in controls} == {m.CTRL_AVR, m.CTRL_OLTC}
