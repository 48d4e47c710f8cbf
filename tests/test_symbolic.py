"""CPU tests of the library's host side: exported C-ABI, seeded generator,
bridges, outage selection, load scenarios, and the multifrontal symbolic layer
(checked by a host emulation of the kernels' index arithmetic)."""
import hashlib
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

import mapol_b200 as m
from mapol_b200._lib import lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module", autouse=True)
def _built(built):
    return built


def test_library_exports_every_declared_entry_point():
    hdr = open(os.path.join(ROOT, "include", "mpf.h")).read()
    declared = set(re.findall(r"^\s*(?:int32_t|void|const char\*)\s+(mpf_\w+)\s*\(", hdr, re.M))
    assert len(declared) >= 20
    L = lib()
    missing = [d for d in declared if not hasattr(L, d)]
    assert not missing, missing
    assert L.mpf_abi_version() == 3


def test_generator_is_deterministic_and_pinned():
    a = m.synth_grid(30, 41, 5, seed=1)
    b = m.synth_grid(30, 41, 5, seed=1)
    c = m.synth_grid(30, 41, 5, seed=2)
    assert a[0].tobytes() == b[0].tobytes() and a[1].tobytes() == b[1].tobytes()
    assert a[1].tobytes() != c[1].tobytes()
    buses, branches = a
    assert (buses["type"] == 3).sum() == 1 and (buses["type"] == 2).sum() == 5
    assert len(branches) == 41 and (branches["status"] == 1).all()
    assert ((branches["r"] >= 0.01) & (branches["r"] <= 0.10)).all()
    xr = branches["x"] / branches["r"]
    assert ((xr >= 2) & (xr <= 6)).all()
    pq = buses["type"] == 1
    assert (-buses["p"][pq] <= 0.5 * 0.2 + 1e-15).all()
    gen = buses["p"][buses["type"] == 2].sum()
    assert abs(gen - 1.02 * -buses["p"][pq].sum()) < 1e-12
    h = hashlib.sha256(buses.tobytes() + branches.tobytes()).hexdigest()[:16]
    g = np.load(os.path.join(ROOT, "tests", "golden", "oracle_cfg0_cfg1.npz"))
    assert buses.tobytes() == g["cfg0_30bus_buses"].tobytes(), h


def _connected(nb, f, t):
    parent = list(range(nb))

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    for a, b in zip(f, t):
        parent[find(a)] = find(b)
    return len({find(i) for i in range(nb)}) == 1


def test_bridges_match_brute_force():
    buses, branches = m.synth_grid(300, 411, 69, 0.1, seed=3)
    br = m.find_bridges(branches, 300)
    f, t = branches["from"], branches["to"]
    for k in range(len(branches)):
        keep = np.arange(len(branches)) != k
        assert br[k] == (not _connected(300, f[keep], t[keep]))
    assert 0 < br.sum() < len(branches)


def test_outage_selection_distinct_non_bridges():
    buses, branches = m.synth_grid(300, 411, 69, 0.1, seed=3)
    out = m.select_outages(branches, 300, 100, 5)
    assert len(set(out.tolist())) == 100
    assert not m.find_bridges(branches, 300)[out].any()
    assert np.array_equal(out, m.select_outages(branches, 300, 100, 5))
    with pytest.raises(m.MpfError):
        m.select_outages(branches, 300, 411, 5)


def test_load_scenarios_scale_loads_only():
    buses, _ = m.synth_grid(1354, 1991, 259, 0.1)
    sb = m.load_scenarios(buses, 400, 0.05, 3)
    load = buses["p"] < 0
    s = sb[:, load, 0] / buses["p"][load]
    assert abs(s.mean() - 1) < 0.003 and abs(s.std() - 0.05) < 0.003
    assert np.allclose(sb[:, load, 1] / buses["q"][load], s)
    assert np.array_equal(sb[:, ~load, 0], np.broadcast_to(buses["p"][~load], sb[:, ~load, 0].shape))


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ missing")
def test_multifrontal_symbolic_by_host_emulation(tmp_path):
    exe = tmp_path / "mf_emulate"
    csrc = os.path.join(ROOT, "mapol_b200", "csrc")
    env = dict(os.environ)
    env.pop("CXX", None)
    subprocess.run(["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), "-I" + csrc,
                    os.path.join(ROOT, "tests", "native", "mf_emulate.cpp"), os.path.join(csrc, "symbolic.cpp"),
                    os.path.join(csrc, "synth.cpp"), "-o", str(exe)], check=True, env=env)
    for args in (["30", "41", "5"], ["300", "411", "69"], ["2869", "4582", "509"]):
        for ordering in ("0", "1", "2", "3"):  # automatic, minimum degree, minimum fill, weighted
            out = subprocess.run([str(exe)] + args + [ordering], capture_output=True, text=True)
            assert out.returncode == 0, out.stdout + out.stderr
            errs = [float(x) for x in out.stdout.split()]
            assert max(errs) < 1e-10
    # a densely meshed grid (uniform-random topology): 76 fronts above 167 rows take the
    # panel / trailing-block split of k_mf_factor_big, equal to the dense loop bit for bit
    out = subprocess.run([str(exe), "1354", "1991", "260", "0", "1"], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "big fronts 76, mismatching entries 0" in out.stderr


def test_python_binding_reports_no_device_without_gpu():
    import torch

    if torch.cuda.is_available():
        pytest.skip("GPU present")
    buses, branches = m.synth_grid(30, 41, 5)
    with pytest.raises(m.MpfError) as e:
        m.PowerFlow(buses, branches)
    assert e.value.code == 7
