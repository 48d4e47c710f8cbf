"""The tuning file (MPF_TUNE_FILE) carries autotuning results between processes.

A first process tunes and appends its choices (one factor and one backward-solve line
per precision); a second process reads them instead of tuning, appends nothing, and
its voltages equal the first's bit for bit.  A file whose entry names a kernel that
is not among the launch's candidates is not trusted: that entry is tuned again and a
valid line appended, and the solve still matches.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import sys
import numpy as np
import mapol_b200 as m
buses, branches, cases = m.workload("cfg1_300bus")
out = {}
with m.PowerFlow(buses, branches) as pf:
    pf.set_cases(cases[:64])
    for prec, name in ((m.MIXED, "mixed"), (m.FP64, "fp64")):
        pf.solve(m.NR, prec)
        r = pf.results()
        assert r.converged.all()
        out[name] = r.v
np.savez(sys.argv[1], **out)
"""


def _run(tmp_path, tune_file, tag):
    out = tmp_path / f"{tag}.npz"
    env = dict(os.environ, MPF_TUNE_FILE=str(tune_file))
    subprocess.run([sys.executable, "-c", SCRIPT, str(out)], cwd=ROOT, env=env, check=True, timeout=600)
    return np.load(out)


def _lines(path):
    return [l.split() for l in path.read_text().splitlines() if l.strip()]


def test_tune_file_round_trip(gpu, tmp_path):
    tf = tmp_path / "tune.txt"
    a = _run(tmp_path, tf, "a")
    first = _lines(tf)
    assert sorted({(l[0], l[2]) for l in first}) == [("bsolve", "0"), ("bsolve", "1"), ("factor", "0"),
                                                      ("factor", "1")]
    for l in first:
        assert int(l[4]) == len(l) - 5
    b = _run(tmp_path, tf, "b")
    assert _lines(tf) == first  # read, not tuned again
    for k in ("mixed", "fp64"):
        assert np.array_equal(a[k], b[k])


def test_tune_file_rejects_unknown_kernel(gpu, tmp_path):
    tf = tmp_path / "tune.txt"
    a = _run(tmp_path, tf, "a")
    lines = _lines(tf)
    bad = []
    for l in lines:
        if l[0] == "factor" and l[2] == "1":
            l = l[:5] + ["9,8,0,1"] + l[6:]  # no kernel of kind 9
        bad.append(l)
    tf.write_text("".join(" ".join(l) + "\n" for l in bad))
    b = _run(tmp_path, tf, "b")
    after = _lines(tf)
    assert len(after) == len(bad) + 1 and after[-1][0] == "factor" and after[-1][2] == "1"
    assert "9,8,0,1" not in after[-1]
    for k in ("mixed", "fp64"):
        assert np.abs(a[k] - b[k]).max() < 1e-8
