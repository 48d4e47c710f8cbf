"""MATPOWER version-2 case files (.m) -> bus / branch arrays of include/mpf.h.

Follows the reference's loader (src/files/loadMatpowerFormat.h:14-209):
  * buses are numbered 0.. in file order; branch ends are mapped through the bus ids
    (loadMatpowerFormat.h:176-191);
  * bus P, Q are net injections in p.u.: -Pd/baseMVA, -Qd/baseMVA, plus Pg/baseMVA,
    Qg/baseMVA of every generator at the bus; the generator status column is not
    read (loadMatpowerFormat.h:87-88, 118-123: all generators inject);
  * shunts Gs/baseMVA, Bs/baseMVA; angles converted to radians;
  * branch R, X, B, ratio (0 = no transformer), angle (degrees), status.
Differences, stated: the generator voltage set-point VG becomes the PV/slack bus
magnitude (the reference stores VG in Bus::VG and its optimiser starts AVR controls
from it, main.cu:276-395; MATPOWER's runpf does the same), and branch rating A
(MVA, returned as p.u.) is kept where the reference discards it.  q_limits()
returns the generators' reactive limits, which the reference parses
(loadMatpowerFormat.h:130-137) and never uses, as net-injection limits per bus.
"""
import re

import numpy as np

from ._types import BRANCH_DTYPE, BUS_DTYPE


def _matrix(text, name):
    m = re.search(r"mpc\." + name + r"\s*=\s*\[(.*?)\];", text, re.S)
    if not m:
        return None
    rows = []
    for line in m.group(1).splitlines():
        line = line.split("%")[0].strip().rstrip(";").strip()
        if not line:
            continue
        rows.append([float(v) for v in line.replace("Inf", "inf").split()])
    return rows


def load_matpower(path):
    """Returns (buses, branches, rating_pu) for a MATPOWER v2 case file."""
    with open(path) as f:
        text = f.read()
    if not re.search(r"mpc\.version\s*=\s*'2'", text):
        raise ValueError("only MATPOWER case format version 2 is supported (loadMatpowerFormat.h:41-47)")
    base = float(re.search(r"mpc\.baseMVA\s*=\s*([0-9.eE+-]+)", text).group(1))
    bus = _matrix(text, "bus")
    gen = _matrix(text, "gen") or []
    branch = _matrix(text, "branch")
    nb = len(bus)
    ids = {int(r[0]): i for i, r in enumerate(bus)}
    buses = np.zeros(nb, BUS_DTYPE)
    for i, r in enumerate(bus):
        buses[i]["type"] = int(r[1])
        buses[i]["p"] = -r[2] / base
        buses[i]["q"] = -r[3] / base
        buses[i]["gsh"] = r[4] / base
        buses[i]["bsh"] = r[5] / base
        buses[i]["vm"] = r[7]
        buses[i]["va"] = r[8] * np.pi / 180.0
    for r in gen:
        i = ids[int(r[0])]
        buses[i]["p"] += r[1] / base
        buses[i]["q"] += r[2] / base
        if buses[i]["type"] in (2, 3):
            buses[i]["vm"] = r[5]
    branches = np.zeros(len(branch), BRANCH_DTYPE)
    rating = np.zeros(len(branch))
    for k, r in enumerate(branch):
        branches[k]["from"] = ids[int(r[0])]
        branches[k]["to"] = ids[int(r[1])]
        branches[k]["r"], branches[k]["x"], branches[k]["b"] = r[2], r[3], r[4]
        rating[k] = r[5] / base
        branches[k]["tap"] = r[8]
        branches[k]["shift"] = r[9]
        branches[k]["status"] = 1 if r[10] != 0 else 0
    return buses, branches, rating


def q_limits(path):
    """(qmin, qmax) per bus in p.u. of net reactive injection: the sum of the Qmin /
    Qmax of the bus's generators (gen columns 5 and 4) minus its reactive load Qd;
    -inf / +inf at buses without generators or with infinite limits."""
    with open(path) as f:
        text = f.read()
    base = float(re.search(r"mpc\.baseMVA\s*=\s*([0-9.eE+-]+)", text).group(1))
    bus = _matrix(text, "bus")
    gen = _matrix(text, "gen") or []
    ids = {int(r[0]): i for i, r in enumerate(bus)}
    nb = len(bus)
    qmin = np.full(nb, -np.inf)
    qmax = np.full(nb, np.inf)
    has = np.zeros(nb, bool)
    sum_min = np.zeros(nb)
    sum_max = np.zeros(nb)
    for r in gen:
        i = ids[int(r[0])]
        has[i] = True
        sum_max[i] += r[3]
        sum_min[i] += r[4]
    for i, r in enumerate(bus):
        if has[i]:
            qmax[i] = (sum_max[i] - r[3]) / base
            qmin[i] = (sum_min[i] - r[3]) / base
    return qmin, qmax
