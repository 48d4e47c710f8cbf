"""Optimiser-facing shim: the reference's particle-swarm power-flow interface over
the batched engine.

Reference (src/pso/Particula.h, src/main.cu, src/powerflow/runpf.h):
  Particula::Estrutura {tipo, min, max, defaultValue, qtd, id}   Particula.h:26-60
  the structures main builds from a grid                          main.cu:232-262
  hybrid_init(topology, nTest, nThreads, estrutura, algPF)        runpf.h:795
  hybrid_runpf(estrutura, enxame): particle i -> case i, fitness
      = total active loss if converged else DBL_MAX               runpf.h:606-791
  hybrid_free()                                                   runpf.h:984

A particle's coordinate k is the value of structure k.  Buses and branches point
at their structure through an index (the reference's Bus/Branch::indiceEstrutura,
-1 for none); which coordinates reach the power flow follows the reference:
  * bus whose structure is AVR  -> |V| set-point of that bus (runpf.h:524-541)
  * bus whose structure is SHC  -> its shunt susceptance Bsh (makeYbus.h:313-318)
  * branch with tap != 0 and a structure -> its tap ratio (makeYbus.h:331)
main.cu binds a PV bus that also has Bsh > 0 to its SHC structure last, so that
bus's AVR coordinate reaches nothing; bind() reproduces that.
"""
from dataclasses import dataclass

import numpy as np

from . import _types as T
from .runpf import PowerFlow

NULO, AVR, OLTC, SHC = 0, T.CTRL_AVR, T.CTRL_OLTC, T.CTRL_SHC
DBL_MAX = np.finfo(np.float64).max


@dataclass
class Estrutura:
    """Particula::Estrutura (Particula.h:26-60)."""
    tipo: int
    min: float
    max: float
    default: float
    qtd: int
    id: int


@dataclass
class Particula:
    """The part of Particula (Particula.h) the power flow reads and writes."""
    X: np.ndarray
    fitness: float = DBL_MAX

    def mudar_fitness(self, f):
        self.fitness = float(f)


def estruturas(buses, branches):
    """The structures main.cu:232-262 builds, and the bus / branch bindings:
    AVR [0.9, 1.1] at every PV bus (default |V|), ShC [0, 0.18] in 3 steps at every
    bus with Bsh > 0 (default Bsh), OLTC [0.9, 1.1] in 20 steps at every branch
    with tap > 0 (default tap).  Returns (estrutura, bus_index, branch_index)."""
    est = []
    bus_ie = np.full(len(buses), -1, np.int32)
    br_ie = np.full(len(branches), -1, np.int32)
    for i, b in enumerate(buses):
        if b["type"] == T.BUS_PV:
            bus_ie[i] = len(est)
            est.append(Estrutura(AVR, 0.9, 1.1, float(b["vm"]), 0, i))
        if b["bsh"] > 0:
            bus_ie[i] = len(est)
            est.append(Estrutura(SHC, 0.0, 0.18, float(b["bsh"]), 3, i))
    for k, br in enumerate(branches):
        if br["tap"] > 0:
            br_ie[k] = len(est)
            est.append(Estrutura(OLTC, 0.9, 1.1, float(br["tap"]), 20, k))
    return est, bus_ie, br_ie


def bind(estrutura, bus_ie, br_ie, branches):
    """(controls, columns): the engine controls a particle drives and, for each, the
    particle coordinate that holds its value."""
    controls, cols = [], []
    for i, ie in enumerate(bus_ie):
        if ie < 0:
            continue
        tipo = estrutura[ie].tipo
        if tipo in (AVR, SHC):
            controls.append((tipo, i))
            cols.append(int(ie))
    for k, ie in enumerate(br_ie):
        if ie >= 0 and branches[k]["tap"] != 0:
            controls.append((OLTC, k))
            cols.append(int(ie))
    return controls, np.array(cols, np.int64)


class Engine:
    """hybrid_init's state: one grid, n_tests particles per hybrid_runpf."""

    def __init__(self, buses, branches, n_tests, estrutura, alg, bus_ie, br_ie, precision=T.FP64, **kw):
        self.pf = PowerFlow(buses, branches, **kw)
        self.n_tests = n_tests
        self.alg = alg
        self.precision = precision
        self.controls, self.cols = bind(estrutura, bus_ie, br_ie, self.pf.branches)
        self.n_struct = len(estrutura)

    def close(self):
        self.pf.close()


def hybrid_init(buses, branches, n_tests, n_threads, estrutura, alg, bus_ie, br_ie, **kw):
    """hybrid_init (runpf.h:795); n_threads is unused (the reference passes it to MKL)."""
    return Engine(buses, branches, n_tests, estrutura, alg, bus_ie, br_ie, **kw)


def hybrid_runpf(engine, estrutura, enxame):
    """hybrid_runpf (runpf.h:606-791): case i = particle i; sets every particle's
    fitness (total active loss, or DBL_MAX when the case did not converge) and
    returns the fitness vector."""
    if len(enxame) != engine.n_tests:
        raise ValueError(f"expected {engine.n_tests} particles, got {len(enxame)}")
    if len(estrutura) != engine.n_struct:
        raise ValueError("estrutura differs from the one given to hybrid_init")
    X = np.array([np.asarray(p.X, np.float64) for p in enxame])
    pf = engine.pf
    pf.set_cases([[] for _ in enxame])
    if engine.controls:
        pf.set_controls(engine.controls, X[:, engine.cols])
    pf.solve(engine.alg, engine.precision)
    fit = pf.fitness()
    for p, f in zip(enxame, fit):
        p.mudar_fitness(f)
    return fit


def hybrid_free(engine):
    """hybrid_free (runpf.h:984)."""
    engine.close()
