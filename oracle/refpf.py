"""ctypes wrapper of oracle/_ref/librefpf.so: the reference's own CPU power-flow code
(mkl_init / mkl_runpf / mkl_clean of src/powerflow/runpf.h with makeYbus.h,
newtonpf.h, makeB.h, fdpf.h), compiled unmodified from the reference tree by
oracle/Makefile with in-project stand-ins for MKL (oracle/refshim/).  TEST
INFRASTRUCTURE: imported only by tests/ (to pin the oracle and the fixtures to the
reference's outputs) and by bench.py's reference arm (the timed CPU baseline).

Solvers: SOLVER_EIGEN = the reference's Eigen_SparseLU option (newtonpf.h:341-363);
SOLVER_DSS = its default MKL_DSS path, here with the stand-in DSS (Eigen SparseLU
underneath), needed by the fast-decoupled solves, which call DSS directly.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "librefpf.so")

SOLVER_DSS, SOLVER_EIGEN = 0, 5

_lib = None


def available():
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"{LIB} missing: build with `make -C oracle` where the reference tree is present")
        L = ctypes.CDLL(LIB)
        c_p, c_i = ctypes.c_void_p, ctypes.c_int
        L.refpf_runpf.restype = c_i
        L.refpf_runpf.argtypes = [c_p, c_i, c_p, c_i, c_i, c_i, c_i, c_p, c_p, c_p, c_p, c_p, c_p, c_p]
        L.refpf_ybus.restype = c_i
        L.refpf_ybus.argtypes = [c_p, c_i, c_p, c_i, c_i, c_p, c_p, c_p, c_p]
        L.refpf_nr_open.restype = c_i
        L.refpf_nr_open.argtypes = [c_p, c_i, c_p, c_i, c_i]
        L.refpf_nr_step.restype = c_i
        L.refpf_nr_step.argtypes = [c_i, c_p, c_p, c_p, c_p, c_p]
        L.refpf_nr_close.restype = c_i
        L.refpf_nr_close.argtypes = []
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _offsets(cases):
    offs = np.zeros(len(cases) + 1, np.int32)
    flat = []
    for i, c in enumerate(cases):
        offs[i + 1] = offs[i] + len(c)
        flat.extend(int(b) for b in c)
    return offs, np.asarray(flat + [0], np.int32)


def runpf(buses, branches, cases, alg=0, solver=SOLVER_EIGEN, sbus=None):
    """The reference's mkl_runpf on every case, one after another (its state is
    global).  Returns dict(v complex (n, nb), iterations, converged (bool), loss)."""
    buses = np.ascontiguousarray(buses)
    branches = np.ascontiguousarray(branches)
    n, nb = len(cases), len(buses)
    offs, flat = _offsets(cases)
    v = np.zeros((n, nb, 2))
    it = np.zeros(n, np.int32)
    cv = np.zeros(n, np.uint8)
    loss = np.zeros(n)
    sb = None if sbus is None else np.ascontiguousarray(sbus, dtype=np.float64)
    rc = lib().refpf_runpf(_p(buses), nb, _p(branches), len(branches), alg, solver, n, _p(offs), _p(flat), _p(sb),
                           _p(v), _p(it), _p(cv), _p(loss))
    if rc != 0:
        raise RuntimeError("refpf_runpf rejected its input")
    return dict(v=v[..., 0] + 1j * v[..., 1], iterations=it, converged=cv.astype(bool), loss=loss)


def ybus(buses, branches, outages=()):
    """The reference's Ybus as a dense complex matrix (small grids only)."""
    buses = np.ascontiguousarray(buses)
    branches = np.ascontiguousarray(branches)
    nb = len(buses)
    out = np.asarray(list(outages) + [0], np.int32)
    rp = np.zeros(nb + 1, np.int32)
    nnz = lib().refpf_ybus(_p(buses), nb, _p(branches), len(branches), len(outages), _p(out), _p(rp), None, None)
    col = np.zeros(nnz, np.int32)
    val = np.zeros((nnz, 2))
    lib().refpf_ybus(_p(buses), nb, _p(branches), len(branches), len(outages), _p(out), _p(rp), _p(col), _p(val))
    Y = np.zeros((nb, nb), complex)
    for i in range(nb):
        for p in range(rp[i] - 1, rp[i + 1] - 1):
            Y[i, col[p] - 1] += val[p, 0] + 1j * val[p, 1]
    return Y, nnz


class Stepper:
    """The reference's Newton-Raphson one iteration per step() (refpf_nr_step), for
    one grid per process."""

    def __init__(self, buses, branches, solver=SOLVER_EIGEN):
        self.buses = np.ascontiguousarray(buses)
        self.branches = np.ascontiguousarray(branches)
        if lib().refpf_nr_open(_p(self.buses), len(self.buses), _p(self.branches), len(self.branches), solver) != 0:
            raise RuntimeError("refpf_nr_open failed (one grid per process)")
        self._d, self._c, self._i = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)

    def step(self, outages, v=None):
        """Starts a case with these outages if none is active, runs one iteration.
        Returns None while the case runs, else (converged, iterations)."""
        out = np.asarray(list(outages) + [0], np.int32)
        rc = lib().refpf_nr_step(len(outages), _p(out), ctypes.byref(self._d), ctypes.byref(self._c),
                                 ctypes.byref(self._i), _p(v))
        if rc != 0:
            raise RuntimeError("refpf_nr_step failed")
        return (bool(self._c.value), self._i.value) if self._d.value else None

    def close(self):
        lib().refpf_nr_close()
