"""ctypes wrapper of the CPU oracle (mpf_oracle.cpp).  TEST INFRASTRUCTURE: imported
only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm,
always as the checker or as the timed CPU baseline.

Parity pin: the oracle reproduces the reference's own CPU power flow (its runpf.h and
the headers it includes, compiled unmodified into oracle/_ref/librefpf.so, see
refpf.py): identical converged flags and iteration counts and voltages to ~1e-13 on
the reference's bundled MATPOWER cases with N-1 outages (tests/test_oracle_reference_pin.py).
It is also cross-checked against an independent numpy/scipy Newton-Raphson and
analytic 2-bus cases.  Solvers: SOLVER_GP (own sparse LU, minimum degree),
SOLVER_EIGEN (the reference's Eigen SparseLU option, compute() every solve),
SOLVER_EIGEN_REUSE (the same with its symbolic analysis done once per case).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_OWN = os.path.join(HERE, "liboracle.so")
LIB_REF = os.path.join(HERE, "_ref", "liboracle.so")

SOLVER_GP, SOLVER_EIGEN, SOLVER_EIGEN_REUSE = 0, 1, 2

_libs = {}


def _load(path):
    if path not in _libs:
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: build with `make -C oracle`")
        L = ctypes.CDLL(path)
        c_p, c_i, c_d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.oracle_runpf.restype = c_i
        L.oracle_runpf.argtypes = [c_p, c_i, c_p, c_i, c_i, c_i, c_d, c_i, c_i, c_i, c_p, c_p, c_p, c_p, c_p, c_p,
                                   c_p, c_i]
        L.oracle_ybus.restype = c_i
        L.oracle_ybus.argtypes = [c_p, c_i, c_p, c_i, c_p, c_i, c_p, c_p, c_p]
        L.oracle_nr_system.restype = c_d
        L.oracle_nr_system.argtypes = [c_p, c_i, c_p, c_i, c_p, c_i, c_p, c_p, c_p, c_p, c_p, c_p]
        L.oracle_loss.restype = c_d
        L.oracle_loss.argtypes = [c_p, c_i, c_p, c_i, c_p, c_i, c_p]
        L.oracle_has_eigen.restype = c_i
        _libs[path] = L
    return _libs[path]


def has_eigen():
    return os.path.exists(LIB_REF) and _load(LIB_REF).oracle_has_eigen() == 1


def _lib_for(solver):
    eigen = solver in (SOLVER_EIGEN, SOLVER_EIGEN_REUSE)
    return _load(LIB_REF if eigen else (LIB_OWN if os.path.exists(LIB_OWN) else LIB_REF))


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def runpf(buses, branches, cases, alg=0, max_it=None, tol=1e-8, solver=SOLVER_GP, angle_mode=0,
          sbus=None, threads=None):
    """Runs the oracle on every case.  Returns dict(v complex (n, nb), iterations,
    converged (bool), max_mis)."""
    nb = len(buses)
    n = len(cases)
    offs = np.zeros(n + 1, np.int32)
    flat = []
    for i, c in enumerate(cases):
        offs[i + 1] = offs[i] + len(c)
        flat.extend(int(b) for b in c)
    flat = np.asarray(flat + [0], np.int32)
    if max_it is None:
        max_it = 10 if alg == 0 else 30
    v = np.zeros((n, nb, 2))
    it = np.zeros(n, np.int32)
    cv = np.zeros(n, np.uint8)
    mm = np.zeros(n)
    sb = None if sbus is None else np.ascontiguousarray(sbus, dtype=np.float64)
    threads = threads or os.cpu_count() or 1
    rc = _lib_for(solver).oracle_runpf(_p(buses), nb, _p(branches), len(branches), alg, max_it, tol, solver,
                                       angle_mode, n, _p(offs), _p(flat), _p(sb), _p(v), _p(it), _p(cv), _p(mm),
                                       threads)
    if rc != 0:
        raise RuntimeError("oracle_runpf rejected its input")
    return dict(v=v[..., 0] + 1j * v[..., 1], iterations=it, converged=cv.astype(bool), max_mis=mm)


def ybus(buses, branches, outages=()):
    L = _lib_for(SOLVER_GP)
    nb = len(buses)
    out = np.asarray(list(outages) + [0], np.int32)
    ptr_ = np.zeros(nb + 1, np.int32)
    nnz = L.oracle_ybus(_p(buses), nb, _p(branches), len(branches), _p(out), len(outages), _p(ptr_), None, None)
    col = np.zeros(nnz, np.int32)
    val = np.zeros((nnz, 2))
    L.oracle_ybus(_p(buses), nb, _p(branches), len(branches), _p(out), len(outages), _p(ptr_), _p(col), _p(val))
    return ptr_, col, val[:, 0] + 1j * val[:, 1]


def nr_system(buses, branches, v, outages=()):
    """Mismatch F and Jacobian (CSR, reference ordering) at complex voltage v."""
    L = _lib_for(SOLVER_GP)
    nb = len(buses)
    out = np.asarray(list(outages) + [0], np.int32)
    vv = np.stack([v.real, v.imag], -1).astype(np.float64).copy()
    npv = int((buses["type"] == 2).sum())
    npq = int((buses["type"] == 1).sum())
    n = npv + 2 * npq
    F = np.zeros(n)
    nnz = ctypes.c_int(0)
    L.oracle_nr_system(_p(buses), nb, _p(branches), len(branches), _p(out), len(outages), _p(vv), _p(F), None, None,
                       None, ctypes.byref(nnz))
    jp = np.zeros(n + 1, np.int32)
    jc = np.zeros(nnz.value, np.int32)
    jv = np.zeros(nnz.value)
    err = L.oracle_nr_system(_p(buses), nb, _p(branches), len(branches), _p(out), len(outages), _p(vv), _p(F),
                             _p(jp), _p(jc), _p(jv), None)
    return F, (jp, jc, jv), err


def loss(buses, branches, v, outages=()):
    L = _lib_for(SOLVER_GP)
    out = np.asarray(list(outages) + [0], np.int32)
    vv = np.stack([v.real, v.imag], -1).astype(np.float64).copy()
    return L.oracle_loss(_p(buses), len(buses), _p(branches), len(branches), _p(out), len(outages), _p(vv))


def runpf_qlim(buses, branches, cases, qmin, qmax, alg=0, tol=1e-8, sbus=None, max_rounds=20, solver=SOLVER_GP):
    """Newton-Raphson with reactive limits of PV buses, case by case (MATPOWER runpf
    with ENFORCE_Q_LIMS = 1; the reference parses the limits but never enforces them,
    loadMatpowerFormat.h:130-137): solve; at the converged voltages compute each PV
    bus's net reactive injection Q = Im(V_i conj((Ybus V)_i)); every PV bus outside
    [qmin, qmax] becomes PQ with Q at the violated limit; solve again; repeat until no
    new violation.  Each round solves from the start point (runpf.h:211-226) with the
    updated bus types, which converges to the same state as continuing from the
    previous round's voltages.  Returns dict(v, converged, iterations (summed over the
    rounds), switched (bool, n_cases x n_bus), rounds)."""
    nb = len(buses)
    n = len(cases)
    lo = np.where(np.isnan(qmin), -np.inf, qmin)
    hi = np.where(np.isnan(qmax), np.inf, qmax)
    out_v = np.zeros((n, nb), complex)
    conv = np.zeros(n, bool)
    iters = np.zeros(n, np.int32)
    switched = np.zeros((n, nb), bool)
    rounds = np.zeros(n, np.int32)
    for c in range(n):
        b = np.array(buses).copy()
        sb = None if sbus is None else np.array(sbus[c:c + 1]).copy()
        for rnd in range(max_rounds + 1):
            r = runpf(b, branches, [cases[c]], alg=alg, tol=tol, sbus=sb, solver=solver, threads=1)
            iters[c] += r["iterations"][0]
            out_v[c] = r["v"][0]
            conv[c] = r["converged"][0]
            if not conv[c] or rnd == max_rounds:
                break
            ptr_, col, val = ybus(b, branches, cases[c])
            v = r["v"][0]
            ib = np.array([np.dot(val[ptr_[i]:ptr_[i + 1]], v[col[ptr_[i]:ptr_[i + 1]]]) for i in range(nb)])
            q = (v * np.conj(ib)).imag
            pv = b["type"] == 2
            over = pv & (q > hi)
            under = pv & (q < lo)
            if not (over | under).any():
                break
            rounds[c] += 1
            for i in np.where(over | under)[0]:
                lim = hi[i] if over[i] else lo[i]
                b["type"][i] = 1
                b["q"][i] = lim
                if sb is not None:
                    sb[0, i, 1] = lim
                switched[c, i] = True
    return dict(v=out_v, converged=conv, iterations=iters, switched=switched, rounds=rounds)
