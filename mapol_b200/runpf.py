"""Host-side mirror of the reference's power-flow entry points, over libmpf.so.

Reference (src/powerflow/runpf.h):
  hybrid_init(topology, nTest, nThreads, estrutura, algPF)   runpf.h:795
  hybrid_runpf(estrutura, enxame)                             runpf.h:606
  hybrid_free()                                               runpf.h:984
  mkl_runpf(estrutura, particula) -> loss or DBL_MAX          runpf.h:259
with algorithms NR / FDXB / FDBX (runpf.h:16-18) and MAX_IT_NR / MAX_IT_FD / EPS
(runpf.h:45-47).  The reference keeps one global engine per process and exits
on error; here an engine is an object and errors raise MpfError.

A "case" is the base grid with a list of outaged branches (N-1, N-k: at most 4
per case) and, optionally, its own bus injections.
"""
import ctypes

import numpy as np

from . import _types as T
from ._lib import MpfError, lib, ptr
from .grid import cases_to_offsets

NR, FDXB, FDBX = T.NR, T.FDXB, T.FDBX
FP64, MIXED = T.FP64, T.MIXED
MAX_IT_NR, MAX_IT_FD, EPS = T.MAX_IT_NR, T.MAX_IT_FD, T.EPS

CONVERGED = T.CASE_CONVERGED


class Results:
    """Per-case outputs: v (n_cases, n_bus) complex, iterations, status, max_mis."""

    def __init__(self, v, iterations, status, max_mis):
        self.v = v
        self.iterations = iterations
        self.status = status
        self.max_mis = max_mis

    @property
    def converged(self):
        return self.status == T.CASE_CONVERGED


class PowerFlow:
    """One grid on one GPU (mpf_create).  Replaces hybrid_init / hybrid_free."""

    def __init__(self, buses, branches, max_it_nr=MAX_IT_NR, max_it_fd=MAX_IT_FD, tol=EPS,
                 angle_mode=0, device=0, use_graph=2, autotune=1, ordering=T.ORDER_AUTO):
        self.buses = np.ascontiguousarray(buses, dtype=T.BUS_DTYPE)
        self.branches = np.ascontiguousarray(branches, dtype=T.BRANCH_DTYPE)
        opt = T.Options()
        lib().mpf_default_options(ctypes.byref(opt))
        opt.max_it_nr, opt.max_it_fd, opt.tol = max_it_nr, max_it_fd, tol
        opt.angle_mode, opt.device, opt.use_graph, opt.autotune = angle_mode, device, use_graph, autotune
        opt.ordering = ordering
        h = ctypes.c_void_p()
        rc = lib().mpf_create(ptr(self.buses), len(self.buses), ptr(self.branches), len(self.branches),
                              ctypes.byref(opt), ctypes.byref(h))
        self._h = h
        self.device = device
        if rc != 0:
            msg = lib().mpf_last_error(h).decode() if h.value else lib().mpf_status_string(rc).decode()
            if h.value:
                lib().mpf_destroy(h)
                self._h = None
            raise MpfError(rc, msg)
        self.n_cases = 0

    # -- lifecycle -----------------------------------------------------------
    def close(self):
        if self._h is not None and self._h.value:
            lib().mpf_destroy(self._h)
        self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise MpfError(rc, lib().mpf_last_error(self._h).decode())

    # -- cases and solves ----------------------------------------------------
    def set_cases(self, cases, sbus=None, islands=None):
        """cases: list of outage lists (branch indices); sbus: (n_cases, n_bus, 2) or None;
        islands (grids with several islands): the island of each case (mpf_set_cases_islands)."""
        offs, flat = cases_to_offsets(cases)
        sb = None if sbus is None else np.ascontiguousarray(sbus, dtype=np.float64)
        if islands is None:
            self._check(lib().mpf_set_cases(self._h, len(cases), ptr(offs), ptr(flat), ptr(sb)))
        else:
            isl = np.ascontiguousarray(islands, dtype=np.int32)
            if isl.shape != (len(cases),):
                raise ValueError("islands needs one entry per case")
            self._check(lib().mpf_set_cases_islands(self._h, len(cases), ptr(isl), ptr(offs), ptr(flat), ptr(sb)))
        self.n_cases = len(cases)

    def set_q_limits(self, qmin, qmax):
        """Reactive limits of PV buses (mpf_set_q_limits): per-bus net-injection limits in
        p.u., +-inf / NaN for none; None for both disables.  Call before set_cases."""
        lo = None if qmin is None else np.ascontiguousarray(qmin, dtype=np.float64)
        hi = None if qmax is None else np.ascontiguousarray(qmax, dtype=np.float64)
        for a in (lo, hi):
            if a is not None and a.shape != (len(self.buses),):
                raise ValueError("limits need one entry per bus")
        self._check(lib().mpf_set_q_limits(self._h, ptr(lo), ptr(hi)))
        self.n_cases = 0

    def bus_types(self):
        """(n_cases, n_bus) bus types after the last solve (switched PV buses read PQ)."""
        out = np.zeros((self.n_cases, len(self.buses)), np.uint8)
        self._check(lib().mpf_get_bus_types(self._h, ptr(out)))
        return out

    def set_controls(self, controls, values):
        """Per-case control overrides of the current cases (mpf_set_controls).
        controls: sequence of (kind, index) with kind CTRL_AVR (PV/slack bus |V|
        set-point), CTRL_OLTC (tap ratio of a tapped branch) or CTRL_SHC (bus shunt
        susceptance); values: (n_cases, n_controls).  An empty sequence clears."""
        ctl = np.array([tuple(c) for c in controls], dtype=T.CONTROL_DTYPE)
        if len(ctl) == 0:
            self._check(lib().mpf_set_controls(self._h, 0, None, None))
            return
        val = np.ascontiguousarray(values, dtype=np.float64)
        if val.shape != (self.n_cases, len(ctl)):
            raise ValueError(f"values must be ({self.n_cases}, {len(ctl)}), got {val.shape}")
        self._check(lib().mpf_set_controls(self._h, len(ctl), ptr(ctl), ptr(val)))

    def solve(self, alg=NR, precision=FP64, stream=None):
        self._check(lib().mpf_solve(self._h, alg, precision, stream))

    def results(self):
        nb = len(self.buses)
        v = np.zeros((self.n_cases, nb, 2))
        it = np.zeros(self.n_cases, np.int32)
        st = np.zeros(self.n_cases, np.uint8)
        mm = np.zeros(self.n_cases)
        self._check(lib().mpf_get_results(self._h, ptr(v), ptr(it), ptr(st), ptr(mm)))
        return Results(v[..., 0] + 1j * v[..., 1], it, st, mm)

    def runpf(self, cases, alg=NR, precision=FP64, sbus=None):
        """End to end from host memory (mpf_runpf_host): cases in, results out."""
        nb = len(self.buses)
        n = len(cases)
        offs, flat = cases_to_offsets(cases)
        sb = None if sbus is None else np.ascontiguousarray(sbus, dtype=np.float64)
        v = np.zeros((n, nb, 2))
        it = np.zeros(n, np.int32)
        st = np.zeros(n, np.uint8)
        mm = np.zeros(n)
        self._check(lib().mpf_runpf_host(self._h, alg, precision, n, ptr(offs), ptr(flat), ptr(sb),
                                         ptr(v), ptr(it), ptr(st), ptr(mm)))
        self.n_cases = n
        return Results(v[..., 0] + 1j * v[..., 1], it, st, mm)

    def set_ratings(self, rating):
        """Branch ratings (p.u. apparent power, [n_branch]) for the overload loss."""
        r = None if rating is None else np.ascontiguousarray(rating, dtype=np.float64)
        self._check(lib().mpf_set_ratings(self._h, ptr(r)))
        self.has_ratings = r is not None

    def branch_flows(self, flows=False):
        """Per-case active loss (and overload loss when ratings are set) at the solved
        voltages; with flows=True also Sf, St (n_cases, n_branch) complex."""
        import torch

        n, nbr = self.n_cases, len(self.branches)
        dev = torch.device("cuda", self.device)
        ploss = torch.zeros(n, dtype=torch.float64, device=dev)
        over = torch.zeros(n, dtype=torch.float64, device=dev) if getattr(self, "has_ratings", False) else None
        sf = torch.zeros((n, nbr, 2), dtype=torch.float64, device=dev) if flows else None
        st = torch.zeros((n, nbr, 2), dtype=torch.float64, device=dev) if flows else None
        dp = lambda t: None if t is None else t.data_ptr()  # noqa: E731
        self._check(lib().mpf_branch_flows(self._h, dp(ploss), dp(over), dp(sf), dp(st), None))
        torch.cuda.synchronize(dev)
        out = {"ploss": ploss.cpu().numpy()}
        if over is not None:
            out["overload"] = over.cpu().numpy()
        if flows:
            a, b = sf.cpu().numpy(), st.cpu().numpy()
            out["sf"] = a[..., 0] + 1j * a[..., 1]
            out["st"] = b[..., 0] + 1j * b[..., 1]
        return out

    def adjoint(self, precision=FP64):
        """Gradients of each converged case's overload loss (ratings must be set):
        dict of (n_cases, n_bus) grad_p, grad_q and (n_cases, n_branch) grad_g, grad_b."""
        import torch

        n, nb, nbr = self.n_cases, len(self.buses), len(self.branches)
        dev = torch.device("cuda", self.device)
        bufs = {"grad_p": (n, nb), "grad_q": (n, nb), "grad_g": (n, nbr), "grad_b": (n, nbr)}
        t = {k: torch.zeros(v, dtype=torch.float64, device=dev) for k, v in bufs.items()}
        self._check(lib().mpf_adjoint(self._h, precision, t["grad_p"].data_ptr(), t["grad_q"].data_ptr(),
                                      t["grad_g"].data_ptr(), t["grad_b"].data_ptr(), None))
        torch.cuda.synchronize(dev)
        return {k: v.cpu().numpy() for k, v in t.items()}

    def fitness(self, results=None):
        """The reference's per-case fitness after hybrid_runpf: total active loss when
        the case converged, DBL_MAX otherwise (runpf.h:748-791)."""
        res = results if results is not None else self.results()
        loss = self.branch_flows()["ploss"]
        return np.where(res.status == T.CASE_CONVERGED, loss, np.finfo(np.float64).max)

    def timing(self):
        t = T.Timing()
        self._check(lib().mpf_get_timing(self._h, ctypes.byref(t)))
        return {k: getattr(t, k) for k, _ in T.Timing._fields_}

    def stats(self):
        s = T.Stats()
        self._check(lib().mpf_get_stats(self._h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in T.Stats._fields_}


# -- the reference's procedural names ------------------------------------------
def hybrid_init(buses, branches, n_tests, alg=NR, **kw):
    """hybrid_init (runpf.h:795): build the engine for n_tests simultaneous cases."""
    pf = PowerFlow(buses, branches, **kw)
    pf.alg = alg
    pf.n_tests = n_tests
    return pf


def hybrid_runpf(pf, cases, precision=FP64, sbus=None):
    """hybrid_runpf (runpf.h:606): solve every case; returns Results."""
    if len(cases) != pf.n_tests:
        raise ValueError(f"expected {pf.n_tests} cases, got {len(cases)}")
    return pf.runpf(cases, alg=pf.alg, precision=precision, sbus=sbus)


def hybrid_free(pf):
    """hybrid_free (runpf.h:984)."""
    pf.close()
