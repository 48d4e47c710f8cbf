"""Independent Newton-Raphson in numpy/scipy (MATPOWER polar formulas: dS/dVa =
j diag(V) conj(diag(Ibus) - Ybus diag(V)), dS/dVm = diag(V) conj(Ybus diag(V/|V|)) +
conj(diag(Ibus)) diag(V/|V|)).  Test-only second formulation used to pin the oracle."""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spl


def ybus(buses, branches, outages=()):
    br = branches.copy()
    for k in outages:
        br["status"][k] = 0
    nb = len(buses)
    f, t, st = br["from"], br["to"], br["status"].astype(float)
    ys = st / (br["r"] + 1j * br["x"])
    tap = np.where(br["tap"] != 0, br["tap"], 1.0) * np.exp(1j * np.pi / 180 * br["shift"])
    ytt = ys + 1j * st * br["b"] / 2
    yff = ytt / (tap * np.conj(tap))
    yft = -ys / np.conj(tap)
    ytf = -ys / tap
    Y = sp.coo_matrix((np.r_[yff, yft, ytf, ytt], (np.r_[f, f, t, t], np.r_[f, t, f, t])), (nb, nb)).tocsr()
    return (Y + sp.diags(buses["gsh"] + 1j * buses["bsh"])).tocsr()


def newton(buses, branches, outages=(), sbus=None, max_it=10, tol=1e-8):
    Y = ybus(buses, branches, outages)
    pv = np.where(buses["type"] == 2)[0]
    pq = np.where(buses["type"] == 1)[0]
    pvpq = np.r_[pv, pq]
    S = buses["p"] + 1j * buses["q"] if sbus is None else sbus[:, 0] + 1j * sbus[:, 1]
    Va = buses["va"].astype(float).copy()
    Vm = buses["vm"].astype(float).copy()
    V = Vm * np.exp(1j * Va)
    for it in range(max_it + 1):
        mis = V * np.conj(Y @ V) - S
        F = np.r_[mis[pvpq].real, mis[pq].imag]
        if np.abs(F).max() < tol:
            return V, it, True
        if it == max_it:
            return V, it, False
        Ib = Y @ V
        dV, dIb, dVn = sp.diags(V), sp.diags(Ib), sp.diags(V / np.abs(V))
        dVm = dV @ np.conj(Y @ dVn) + np.conj(dIb) @ dVn
        dVa = 1j * dV @ np.conj(dIb - Y @ dV)
        J = sp.vstack([sp.hstack([dVa[pvpq][:, pvpq].real, dVm[pvpq][:, pq].real]),
                       sp.hstack([dVa[pq][:, pvpq].imag, dVm[pq][:, pq].imag])]).tocsc()
        dx = spl.spsolve(J, F)
        Va[pvpq] -= dx[: len(pvpq)]
        Vm[pq] -= dx[len(pvpq):]
        V = Vm * np.exp(1j * Va)
