"""numpy / ctypes mirrors of the POD records declared in include/mpf.h."""
import ctypes

import numpy as np

# mpf_bus: the fields of Bus (src/powersystem/Bus.h:18-31) the power flow reads
BUS_DTYPE = np.dtype(
    [
        ("type", np.int32),
        ("pad_", np.int32),
        ("vm", np.float64),
        ("va", np.float64),
        ("p", np.float64),
        ("q", np.float64),
        ("gsh", np.float64),
        ("bsh", np.float64),
    ],
    align=True,
)

# mpf_branch: the fields of Branch (src/powersystem/Branch.h:18-26)
BRANCH_DTYPE = np.dtype(
    [
        ("from", np.int32),
        ("to", np.int32),
        ("status", np.int32),
        ("pad_", np.int32),
        ("r", np.float64),
        ("x", np.float64),
        ("b", np.float64),
        ("tap", np.float64),
        ("shift", np.float64),
    ],
    align=True,
)

assert BUS_DTYPE.itemsize == 56 and BRANCH_DTYPE.itemsize == 56

# bus types (Bus::Type, src/powersystem/Bus.h:11-13)
BUS_NONE, BUS_PQ, BUS_PV, BUS_SLACK, BUS_ISOLATED = 0, 1, 2, 3, 4
# algorithms (src/powerflow/runpf.h:16-18)
NR, FDXB, FDBX = 0, 1, 2
FP64, MIXED = 0, 1
# limits (src/powerflow/runpf.h:45-47)
MAX_IT_NR, MAX_IT_FD, EPS = 10, 30, 1e-8

CASE_RUNNING, CASE_CONVERGED, CASE_MAX_ITER, CASE_DIVERGED, CASE_SINGULAR = 0, 1, 2, 3, 4
# fill-reducing orderings of the Newton system (mpf_options.ordering)
ORDER_AUTO, ORDER_MIN_DEGREE, ORDER_MIN_FILL, ORDER_MIN_FILL_WEIGHTED = 0, 1, 2, 3
# per-case control kinds (the values of Particula::Estrutura::Tipo, src/pso/Particula.h:27-29)
CTRL_AVR, CTRL_OLTC, CTRL_SHC = 1, 2, 3
CONTROL_DTYPE = np.dtype([("kind", "<i4"), ("index", "<i4")])


class SynthParams(ctypes.Structure):
    _fields_ = [
        ("n_bus", ctypes.c_int32),
        ("n_branch", ctypes.c_int32),
        ("n_pv", ctypes.c_int32),
        ("topology", ctypes.c_int32),
        ("tap_fraction", ctypes.c_double),
        ("tap_lo", ctypes.c_double),
        ("tap_hi", ctypes.c_double),
        ("r_lo", ctypes.c_double),
        ("r_hi", ctypes.c_double),
        ("xr_lo", ctypes.c_double),
        ("xr_hi", ctypes.c_double),
        ("b_hi", ctypes.c_double),
        ("vset_lo", ctypes.c_double),
        ("vset_hi", ctypes.c_double),
        ("pload_hi", ctypes.c_double),
        ("qp_lo", ctypes.c_double),
        ("qp_hi", ctypes.c_double),
        ("gen_factor", ctypes.c_double),
        ("loading", ctypes.c_double),
        ("seed", ctypes.c_uint64),
    ]


class Options(ctypes.Structure):
    _fields_ = [
        ("max_it_nr", ctypes.c_int32),
        ("max_it_fd", ctypes.c_int32),
        ("tol", ctypes.c_double),
        ("angle_mode", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("use_graph", ctypes.c_int32),
        ("autotune", ctypes.c_int32),
        ("ordering", ctypes.c_int32),
        ("reserved", ctypes.c_int32 * 3),
    ]


class Timing(ctypes.Structure):
    _fields_ = [
        ("total_ms", ctypes.c_double),
        ("mismatch_ms", ctypes.c_double),
        ("jacobian_ms", ctypes.c_double),
        ("factor_ms", ctypes.c_double),
        ("solve_ms", ctypes.c_double),
        ("update_ms", ctypes.c_double),
        ("other_ms", ctypes.c_double),
        ("iterations_max", ctypes.c_int32),
        ("launches", ctypes.c_int32),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("n_bus", ctypes.c_int32),
        ("n_branch", ctypes.c_int32),
        ("n_pv", ctypes.c_int32),
        ("n_pq", ctypes.c_int32),
        ("n_slack", ctypes.c_int32),
        ("nnz_ybus", ctypes.c_int32),
        ("n_jac", ctypes.c_int32),
        ("nnz_jac", ctypes.c_int32),
        ("nnz_lu", ctypes.c_int32),
        ("lu_levels", ctypes.c_int32),
        ("lu_flops", ctypes.c_int64),
        ("n_bp", ctypes.c_int32),
        ("nnz_bp_lu", ctypes.c_int32),
        ("bp_levels", ctypes.c_int32),
        ("n_bpp", ctypes.c_int32),
        ("nnz_bpp_lu", ctypes.c_int32),
        ("bpp_levels", ctypes.c_int32),
        ("n_cases", ctypes.c_int32),
        ("case_groups", ctypes.c_int32),
        ("device_bytes", ctypes.c_int64),
        ("nnz_lu_upper", ctypes.c_int64),
        ("ordering", ctypes.c_int32),
        ("pad_", ctypes.c_int32),
    ]
