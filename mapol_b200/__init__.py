"""mapol_b200 — B200-native batched AC power flow (Newton-Raphson, fast-decoupled
XB/BX) over many contingency cases at once, behind the C-ABI of include/mpf.h.

The compute path is libmpf.so (sm_100a CUDA); this package is its ctypes binding.
"""
from ._lib import MpfError, lib  # noqa: F401
from ._types import (BRANCH_DTYPE, BUS_DTYPE, CTRL_AVR, CTRL_OLTC, CTRL_SHC, EPS, FDBX, FDXB,  # noqa: F401
                     FP64, MAX_IT_FD, MAX_IT_NR, MIXED, NR)
from .grid import (find_bridges, load_scenarios, n1_cases, select_outages, synth_grid,  # noqa: F401
                   workload, WORKLOADS)
from .runpf import PowerFlow, Results, hybrid_free, hybrid_init, hybrid_runpf  # noqa: F401
from .multigrid import MultiGrid  # noqa: F401

__version__ = "0.1.0"
