"""ctypes binding of libmpf.so (include/mpf.h).

The library is the product: nothing here falls back to Python or CPU code.  If
libmpf.so is missing the import of an entry point raises, naming the build step.
"""
import ctypes
import os

from . import _types as T

_HERE = os.path.dirname(os.path.abspath(__file__))
# MPF_LIB_PATH: load another build of the same library (e.g. to compare two builds)
LIB_PATH = os.environ.get("MPF_LIB_PATH") or os.path.join(_HERE, "libmpf.so")

_lib = None

c_p = ctypes.c_void_p
c_i32 = ctypes.c_int32
c_u64 = ctypes.c_uint64
c_dbl = ctypes.c_double

_SIGNATURES = {
    "mpf_abi_version": (c_i32, []),
    "mpf_default_options": (None, [ctypes.POINTER(T.Options)]),
    "mpf_status_string": (ctypes.c_char_p, [c_i32]),
    "mpf_create": (c_i32, [c_p, c_i32, c_p, c_i32, ctypes.POINTER(T.Options), ctypes.POINTER(c_p)]),
    "mpf_destroy": (c_i32, [c_p]),
    "mpf_last_error": (ctypes.c_char_p, [c_p]),
    "mpf_get_stats": (c_i32, [c_p, ctypes.POINTER(T.Stats)]),
    "mpf_set_cases": (c_i32, [c_p, c_i32, c_p, c_p, c_p]),
    "mpf_set_controls": (c_i32, [c_p, c_i32, c_p, c_p]),
    "mpf_set_cases_islands": (c_i32, [c_p, c_i32, c_p, c_p, c_p, c_p]),
    "mpf_set_q_limits": (c_i32, [c_p, c_p, c_p]),
    "mpf_get_bus_types": (c_i32, [c_p, c_p]),
    "mpf_solve": (c_i32, [c_p, c_i32, c_i32, c_p]),
    "mpf_get_results": (c_i32, [c_p, c_p, c_p, c_p, c_p]),
    "mpf_get_results_device": (c_i32, [c_p, c_p, c_p, c_p, c_p, c_p]),
    "mpf_runpf_host": (c_i32, [c_p, c_i32, c_i32, c_i32, c_p, c_p, c_p, c_p, c_p, c_p, c_p]),
    "mpf_get_timing": (c_i32, [c_p, ctypes.POINTER(T.Timing)]),
    "mpf_mismatch": (c_i32, [c_p, c_p, c_p, c_p]),
    "mpf_mismatch_noalloc": (c_i32, [c_p, c_p, c_p, c_p]),
    "mpf_set_ratings": (c_i32, [c_p, c_p]),
    "mpf_branch_flows": (c_i32, [c_p, c_p, c_p, c_p, c_p, c_p]),
    "mpf_adjoint": (c_i32, [c_p, c_i32, c_p, c_p, c_p, c_p, c_p]),
    "mpf_synth_default": (None, [ctypes.POINTER(T.SynthParams)]),
    "mpf_synth_grid": (c_i32, [ctypes.POINTER(T.SynthParams), c_p, c_p]),
    "mpf_find_bridges": (c_i32, [c_p, c_i32, c_i32, c_p]),
    "mpf_select_outages": (c_i32, [c_p, c_i32, c_i32, c_i32, c_u64, c_p]),
    "mpf_synth_load_scenarios": (c_i32, [c_p, c_i32, c_i32, c_dbl, c_u64, c_p]),
}


class MpfError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"mpf error {code}: {msg}")
        self.code = code


def lib():
    """Loads libmpf.so once; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m mapol_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return list(_SIGNATURES)


def ptr(a):
    """Data pointer of a numpy array (or None)."""
    return None if a is None else a.ctypes.data_as(c_p)
