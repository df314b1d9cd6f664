"""ctypes binding of the C ABI declared in include/amrclaw_b200.h."""
from __future__ import annotations

import ctypes
import os

from .build import LIB

_lib = None

c_int_p = ctypes.POINTER(ctypes.c_int)
c_double_p = ctypes.POINTER(ctypes.c_double)
c_ll_p = ctypes.POINTER(ctypes.c_longlong)

SIGNATURES = {
    "amrgpu_last_error": (ctypes.c_char_p, []),
    "amrgpu_init": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "amrgpu_init_precision": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                             ctypes.POINTER(ctypes.c_void_p)]),
    "amrgpu_set_batched": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "amrgpu_set_profile": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "amrgpu_set_graphs": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "amrgpu_set_schedule": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "amrgpu_set_solver": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, c_double_p, ctypes.c_int]),
    "amrgpu_set_pool_limit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong]),
    "amrgpu_set_step_batching": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "amrgpu_checkpoint": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p]),
    "amrgpu_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "amrgpu_level_advance": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_double_p, c_double_p]),
    "amrgpu_level_advance_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_double_p, c_double_p]),
    "amrgpu_update": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "amrgpu_regrid": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "amrgpu_valout": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p]),
    "amrgpu_mass": (ctypes.c_int, [ctypes.c_void_p, c_double_p]),
    "amrgpu_info": (ctypes.c_int, [ctypes.c_void_p, c_double_p, ctypes.c_int]),
    "amrgpu_grids": (ctypes.c_int, [ctypes.c_void_p, c_int_p, ctypes.c_int, c_int_p]),
    "amrgpu_values": (ctypes.c_int, [ctypes.c_void_p, c_double_p, ctypes.c_longlong, c_ll_p]),
    "amrgpu_gauges": (ctypes.c_int, [ctypes.c_void_p, c_double_p, ctypes.c_int, c_int_p]),
    "amrgpu_num_dim": (ctypes.c_int, [ctypes.c_void_p]),
    "amrgpu_destroy": (ctypes.c_int, [ctypes.c_void_p]),
}


def load(path: str = LIB) -> ctypes.CDLL:
    """Load the in-tree CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError("amrclaw_b200: CUDA library %s is missing; run amrclaw_b200.build.build()" % path)
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib
