"""ctypes bindings of libstophys_b200.so (the C ABI in include/stophys_b200.h).

The library is built in-tree by :func:`stochasticphysics_b200.build.build`.  There
is no fallback: if the shared library is missing or no CUDA device is present
the calls raise.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

from ._abi import (sp_ensemble_desc, sp_launch_config, sp_particles, sp_result, sp_server_config, sp_stats, Status)

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libstophys_b200.so"

SYMBOLS = [
    "sp_last_error", "sp_abi_version", "sp_query_dims", "sp_validate", "sp_kernel_launch_count",
    "sp_create", "sp_destroy", "sp_simulate", "sp_ensemble_create", "sp_ensemble_advance",
    "sp_ensemble_steps_done", "sp_ensemble_read", "sp_ensemble_destroy", "sp_ensemble_footprint",
    "sp_server_create", "sp_server_submit", "sp_server_poll", "sp_server_wait", "sp_server_cancel",
    "sp_server_destroy", "sp_debug_philox_normals", "sp_measure_fma_peak", "sp_simulate_noalloc",
    "sp_autotune", "sp_launch_config_for", "sp_tuning_save", "sp_tuning_load", "sp_tuning_reset",
    "sp_provide_particles", "sp_ensemble_create_shaped", "sp_server_submit_many", "sp_merge_shards",
]

_lib = None


class SPError(RuntimeError):
    def __init__(self, status: int, message: str):
        try:
            name = Status(status).name
        except ValueError:
            name = str(status)
        super().__init__(f"{name}: {message}")
        self.status = status


def load():
    """Load the shared library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build the CUDA extension first "
                           "(python -c 'import __graft_entry__ as g; g.build()')")
    L = C.CDLL(str(LIB_PATH))
    vp, u64, i32, dp = C.c_void_p, C.c_uint64, C.c_int32, C.POINTER(C.c_double)
    L.sp_last_error.restype = C.c_char_p
    L.sp_abi_version.restype = C.c_uint32
    L.sp_kernel_launch_count.restype = u64
    L.sp_query_dims.argtypes = [i32, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32)]
    L.sp_validate.argtypes = [C.POINTER(sp_ensemble_desc)]
    L.sp_create.argtypes = [C.POINTER(vp), i32]
    L.sp_destroy.argtypes = [vp]
    L.sp_simulate.argtypes = [vp, C.POINTER(sp_ensemble_desc), C.POINTER(sp_result), C.POINTER(sp_stats)]
    L.sp_ensemble_create.argtypes = [vp, C.POINTER(sp_ensemble_desc), C.POINTER(vp)]
    L.sp_ensemble_create_shaped.argtypes = [vp, C.POINTER(sp_ensemble_desc), C.POINTER(sp_launch_config), C.POINTER(vp)]
    L.sp_ensemble_advance.argtypes = [vp, u64, vp]
    L.sp_ensemble_steps_done.argtypes = [vp, C.POINTER(u64), C.POINTER(u64)]
    L.sp_ensemble_read.argtypes = [vp, C.POINTER(sp_result), C.POINTER(sp_stats)]
    L.sp_ensemble_destroy.argtypes = [vp]
    L.sp_ensemble_footprint.argtypes = [C.POINTER(sp_ensemble_desc), C.POINTER(u64)]
    L.sp_server_create.argtypes = [vp, C.POINTER(sp_server_config), C.POINTER(vp)]
    L.sp_server_submit.argtypes = [vp, C.POINTER(sp_ensemble_desc), C.POINTER(u64)]
    L.sp_server_submit_many.argtypes = [vp, C.POINTER(sp_ensemble_desc), i32, C.POINTER(u64)]
    L.sp_server_poll.argtypes = [vp, u64, C.POINTER(i32)]
    L.sp_server_wait.argtypes = [vp, u64, C.c_double, C.POINTER(sp_result), C.POINTER(sp_stats), dp]
    L.sp_server_cancel.argtypes = [vp, u64]
    L.sp_server_destroy.argtypes = [vp]
    L.sp_debug_philox_normals.argtypes = [vp, u64, u64, u64, u64, u64, i32, i32, dp]
    L.sp_measure_fma_peak.argtypes = [vp, i32, dp]
    L.sp_simulate_noalloc.argtypes = [C.POINTER(sp_ensemble_desc), C.POINTER(sp_particles), dp, dp, vp]
    L.sp_autotune.argtypes = [vp, C.POINTER(sp_ensemble_desc), u64, C.POINTER(sp_launch_config),
                              C.POINTER(sp_launch_config), i32, C.POINTER(i32)]
    L.sp_launch_config_for.argtypes = [vp, C.POINTER(sp_ensemble_desc), C.POINTER(sp_launch_config)]
    L.sp_tuning_save.argtypes = [C.c_char_p]
    L.sp_tuning_load.argtypes = [C.c_char_p]
    L.sp_tuning_reset.argtypes = []
    L.sp_provide_particles.argtypes = [vp, C.POINTER(sp_ensemble_desc), dp]
    L.sp_merge_shards.argtypes = [i32, u64, i32, C.POINTER(dp), C.POINTER(dp), dp, dp, dp]
    for name in SYMBOLS:
        if name not in ("sp_last_error", "sp_abi_version", "sp_kernel_launch_count"):
            getattr(L, name).restype = C.c_int
    _lib = L
    return L


def check(status: int) -> None:
    if status != 0:
        msg = load().sp_last_error()
        raise SPError(status, msg.decode() if msg else "")
