"""Loading libv2m_cuda.so (built in-tree by trussnet_b200.build) and its C ABI.

There is no fallback: if the library is missing or fails to load, every call
raises. The library itself returns V2M_ERR_CUDA when no CUDA device is usable.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

from .types import GridView, NodesView, RelaxParamsC, RelaxStatsC

HERE = os.path.dirname(os.path.abspath(__file__))
# V2M_CUDA_LIBRARY selects another build of the library: libv2m_cuda_check.so,
# the one with device bounds checks, for checked runs
LIB_PATH = os.environ.get("V2M_CUDA_LIBRARY") or os.path.join(HERE, "libv2m_cuda.so")

V2M_OK, V2M_ERR_ARG, V2M_ERR_CUDA, V2M_ERR_KERNEL, V2M_ERR_STATE = 0, -1, -2, -3, -4

# every symbol include/v2m_cuda.h declares
EXPORTS = [
    "v2m_relax_params_default", "v2m_cuda_last_error", "v2m_cuda_device_count", "v2m_relax_cuda",
    "v2m_relax_cuda_batch", "v2m_session_create", "v2m_session_destroy", "v2m_session_reset", "v2m_session_rebuild",
    "v2m_session_force", "v2m_session_step_tail", "v2m_session_iterate", "v2m_session_run", "v2m_session_synchronize",
    "v2m_session_read_nodes", "v2m_session_stats", "v2m_session_read_array", "v2m_session_write_array",
    "v2m_session_write_lists", "v2m_session_info", "v2m_session_counters", "v2m_session_timed_runs",
    "v2m_session_clear_counters", "v2m_unroll_create", "v2m_unroll_destroy", "v2m_unroll_forward",
    "v2m_unroll_loss", "v2m_unroll_loss_backward", "v2m_unroll_backward", "v2m_unroll_tape", "v2m_unroll_timing",
    "v2m_unroll_set_constraints",
    "v2m_unroll_last_error", "v2m_session_autotune", "v2m_session_shapes",
    "v2m_session_profile_stages", "v2m_session_queue_sizes", "v2m_bin_sort_noalloc", "v2m_bin_sort_noalloc_error",
    "v2m_validate_lists", "v2m_grid_params_default", "v2m_grid_build_cuda", "v2m_grid_result_view",
    "v2m_grid_result_info", "v2m_grid_free", "v2m_points_cuda",
    "v2m_seed_cuda", "v2m_seed_copy", "v2m_seed_free",
]

_lock = threading.Lock()
_lib = None


class V2mError(RuntimeError):
    """A failed library call (the reference's relax_cl throws std::runtime_error)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"v2m_cuda error {code}: {msg}")
        self.code = code


def load(path: str = LIB_PATH) -> C.CDLL:
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise V2mError(V2M_ERR_CUDA, f"{path} is not built (python -m trussnet_b200.build)")
        L = C.CDLL(path)
        vp = C.c_void_p
        P = C.POINTER
        L.v2m_cuda_last_error.restype = C.c_char_p
        L.v2m_relax_params_default.argtypes = [P(RelaxParamsC)]
        L.v2m_relax_params_default.restype = None
        L.v2m_relax_cuda.argtypes = [P(GridView), P(RelaxParamsC), P(NodesView), P(RelaxStatsC), C.c_int]
        L.v2m_relax_cuda_batch.argtypes = [C.c_int, P(GridView), P(RelaxParamsC), P(NodesView), P(RelaxStatsC),
                                           C.c_int]
        L.v2m_session_create.argtypes = [C.c_int, P(GridView), P(RelaxParamsC), P(NodesView), C.c_int, P(vp)]
        for f in ("v2m_session_destroy", "v2m_session_reset", "v2m_session_rebuild", "v2m_session_force",
                  "v2m_session_step_tail", "v2m_session_synchronize"):
            getattr(L, f).argtypes = [vp]
        L.v2m_session_iterate.argtypes = [vp, C.c_int, C.c_int]
        L.v2m_session_run.argtypes = [vp, C.c_int]
        L.v2m_session_read_nodes.argtypes = [vp, C.c_int, P(NodesView)]
        L.v2m_session_stats.argtypes = [vp, C.c_int, P(RelaxStatsC)]
        L.v2m_session_read_array.argtypes = [vp, C.c_int, C.c_int, vp, C.c_int64]
        L.v2m_session_write_array.argtypes = [vp, C.c_int, C.c_int, vp, C.c_int64]
        L.v2m_session_write_lists.argtypes = [vp, C.c_int, vp, vp]
        L.v2m_session_info.argtypes = [vp, C.c_int, P(C.c_int64), P(C.c_int64), P(C.c_int32)]
        L.v2m_session_counters.argtypes = [vp, P(C.c_int64), P(C.c_int64), P(C.c_double)]
        L.v2m_session_timed_runs.argtypes = [vp, C.c_int, C.c_int, C.c_int, P(C.c_float)]
        L.v2m_session_clear_counters.argtypes = [vp]
        L.v2m_unroll_last_error.restype = C.c_char_p
        L.v2m_session_autotune.argtypes = [vp, C.c_int, C.c_char_p, C.c_int64]
        L.v2m_session_shapes.argtypes = [vp, P(C.c_int32), P(C.c_int32)]
        L.v2m_session_profile_stages.argtypes = [vp, C.c_int, vp]
        L.v2m_session_queue_sizes.argtypes = [vp, P(C.c_int32), P(C.c_int32)]
        L.v2m_bin_sort_noalloc.argtypes = [vp, C.c_int64, C.c_int64, vp, vp, vp]
        L.v2m_validate_lists.argtypes = [C.c_int64, vp, vp, vp, vp, C.c_char_p, C.c_int64]
        L.v2m_grid_params_default.argtypes = [vp]
        L.v2m_grid_params_default.restype = None
        L.v2m_grid_build_cuda.argtypes = [vp, C.c_int32, C.c_int32, C.c_int32, vp, vp, C.c_int, vp]
        L.v2m_grid_result_view.argtypes = [vp, vp]
        L.v2m_grid_result_info.argtypes = [vp, vp, vp, vp, vp]
        L.v2m_points_cuda.argtypes = [vp, C.c_int32, C.c_int32, C.c_int32, vp, vp, vp, C.c_int, vp, vp, vp]
        L.v2m_grid_free.argtypes = [vp]
        L.v2m_grid_free.restype = None
        L.v2m_bin_sort_noalloc_error.restype = C.c_char_p
        L.v2m_seed_cuda.argtypes = [P(GridView), P(RelaxParamsC), C.c_int, P(vp), P(C.c_int64)]
        L.v2m_seed_copy.argtypes = [vp, vp, vp, vp, vp, vp]
        L.v2m_seed_free.argtypes = [vp]
        L.v2m_seed_free.restype = None
        L.v2m_unroll_create.argtypes = [C.c_int64, vp, vp, vp, vp, vp, C.c_float, C.c_float, C.c_float, C.c_int,
                                        C.c_int, C.c_int, P(vp)]
        L.v2m_unroll_destroy.argtypes = [vp]
        L.v2m_unroll_forward.argtypes = [vp, vp, vp, vp, C.c_int]
        L.v2m_unroll_loss.argtypes = [vp, vp, vp, P(C.c_double)]
        L.v2m_unroll_loss_backward.argtypes = [vp, vp, vp, C.c_float, vp, vp, C.c_int]
        L.v2m_unroll_backward.argtypes = [vp, vp, vp, vp, vp, vp]
        L.v2m_unroll_tape.argtypes = [vp, vp, C.c_int64]
        L.v2m_unroll_set_constraints.argtypes = [vp, vp]
        L.v2m_unroll_timing.argtypes = [vp, P(C.c_float), P(C.c_float)]
        _lib = L
        return L


def check(rc: int) -> None:
    if rc != V2M_OK:
        msg = load().v2m_cuda_last_error().decode(errors="replace")
        raise V2mError(rc, msg)


def check_unroll(rc: int) -> None:
    if rc != V2M_OK:
        msg = load().v2m_unroll_last_error().decode(errors="replace")
        raise V2mError(rc, msg)
