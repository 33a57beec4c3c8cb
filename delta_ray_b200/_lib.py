"""Loads libdr_b200.so (the CUDA renderer) and declares its C ABI.

There is no fallback: if the library is missing or no CUDA device is present,
``lib()`` raises.  Build it with ``python -m delta_ray_b200.build``.  The
environment variable ``DELTA_RAY_B200_LIB`` names another build of the same
library to load instead (e.g. one compiled with different nvcc flags).
"""
import ctypes as C
import os

from . import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("DELTA_RAY_B200_LIB") or os.path.join(HERE, "libdr_b200.so")
_lib = None


class DrError(RuntimeError):
    """A failed C ABI call; ``status`` holds the dr_status code."""

    def __init__(self, status, msg):
        super().__init__(f"delta_ray_b200 error {status}: {msg}")
        self.status = status


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing; build it with `python -m delta_ray_b200.build`")
    L = C.CDLL(LIB_PATH)
    L.dr_abi_version.restype = C.c_int
    L.dr_scene_create.argtypes = [C.POINTER(_abi.dr_scene_desc), C.c_int, C.POINTER(C.c_void_p)]
    L.dr_scene_update.argtypes = [C.c_void_p, C.POINTER(_abi.dr_scene_desc)]
    L.dr_scene_destroy.argtypes = [C.c_void_p]
    L.dr_scene_grad_layout.argtypes = [C.c_void_p, C.POINTER(_abi.dr_grad_layout)]
    L.dr_render_forward.argtypes = [C.c_void_p, C.POINTER(_abi.dr_render_desc), C.c_void_p, C.c_void_p]
    L.dr_render_backward.argtypes = [C.c_void_p, C.POINTER(_abi.dr_render_desc), C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p]
    L.dr_scene_last_launch_count.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
    L.dr_trace_rays.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]
    L.dr_eval_math.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]
    L.dr_scene_last_work.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
    L.dr_set_item_queue_limit.argtypes = [C.c_int64]
    L.dr_scene_edge_data.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int64, C.POINTER(C.c_int64),
                                     C.POINTER(C.c_float)]
    L.dr_scene_set_profiling.argtypes = [C.c_void_p, C.c_int]
    L.dr_scene_last_timings.argtypes = [C.c_void_p, C.c_int, C.c_char_p, C.c_size_t, C.POINTER(C.c_float)]
    L.dr_scene_last_counts.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.dr_last_error.argtypes = [C.c_char_p, C.c_size_t]
    L.dr_mlp_param_count.restype = C.c_int
    L.dr_scene_set_proposal.argtypes = [C.c_void_p, C.POINTER(_abi.dr_proposal_desc)]
    L.dr_render_backward_views.argtypes = [C.c_void_p, C.c_int, C.POINTER(_abi.dr_view_desc), C.c_void_p, C.c_void_p,
                                           C.c_void_p]
    L.dr_scene_proposal_state.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_int64)]
    L.dr_mlp_forward.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
    L.dr_mlp_gradient.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]
    L.dr_scene_get_tuning.argtypes = [C.c_void_p, C.POINTER(_abi.dr_tuning)]
    L.dr_scene_set_tuning.argtypes = [C.c_void_p, C.POINTER(_abi.dr_tuning)]
    L.dr_scene_autotune.argtypes = [C.c_void_p, C.POINTER(_abi.dr_render_desc), C.c_void_p, C.c_void_p, C.c_int,
                                    C.POINTER(_abi.dr_tune_report), C.c_void_p]
    L.dr_last_error.restype = C.c_size_t
    for name in ("dr_scene_create", "dr_scene_update", "dr_scene_destroy", "dr_scene_grad_layout",
                 "dr_render_forward", "dr_render_backward", "dr_scene_last_launch_count", "dr_trace_rays",
                 "dr_scene_set_profiling", "dr_scene_last_timings", "dr_scene_last_counts", "dr_eval_math",
                 "dr_scene_edge_data", "dr_scene_last_work",
                 "dr_set_item_queue_limit", "dr_scene_get_tuning", "dr_scene_set_tuning", "dr_scene_autotune"):
        getattr(L, name).restype = C.c_int
    if L.dr_abi_version() != 2:
        raise ImportError("libdr_b200.so has an unexpected ABI version")
    _lib = L
    return L


def last_error():
    buf = C.create_string_buffer(1024)
    lib().dr_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status):
    if status != 0:
        raise DrError(status, last_error())
