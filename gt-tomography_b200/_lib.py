"""ctypes binding of libcbct.so (the C ABI declared in include/cbct.h).

The shared library is built in-tree by gt-tomography_b200/build.py.  A missing
library is an error: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libcbct.so")

CBCT_F32, CBCT_F16, CBCT_BF16 = 0, 1, 2

CBCT_BP_OFFSET_WEIGHT = 0x1
CBCT_BP_FDK_WEIGHT = 0x2
CBCT_FDK_COSINE = 0x1
CBCT_FDK_PARKER = 0x2
CBCT_FDK_OFFSET = 0x4
CBCT_FDK_RAMP = 0x8
CBCT_OPT_DEBUG_CHECKS = 1
CBCT_OPT_FORCE_GATHER = 2
CBCT_OPT_FORWARD_KERNEL = 3
CBCT_OPT_WAIT_LIMIT = 4
CBCT_OPT_STATUS_CHECK = 5
CBCT_ERR_INVALID_ARGUMENT = 1
CBCT_ERR_CUDA = 2
CBCT_ERR_OUT_OF_MEMORY = 3
CBCT_ERR_UNSUPPORTED = 4
CBCT_ERR_DEVICE_CHECK = 5
CBCT_ERR_TIMEOUT = 6
CBCT_ERR_BUDGET = 7
CBCT_ERR_CANCELLED = 8
CBCT_ERR_INTERNAL = 9

# Every symbol the header declares (checked by the CPU tests).
EXPORTED = [
    "cbct_status_string", "cbct_last_error", "cbct_version", "cbct_subset_partition",
    "cbct_default_frequency_filter", "cbct_cosine_weights", "cbct_is_short_scan",
    "cbct_offset_override", "cbct_plan_create", "cbct_plan_destroy", "cbct_plan_subset",
    "cbct_plan_forward_variant", "cbct_plan_set_option", "cbct_plan_read_flags", "cbct_plan_check", "cbct_microbench_interp",
    "cbct_forward",
    "cbct_backproject", "cbct_offset_correct", "cbct_fdk_filter", "cbct_fdk",
    "cbct_forward_residual", "cbct_osmom_precon", "cbct_osmom_step", "cbct_osmom_update", "cbct_reduce_f64", "cbct_reduce_f64_noalloc",
    "cbct_osmom_solve",
    "cbct_ossart_solve", "cbct_batch_osmom", "cbct_batch_osmom_fused", "cbct_phantom_voxelize", "cbct_phantom_project", "cbct_convert",
    "cbct_spacecarver", "cbct_apply_mask", "cbct_plan_set_mask", "cbct_plan_set_projection_weights",
    "cbct_fdk_filter_ex", "cbct_fdk_ex", "cbct_host_forward", "cbct_host_backproject", "cbct_plan_set_bins",
    "cbct_tv_step", "cbct_plan_autotune",
    "cbct_server_create", "cbct_server_request_bytes", "cbct_server_submit", "cbct_server_wait",
    "cbct_server_now", "cbct_server_destroy",
]
# The plain reference-replica path (include/cbct_plain.h), a measurement baseline.
EXPORTED_PLAIN = ["cbct_plain_forward", "cbct_plain_backproject", "cbct_plain_osmom_solve", "cbct_plain_fdk",
                  "cbct_plain_kernel_times"]


class CbctGeometry(C.Structure):
    _fields_ = [("SAD", C.c_float), ("SDD", C.c_float), ("fov_u", C.c_float), ("fov_v", C.c_float),
                ("width", C.c_int32), ("height", C.c_int32),
                ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("lx", C.c_float), ("ly", C.c_float), ("lz", C.c_float),
                ("samples_per_pixel", C.c_float)]


class CbctSolverParams(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("beta", C.c_float), ("gamma", C.c_float),
                ("non_negativity", C.c_int32), ("use_graph", C.c_int32), ("storage", C.c_int32),
                ("refine_every", C.c_int32), ("proj_storage", C.c_int32), ("tv_weight", C.c_float),
                ("tv_alpha", C.c_float), ("tau", C.c_float), ("reg_steps", C.c_int32)]


class CbctBatchItem(C.Structure):
    _fields_ = [("plan", C.c_void_p), ("b", C.c_void_p), ("x0", C.c_void_p), ("z_out", C.c_void_p),
                ("params", CbctSolverParams), ("resid_norm2_out", C.c_void_p)]


CBCT_REQ_FDK, CBCT_REQ_OSMOM = 0, 1


class CbctServerConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_size_t), ("max_inflight", C.c_int32), ("device", C.c_int32)]


class CbctRequest(C.Structure):
    _fields_ = [("kind", C.c_int32), ("geometry", CbctGeometry), ("angles_deg", C.c_void_p),
                ("offsets_xy", C.c_void_p), ("n_views", C.c_int32), ("n_subsets", C.c_int32),
                ("storage", C.c_int32), ("proj_host", C.c_void_p), ("vol_host", C.c_void_p),
                ("params", CbctSolverParams), ("filter", C.c_void_p), ("fdk_flags", C.c_uint32),
                ("offset_correction", C.c_int32)]


class CbctRequestInfo(C.Structure):
    _fields_ = [("status", C.c_int), ("slot", C.c_int32), ("t_submit", C.c_double), ("t_admit", C.c_double),
                ("t_done", C.c_double), ("bytes_reserved", C.c_size_t), ("bytes_peak", C.c_size_t),
                ("message", C.c_char * 256)]


class CbctError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: {status_string(status)}: {msg}")
        self.status = status


_lib: C.CDLL | None = None

_vp = C.c_void_p
_i32 = C.c_int32
_u32 = C.c_uint32
_f = C.c_float
_sz = C.c_size_t
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)
_gp = C.POINTER(CbctGeometry)

_SIGS = {
    "cbct_status_string": (C.c_char_p, [C.c_int]),
    "cbct_last_error": (C.c_char_p, []),
    "cbct_version": (C.c_char_p, []),
    "cbct_subset_partition": (C.c_int, [_i32, _vp, _i32, _vp, _vp, _vp]),
    "cbct_default_frequency_filter": (C.c_int, [_i32, _vp]),
    "cbct_cosine_weights": (C.c_int, [_gp, _vp]),
    "cbct_is_short_scan": (C.c_int, [_gp, _vp, _i32, _vp]),
    "cbct_offset_override": (C.c_int, [_gp, _vp, _i32, _vp]),
    "cbct_plan_create": (C.c_int, [_gp, _vp, _vp, _i32, _vp, _i32, _vp, C.POINTER(_vp)]),
    "cbct_plan_destroy": (C.c_int, [_vp]),
    "cbct_plan_subset": (C.c_int, [_vp, _i32, _vp, _vp]),
    "cbct_plan_forward_variant": (C.c_char_p, [_vp]),
    "cbct_plan_set_option": (C.c_int, [_vp, _i32, _i32]),
    "cbct_plan_read_flags": (C.c_int, [_vp, _vp, _i32]),
    "cbct_plan_check": (C.c_int, [_vp, _vp]),
    "cbct_microbench_interp": (C.c_int, [_i32, _i32, C.POINTER(C.c_double), _vp]),
    "cbct_forward": (C.c_int, [_vp, _i32, C.c_int, _vp, _vp, _i32, _vp]),
    "cbct_backproject": (C.c_int, [_vp, _i32, _vp, _vp, _u32, _i32, _i32, _vp]),
    "cbct_offset_correct": (C.c_int, [_vp, _i32, _vp, _i32, _vp]),
    "cbct_fdk_filter": (C.c_int, [_vp, _i32, _vp, _vp, _vp, _u32, _vp]),
    "cbct_fdk": (C.c_int, [_vp, _vp, _vp, _vp, _u32, _vp, _vp]),
    "cbct_forward_residual": (C.c_int, [_vp, _i32, C.c_int, _vp, _vp, _vp, _f, _i32, _vp, _vp]),
    "cbct_osmom_precon": (C.c_int, [_vp, _vp, _vp]),
    "cbct_osmom_step": (C.c_int, [_vp, _i32, C.c_int, _vp, _vp, _vp, _vp, _vp, _f, _f, _i32, _vp, _vp]),
    "cbct_osmom_update": (C.c_int, [_vp, _vp, _vp, _vp, _sz, _f, _f, _i32, _vp]),
    "cbct_reduce_f64": (C.c_int, [_i32, _vp, _vp, _sz, _vp, _vp]),
    "cbct_reduce_f64_noalloc": (C.c_int, [_i32, _vp, _vp, _sz, _vp, _vp]),
    "cbct_osmom_solve": (C.c_int, [_vp, _vp, _vp, _vp, C.POINTER(CbctSolverParams), _vp, _vp]),
    "cbct_ossart_solve": (C.c_int, [_vp, _vp, _vp, _vp, C.POINTER(CbctSolverParams), _vp, _vp]),
    "cbct_batch_osmom": (C.c_int, [C.POINTER(CbctBatchItem), _i32, _i32, _vp]),
    "cbct_batch_osmom_fused": (C.c_int, [C.POINTER(CbctBatchItem), _i32, _vp]),
    "cbct_phantom_voxelize": (C.c_int, [_gp, _vp, _i32, _i32, _vp, _vp]),
    "cbct_phantom_project": (C.c_int, [_vp, _i32, _vp, _i32, _vp, _vp]),
    "cbct_convert": (C.c_int, [_vp, _vp, _sz, C.c_int, _vp]),
    "cbct_spacecarver": (C.c_int, [_vp, _i32, _vp, _f, _vp, _i32, _vp]),
    "cbct_apply_mask": (C.c_int, [_vp, _vp, _sz, _vp]),
    "cbct_plan_set_mask": (C.c_int, [_vp, _vp]),
    "cbct_plan_set_projection_weights": (C.c_int, [_vp, _vp]),
    "cbct_fdk_filter_ex": (C.c_int, [_vp, _i32, C.c_int, _vp, _vp, _vp, _u32, _vp]),
    "cbct_fdk_ex": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp, _u32, _vp, _vp]),
    "cbct_host_forward": (C.c_int, [_vp, _i32, _i32, _vp, _vp, _vp, _i32, _vp]),
    "cbct_plan_set_bins": (C.c_int, [_vp, _i32, _vp]),
    "cbct_tv_step": (C.c_int, [_vp, _vp, _vp, _vp, _i32, _i32, _i32, _f, _f, _f, _vp]),
    "cbct_plan_autotune": (C.c_int, [_vp, _vp, _vp]),
    "cbct_host_backproject": (C.c_int, [_vp, _i32, _i32, _vp, _vp, _vp, _i32, _vp, _u32, _i32, _f, _i32, _vp]),
    "cbct_server_create": (C.c_int, [C.POINTER(CbctServerConfig), C.POINTER(_vp)]),
    "cbct_server_request_bytes": (C.c_int, [C.POINTER(CbctRequest), C.POINTER(_sz)]),
    "cbct_server_submit": (C.c_int, [_vp, C.POINTER(CbctRequest), C.POINTER(C.c_uint64)]),
    "cbct_server_wait": (C.c_int, [_vp, C.c_uint64, C.c_double, C.POINTER(CbctRequestInfo)]),
    "cbct_server_now": (C.c_int, [_vp, C.POINTER(C.c_double)]),
    "cbct_server_destroy": (C.c_int, [_vp]),
    "cbct_plain_forward": (C.c_int, [_gp, _vp, _vp, _i32, _vp, _vp, _i32]),
    "cbct_plain_backproject": (C.c_int, [_gp, _vp, _vp, _i32, _vp, _vp, _i32, _i32]),
    "cbct_plain_osmom_solve": (C.c_int, [_gp, _vp, _vp, _i32, _vp, _i32, _vp, _vp, _vp, _i32, _i32, _vp]),
    "cbct_plain_fdk": (C.c_int, [_gp, _vp, _vp, _i32, _vp, _vp, _vp, _i32, _i32]),
    "cbct_plain_kernel_times": (C.c_int, [_gp, _vp, _vp, _i32, _vp, _vp, _vp, _vp, _i32, _vp]),
}


def lib() -> C.CDLL:
    """Loads libcbct.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python gt-tomography_b200/build.py` "
                "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def status_string(st: int) -> str:
    return lib().cbct_status_string(st).decode()


def check(st: int, where: str):
    if st != 0:
        raise CbctError(st, where, lib().cbct_last_error().decode())


def call(name: str, *args):
    check(getattr(lib(), name)(*args), name)
