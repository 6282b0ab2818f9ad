"""ctypes binding of the C ABI in include/custinger_tc.h (libcustinger_tc.so).

The library is loaded from this package directory only; a missing library raises instead of
falling back to anything else.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcustinger_tc.so")

TC_OK = 0
TC_ERR_INVALID_ARG = 1
TC_ERR_CUDA = 2
TC_ERR_OOM = 3
TC_ERR_BAD_GRAPH = 4
TC_ERR_NOT_SYMMETRIC = 5
TC_ERR_CAPACITY = 6
TC_ERR_TIMEOUT = 7
TC_ERR_STATE = 8

MLP_IN = 4
MLP_HIDDEN = 64
MLP_OUT = 3
MLP_PARAMS = MLP_HIDDEN * MLP_IN + MLP_HIDDEN + MLP_HIDDEN * MLP_HIDDEN + MLP_HIDDEN + MLP_OUT * MLP_HIDDEN + MLP_OUT

NOALLOC_MAX_NV = 1 << 20
NOALLOC_MAX_EDGES = 1 << 22

TC_PV_NONE = 0
TC_PV_HANDLE = 1
TC_PV_CSR = 2
TC_PV_HANDLE64 = 3

TC_MEM_DEVICE = 0
TC_MEM_HOST = 1

_P = ctypes.c_void_p
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64


class Sched(ctypes.Structure):
    _fields_ = [("warp_max_deg", _i32), ("search_ratio_x16", _i32), ("blocks_per_sm", _i32),
                ("chunk", _i32), ("use_table", _i32), ("table", (ctypes.c_uint8 * 16) * 16),
                ("shard", _i32), ("nshards", _i32), ("cell_filter", _i32), ("lane_max_deg", _i32),
                ("packed_max_deg", _i32), ("stream_hub_min", _i32)]


class CountInfo(ctypes.Structure):
    _fields_ = [("triangles", _i64), ("edges_intersected", _i64), ("oriented_work", _i64),
                ("max_out_degree", _i32), ("status", _i32), ("shard_lo", _i32), ("shard_hi", _i32),
                ("shard_work", _i64), ("total_work", _i64)]


class PhaseTimes(ctypes.Structure):
    _fields_ = [("orient_ms", ctypes.c_float), ("count_ms", ctypes.c_float), ("launches", _i32)]


class BatchInfo(ctypes.Structure):
    _fields_ = [("updates", _i64), ("inserted", _i64), ("deleted", _i64), ("ignored", _i64),
                ("triangles_added", _i64), ("triangles_removed", _i64), ("status", _i32)]


class PipelinePlan(ctypes.Structure):
    _fields_ = [("nbins", _i32), ("bin_cap", _i64 * 16), ("serve", _i32 * 16), ("ctas_per_sm", _i32 * 16),
                ("chunk", _i32 * 16), ("split_min", _i32 * 16)]


class TcError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


# Every exported function of the C ABI with (restype, argtypes). tests/ checks this table
# against the declarations in include/*.h.
SIGNATURES = {
    "tc_last_error": (ctypes.c_char_p, []),
    "tc_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "tc_sched_default": (None, [ctypes.POINTER(Sched)]),
    "tc_graph_create": (ctypes.c_int, [_i32, _P, _P, ctypes.c_int, ctypes.c_double, ctypes.c_int, _P,
                                       ctypes.POINTER(_P)]),
    "tc_graph_destroy": (ctypes.c_int, [_P]),
    "tc_graph_info": (ctypes.c_int, [_P, ctypes.POINTER(_i32), ctypes.POINTER(_i64), ctypes.POINTER(_i64)]),
    "tc_graph_export": (ctypes.c_int, [_P, _P, _P]),
    "tc_graph_validate": (ctypes.c_int, [_P, _P]),
    "tc_graph_device_view": (ctypes.c_int, [_P, ctypes.POINTER(_P), ctypes.POINTER(_P), ctypes.POINTER(_P)]),
    "tc_count_static": (ctypes.c_int, [_P, ctypes.c_int, _P, _P, ctypes.POINTER(CountInfo),
                                       ctypes.POINTER(Sched), _P]),
    "tc_count_csr32": (ctypes.c_int, [_i32, _P, _P, ctypes.c_int, _P, _P, ctypes.POINTER(CountInfo),
                                      ctypes.POINTER(Sched), _P]),
    "tc_count_csr64": (ctypes.c_int, [_i32, _P, _P, ctypes.c_int, _P, _P, ctypes.POINTER(CountInfo),
                                      ctypes.POINTER(Sched), _P]),
    "tc_workspace_status": (ctypes.c_int, [_P, ctypes.POINTER(CountInfo)]),
    "tc_workspace_release": (ctypes.c_int, []),
    "tc_shard_ranges": (ctypes.c_int, [_P, _i32, _i32, _P]),
    "tc_debug_alloc_cap": (ctypes.c_int, [_i64]),
    "tc_count_csr32_noalloc": (ctypes.c_int, [_i32, _P, _P, ctypes.c_int, _P, _P, ctypes.POINTER(CountInfo),
                                              ctypes.POINTER(Sched), _P]),
    "tc_apply_batch": (ctypes.c_int, [_P, _P, _P, _P, _i64, ctypes.c_int, _P, _P, ctypes.POINTER(BatchInfo),
                                      ctypes.POINTER(Sched), _P]),
    "tc_batch_sort": (ctypes.c_int, [_i32, _P, _P, _i64, _P, _P, _P]),
    "tc_insert_sorted": (ctypes.c_int, [_P, _P, _P, _i64, _P, ctypes.POINTER(_i64), _P]),
    "tc_delete_sorted": (ctypes.c_int, [_P, _P, _P, _P, _i64, _P]),
    "tc_count_batch": (ctypes.c_int, [_P, _P, _P, _P, _P, _i64, ctypes.c_int, _P, _P, ctypes.POINTER(Sched), _P]),
    "tc_autotune_static": (ctypes.c_int, [_P, ctypes.c_int, _P, _i32, ctypes.POINTER(Sched),
                                          ctypes.POINTER(ctypes.c_float), _P]),
    "tc_autotune_lookup": (ctypes.c_int, [_i32, _i64, _i32, ctypes.POINTER(Sched)]),
    "tc_autotune_save": (ctypes.c_int, [ctypes.c_char_p]),
    "tc_autotune_load": (ctypes.c_int, [ctypes.c_char_p]),
    "tc_cell_stats": (ctypes.c_int, [_P, _P, _P]),
    "tc_sched_learned": (ctypes.c_int, [_P, ctypes.c_int, _P, ctypes.POINTER(Sched), _P]),
    "tc_sched_from_costs": (ctypes.c_int, [ctypes.c_int, _P, _P, ctypes.POINTER(Sched)]),
    "tc_mlp_init": (ctypes.c_int, [_P, ctypes.c_uint64]),
    "tc_mlp_forward": (ctypes.c_int, [_P, _P, _i32, _P, _P]),
    "tc_mlp_backward": (ctypes.c_int, [_P, _P, _P, _P, _i32, _P, _P, _P]),
    "tc_mlp_adam_step": (ctypes.c_int, [_P, _P, _P, _P, _i32, ctypes.c_float, _P]),
    "tc_mlp_train": (ctypes.c_int, [_P, _P, _P, _P, _i32, _i32, ctypes.c_float, _P, _P]),
    "tc_pipeline_create": (ctypes.c_int, [_P, _i64, ctypes.POINTER(Sched), ctypes.POINTER(_P)]),
    "tc_pipeline_apply": (ctypes.c_int, [_P, _P, _P, _P, _i64, _P, _P, _P]),
    "tc_pipeline_prepare": (ctypes.c_int, [_P, _P, _P, _P]),
    "tc_pipeline_sync": (ctypes.c_int, [_P, ctypes.POINTER(BatchInfo)]),
    "tc_pipeline_autotune": (ctypes.c_int, [_P, _i32]),
    "tc_pipeline_info": (ctypes.c_int, [_P, _P, _P, _P]),
    "tc_pipeline_plan_get": (ctypes.c_int, [_P, _P]),
    "tc_pipeline_plan_set": (ctypes.c_int, [_P, _P]),
    "tc_pipeline_profile": (ctypes.c_int, [_P, ctypes.c_int]),
    "tc_pipeline_stats": (ctypes.c_int, [_P, ctypes.POINTER(_i64), ctypes.POINTER(ctypes.c_double),
                                         ctypes.POINTER(_i64)]),
    "tc_pipeline_set_wait_bound": (ctypes.c_int, [_P, ctypes.c_uint64, _i32]),
    "tc_pipeline_destroy": (ctypes.c_int, [_P]),
    "tc_profile_enable": (ctypes.c_int, [ctypes.c_int]),
    "tc_profile_last": (ctypes.c_int, [ctypes.POINTER(PhaseTimes)]),
}

_lib = None


def lib():
    """Load libcustinger_tc.so (raises when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m custingeralg_b200.build` "
                               "(or __graft_entry__.build()); there is no fallback path")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != TC_OK:
        msg = lib().tc_last_error()
        raise TcError(status, msg.decode() if msg else "")


def default_sched() -> Sched:
    s = Sched()
    lib().tc_sched_default(ctypes.byref(s))
    return s
