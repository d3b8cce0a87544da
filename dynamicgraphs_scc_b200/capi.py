"""ctypes binding of the engine's C ABI (include/scc_capi.h, include/scc_gen_api.h).

The library is loaded from the package's lib/ folder.  There is no fallback:
if the native library is missing, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libscc_b200.so")

SCC_OK = 0
STATUS_NAMES = {
    0: "SCC_OK", 1: "SCC_ERR_INVALID", 2: "SCC_ERR_CUDA", 3: "SCC_ERR_OOM", 4: "SCC_ERR_TIMEOUT",
    5: "SCC_ERR_STATE", 6: "SCC_ERR_IO", 7: "SCC_ERR_NOT_FOUND", 8: "SCC_ERR_UNSUPPORTED", 9: "SCC_ERR_BUSY",
}
SCC_ERR_BUSY = 9
SCC_BUILD_KEEP_ALL = 0
SCC_BUILD_DEDUP = 1
SCC_BUILD_NO_SELF_LOOPS = 2
SCC_COLOR_INIT = -1
SCC_COLOR_DONE = -2
SCC_NIL_NODE = -1


class SccError(RuntimeError):
    def __init__(self, status: int, func: str, msg: str):
        self.status = status
        super().__init__(f"{func}: {STATUS_NAMES.get(status, status)}: {msg}")


class RunStats(C.Structure):
    _fields_ = [
        ("ms_total", C.c_double), ("ms_trim1", C.c_double), ("ms_global_fb", C.c_double),
        ("ms_trim12", C.c_double), ("ms_wcc", C.c_double), ("ms_fb", C.c_double),
        ("trimmed_first", C.c_int32), ("first_scc_size", C.c_int32), ("trimmed_second", C.c_int32),
        ("num_sccs", C.c_int32), ("num_wcc_classes", C.c_int32), ("fb_rounds", C.c_int32),
        ("traversal_steps", C.c_int64), ("kernels_launched", C.c_int32), ("pivot_mode", C.c_int32),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class UpdateStats(C.Structure):
    _fields_ = [
        ("ms_total", C.c_double), ("ms_merge", C.c_double), ("ms_delete", C.c_double), ("ms_insert", C.c_double),
        ("affected_delete", C.c_int32), ("affected_insert", C.c_int32), ("m_after", C.c_int64),
        ("num_sccs", C.c_int32),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class RequestResult(C.Structure):
    _fields_ = [("status", C.c_int), ("session", C.c_int32), ("latency_ms", C.c_double), ("queue_ms", C.c_double),
                ("update", UpdateStats)]


class ServerStats(C.Structure):
    _fields_ = [("completed", C.c_int64), ("rejected", C.c_int64), ("updates", C.c_int64),
                ("max_inflight", C.c_int64), ("bytes_in_use", C.c_int64), ("p50_ms", C.c_double),
                ("p99_ms", C.c_double), ("max_ms", C.c_double), ("updates_per_s", C.c_double),
                ("groups", C.c_int64), ("offered_edges", C.c_int64), ("shed", C.c_int64), ("shed_edges", C.c_int64),
                ("expired", C.c_int64), ("max_queued_edges", C.c_int64), ("offered_per_s", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Tuning(C.Structure):
    _fields_ = [(k, C.c_int32) for k in ("bu_alpha", "bu_div", "async_max", "async_after", "async_keep",
                                         "async_blocks_per_sm", "huge_deg", "tile_min_live", "tile_min_span",
                                         "pivot_salt", "tail_live", "tail_class", "cta_deg")]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class BatchTuning(C.Structure):
    _fields_ = [("threads", C.c_int32), ("blocks_per_sm", C.c_int32), ("warp_deg", C.c_int32)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class BatchStats(C.Structure):
    _fields_ = [("ms_total", C.c_double), ("graphs", C.c_int32), ("rounds", C.c_int32), ("levels", C.c_int32),
                ("max_rounds", C.c_int32), ("host_submissions", C.c_int32), ("kernels", C.c_int32)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class GenParams(C.Structure):
    _fields_ = [
        ("rmat_scale", C.c_int), ("edge_factor", C.c_int), ("grid_side", C.c_int), ("num_cycles", C.c_int),
        ("cycle_min", C.c_int), ("cycle_max", C.c_int), ("seed", C.c_uint64),
    ]


class BatchParams(C.Structure):
    _fields_ = [("num_graphs", C.c_int32), ("n_min", C.c_int32), ("n_max", C.c_int32), ("mean_degree", C.c_double),
                ("rmat_fraction", C.c_double), ("seed", C.c_uint64)]


_P = C.c_void_p
_I32P = C.POINTER(C.c_int32)
_I64P = C.POINTER(C.c_int64)
_F32P = C.POINTER(C.c_float)

# name -> argtypes (all return int status unless listed in _RESTYPES)
_SIGS = {
    "scc_status_string": [C.c_int],
    "scc_last_error": [],
    "scc_version": [],
    "scc_device_count": [C.POINTER(C.c_int)],
    "scc_graph_create_edges": [C.c_int32, C.c_int64, _I32P, _I32P, C.c_int, C.c_int, C.POINTER(_P)],
    "scc_graph_create_edges_device": [C.c_int32, C.c_int64, _P, _P, C.c_int, C.c_int, C.POINTER(_P)],
    "scc_graph_create_csr": [C.c_int32, C.c_int32, _I32P, _I32P, _I32P, _I32P, C.c_int, C.POINTER(_P)],
    "scc_graph_create_csr_device": [C.c_int32, C.c_int32, _P, _P, _P, _P, C.c_int, C.POINTER(_P)],
    "scc_graph_load_edge_list": [C.c_char_p, C.c_int, C.POINTER(_P)],
    "scc_graph_upload_csr": [_P, _P, _P, _P, _P, _P],
    "scc_graph_free": [_P],
    "scc_graph_num_nodes": [_P, _I32P],
    "scc_graph_num_edges": [_P, _I64P],
    "scc_graph_copy_csr": [_P, _I32P, _I32P, _I32P, _I32P],
    "scc_graph_device_csr": [_P, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P), C.POINTER(_P)],
    "scc_graph_save_binary": [_P, C.c_char_p],
    "scc_graph_load_binary": [C.c_char_p, C.c_int, C.POINTER(_P)],
    "scc_state_create": [_P, C.POINTER(_P)],
    "scc_state_reset": [_P],
    "scc_state_free": [_P],
    "scc_state_synchronize": [_P],
    "scc_state_stream": [_P, C.POINTER(_P)],
    "scc_state_get_color": [_P, _I32P],
    "scc_state_get_scc": [_P, _I32P],
    "scc_state_set_color": [_P, _I32P],
    "scc_state_set_scc": [_P, _I32P],
    "scc_state_get_wcc": [_P, _I32P],
    "scc_state_get_trim_targets": [_P, _I32P, C.c_int32, _I32P],
    "scc_state_device_arrays": [_P, C.POINTER(_P), C.POINTER(_P)],
    "scc_state_profile": [_P, C.c_int],
    "scc_state_get_tuning": [_P, C.POINTER(Tuning)],
    "scc_state_set_tuning": [_P, C.POINTER(Tuning)],
    "scc_autotune": [_P, _P, C.c_int, C.c_int, C.POINTER(Tuning), C.POINTER(C.c_double)],
    "scc_state_profile_read": [_P, C.POINTER(C.c_double), _I64P, _I64P, _I64P],
    "scc_get_new_color": [_P, _I32P],
    "scc_get_curr_color": [_P, _I32P],
    "scc_choose_pivot_from_color": [_P, _P, C.c_int32, _I32P],
    "scc_generate_compact_set": [_P, _P, C.c_int32, _I32P, C.c_int32, _I32P],
    "scc_do_global_trim1": [_P, _P, _I32P],
    "scc_do_global_trim1_compact": [_P, _P, _I32P],
    "scc_repeat_global_trim1": [_P, _P, C.c_int32, _I32P],
    "scc_repeat_global_trim1_compact": [_P, _P, C.c_int32, _I32P],
    "scc_create_trim1_compact": [_P, _P, _I32P],
    "scc_trim1_noalloc": [C.c_int32, _P, _P, _P, _P, _P, _P, _I32P, _P],
    "scc_do_global_trim2_new": [_P, _P, _I32P],
    "scc_do_global_trim2": [_P, _P, _I32P],
    "scc_repeat_global_trim2_new": [_P, _P, C.c_int32, _I32P],
    "scc_do_fw_bw_global_main": [_P, _P, C.c_int32, C.c_int32, C.c_int, _I32P],
    "scc_do_fw_bw_global_pivot": [_P, _P, C.c_int32, C.c_int32, C.c_int, _I32P],
    "scc_create_works_after_bfs_trim": [_P, _P, _I32P],
    "scc_start_workers_fw_bw": [_P, _P, C.c_int32],
    "scc_start_workers_fw_bw_dfs": [_P, _P, C.c_int32],
    "scc_work_q_size": [_P, _I32P],
    "scc_work_q_items": [_P, _I32P, _I32P, C.c_int32, _I32P],
    "scc_do_global_wcc": [_P, _P],
    "scc_create_work_items_from_wcc": [_P, _P, _I32P],
    "scc_run": [_P, _P, C.c_int, C.c_int, C.POINTER(RunStats)],
    "scc_count_sccs": [_P, _I32P],
    "scc_canonical_labels": [_P, _I32P],
    "scc_canonical_labels_device": [_P, _P],
    "scc_output_scc_list": [_P, C.c_char_p],
    "scc_read_scc_list": [C.c_char_p, C.c_int32, _I32P, _I32P],
    "scc_histogram": [_P, _I32P, _I32P, C.c_int32, _I32P],
    "scc_decompose_csr": [C.c_int32, C.c_int32, _I32P, _I32P, _I32P, _I32P, C.c_int, C.c_int, _I32P, _I32P,
                          C.POINTER(RunStats)],
    "scc_update_batch": [_P, _P, C.c_int64, _P, _P, C.c_int64, _P, _P, C.c_int, C.POINTER(UpdateStats)],
    "scc_incremental_insert": [_P, _P, C.c_int64, _I32P, _I32P, C.POINTER(UpdateStats)],
    "scc_decremental_delete": [_P, _P, C.c_int64, _I32P, _I32P, C.POINTER(UpdateStats)],
    "scc_insert_idea1": [_P, _P, C.c_int64, _I32P, _I32P, C.POINTER(RunStats)],
    "scc_condensation_graph": [_P, _I32P, C.c_int32, C.c_int64, _I32P, _I32P, C.POINTER(_P)],
    "scc_topological_levels": [_P, _I32P, _I32P],
    "scc_read_edge_list": [C.c_char_p, C.c_int64, _I32P, _I32P, C.POINTER(C.c_int64), _I32P],
    "scc_affected_levels": [_P, _I32P, C.c_int32, C.c_int32, _I32P, C.c_int64, _I32P, _I32P, _I32P, _I32P],
    "scc_state_finish_unaffected": [_P, _I32P, _I32P, C.c_int32, _I32P],
    "scc_batch_default_tuning": [C.POINTER(BatchTuning)],
    "scc_batch_plan_create": [_P, _P, _I32P, C.c_int32, C.POINTER(BatchTuning), C.POINTER(_P)],
    "scc_batch_plan_run": [_P, C.POINTER(BatchStats)],
    "scc_batch_plan_free": [_P],
    "scc_batch_autotune": [_P, _P, _I32P, C.c_int32, C.POINTER(BatchTuning), C.POINTER(C.c_double)],
    "scc_server_create": [C.c_int, C.c_int, C.c_int64, C.POINTER(_P)],
    "scc_server_add_graph": [_P, _P, _I32P],
    "scc_server_submit": [_P, C.c_int32, C.c_int64, _I32P, _I32P, C.c_int64, _I32P, _I32P, _I64P],
    "scc_server_set_coalesce": [_P, C.c_int32, C.c_int64],
    "scc_graph_upload_csr_out": [_P, _P, _P, _P],
    "scc_release_cached_memory": [C.c_int],
    "scc_debug_inject": [C.c_int, C.c_int64],
    "scc_server_wait": [_P, C.c_int64, C.POINTER(RequestResult)],
    "scc_server_set_admission": [_P, C.c_int64, C.c_double],
    "scc_server_drain": [_P],
    "scc_server_get_stats": [_P, C.POINTER(ServerStats)],
    "scc_server_labels": [_P, C.c_int32, _I32P],
    "scc_server_session_graph": [_P, C.c_int32, C.POINTER(_P)],
    "scc_server_free": [_P],
    "scc_gen_sizes": [C.POINTER(GenParams), _I32P, _I64P],
    "scc_gen_edges_host": [C.POINTER(GenParams), _I32P, _I32P, C.c_int64, _I64P],
    "scc_gen_graph": [C.POINTER(GenParams), C.c_int, C.c_int, C.POINTER(_P)],
    "scc_gen_batch_layout": [C.POINTER(BatchParams), _I32P, _I32P, _I64P],
    "scc_gen_batch_edges_host": [C.POINTER(BatchParams), _I32P, _I32P, C.c_int64, _I64P],
    "scc_gen_batch_graph": [C.POINTER(BatchParams), C.c_int, C.c_int, C.POINTER(_P)],
    "scc_graph_subgraph": [_P, C.c_int32, C.c_int32, C.POINTER(_P)],
    "scc_pivot_model_create": [C.c_int, C.c_uint64, C.POINTER(_P)],
    "scc_pivot_model_free": [_P],
    "scc_pivot_model_get_params": [_P, _F32P],
    "scc_pivot_model_set_params": [_P, _F32P],
    "scc_pivot_model_save": [_P, C.c_char_p],
    "scc_pivot_model_load": [C.c_int, C.c_char_p, C.POINTER(_P)],
    "scc_pivot_model_forward": [_P, _F32P, C.c_int64, C.c_int, _F32P],
    "scc_pivot_model_bench": [_P, C.c_int64, C.c_int, C.POINTER(C.c_double)],
    "scc_pivot_model_loss_grad": [_P, _F32P, _F32P, C.c_int64, _F32P, _F32P],
    "scc_pivot_model_train": [_P, _F32P, _F32P, C.c_int64, C.c_int, C.c_int, C.c_float, C.c_uint64, _F32P],
    "scc_state_set_pivot_model": [_P, _P],
    "scc_state_pivot_log": [_P, C.c_int64, C.c_int32],
    "scc_state_pivot_records": [_P, _F32P, _F32P, _I32P, _I32P, C.c_int64, _I64P],
}
_RESTYPES = {"scc_status_string": C.c_char_p, "scc_last_error": C.c_char_p, "scc_version": C.c_int}

_lib = None


def lib() -> C.CDLL:
    """Load the native library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"native library missing: {LIB_PATH} (run python -m dynamicgraphs_scc_b200.build)")
        L = C.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = _RESTYPES.get(name, C.c_int)
        _lib = L
    return _lib


def declared_symbols() -> list[str]:
    return list(_SIGS)


def call(name: str, *args):
    rc = getattr(lib(), name)(*args)
    if rc != SCC_OK:
        msg = lib().scc_last_error().decode(errors="replace")
        raise SccError(rc, name, msg)
    return rc


def i32p(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"], "need contiguous int32"
    return a.ctypes.data_as(_I32P)


def f32p(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"], "need contiguous float32"
    return a.ctypes.data_as(_F32P)


def out_i32() -> C.c_int32:
    return C.c_int32(0)
