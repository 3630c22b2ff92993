"""ctypes declarations of libsigmo_b200.so (include/sigmo_b200.h)."""
from __future__ import annotations

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libsigmo_b200.so"


class SigmoError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code


class HostGraphsC(ctypes.Structure):
    _fields_ = [
        ("num_graphs", ctypes.c_uint32),
        ("total_nodes", ctypes.c_uint64),
        ("total_edges", ctypes.c_uint64),
        ("graph_offsets", ctypes.c_void_p),
        ("row_offsets", ctypes.c_void_p),
        ("column_indices", ctypes.c_void_p),
        ("node_labels", ctypes.c_void_p),
        ("edge_labels", ctypes.c_void_p),
    ]


class OptionsC(ctypes.Structure):
    _fields_ = [("profile", ctypes.c_int), ("join_work_group_size", ctypes.c_uint32),
                ("filter_work_group_size", ctypes.c_uint32)]


class MatchResultC(ctypes.Structure):
    _fields_ = [
        ("total_matches", ctypes.c_uint64),
        ("admitted_pairs", ctypes.c_uint64),
        ("pairs", ctypes.c_uint64),
        ("ms_signatures", ctypes.c_double),
        ("ms_filter", ctypes.c_double),
        ("ms_mapping", ctypes.c_double),
        ("ms_join", ctypes.c_double),
        ("ms_total", ctypes.c_double),
    ]


class TuningC(ctypes.Structure):
    _fields_ = [
        ("join_blocks_per_sm", ctypes.c_uint32),
        ("join_chunk", ctypes.c_uint32),
        ("overflow_blocks", ctypes.c_uint32),
        ("overflow_serial", ctypes.c_uint32),
        ("mask_chunk_slots", ctypes.c_uint32),
        ("overflow_split", ctypes.c_uint32),
        ("join_kernel", ctypes.c_uint32),
        ("join_pool", ctypes.c_uint32),
    ]


class ServerOptionsC(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_uint32),
        ("find_first", ctypes.c_int32),
        ("max_inflight", ctypes.c_uint32),
        ("max_batch_queries", ctypes.c_uint32),
        ("memory_budget", ctypes.c_uint64),
        ("batch_window_us", ctypes.c_uint32),
        ("join_step_budget", ctypes.c_uint64),
    ]


class RequestResultC(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int32),
        ("num_queries", ctypes.c_uint32),
        ("pairs", ctypes.c_uint64),
        ("matched_pairs", ctypes.c_uint64),
        ("total_matches", ctypes.c_uint64),
        ("batch_id", ctypes.c_uint64),
        ("batch_queries", ctypes.c_uint32),
        ("batch_requests", ctypes.c_uint32),
        ("projected_bytes", ctypes.c_uint64),
        ("ms_queue", ctypes.c_double),
        ("ms_device", ctypes.c_double),
        ("ms_latency", ctypes.c_double),
        ("ms_filter", ctypes.c_double),
        ("ms_mapping", ctypes.c_double),
        ("ms_join", ctypes.c_double),
        ("gathered_plane_bytes", ctypes.c_uint64),
    ]


class ServerStatsC(ctypes.Structure):
    _fields_ = [
        ("requests_submitted", ctypes.c_uint64),
        ("requests_completed", ctypes.c_uint64),
        ("requests_failed", ctypes.c_uint64),
        ("queries_completed", ctypes.c_uint64),
        ("batches", ctypes.c_uint64),
        ("pairs", ctypes.c_uint64),
        ("admitted_pairs", ctypes.c_uint64),
        ("device_ms", ctypes.c_double),
        ("peak_reserved_bytes", ctypes.c_uint64),
        ("max_batches_in_flight", ctypes.c_uint32),
        ("pending_requests", ctypes.c_uint32),
        ("resident_bytes", ctypes.c_uint64),
        ("memory_budget", ctypes.c_uint64),
    ]


_vp, _i, _u32, _u64, _sz, _d = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_size_t, ctypes.c_double
_P = ctypes.POINTER

# name -> (restype, argtypes)
SIGNATURES = {
    "sigmo_last_error": (ctypes.c_char_p, []),
    "sigmo_version": (ctypes.c_char_p, []),
    "sigmo_parse_graphs": (_i, [ctypes.c_char_p, _sz, _P(HostGraphsC)]),
    "sigmo_host_graphs_concat": (_i, [_P(HostGraphsC), _P(HostGraphsC), _P(HostGraphsC)]),
    "sigmo_host_graphs_slice": (_i, [_P(HostGraphsC), _u32, _u32, _P(HostGraphsC)]),
    "sigmo_format_graphs": (_i, [_P(HostGraphsC), _vp, _P(_sz)]),
    "sigmo_host_graphs_free": (None, [_P(HostGraphsC)]),
    "sigmo_graphs_save": (_i, [_P(HostGraphsC), ctypes.c_char_p]),
    "sigmo_graphs_load": (_i, [ctypes.c_char_p, _P(HostGraphsC)]),
    "sigmo_graph_create_from_local": (_i, [_vp, _u32, _vp, _vp, _vp, _vp, _vp, _vp, _P(_vp)]),
    "sigmo_graph_set_vertex_base": (_i, [_vp, _u32]),
    "sigmo_generate_molecules": (_i, [_i, _u32, _u32, _u32, _d, _u64, _P(HostGraphsC)]),
    "sigmo_generate_queries": (_i, [_i, _u32, _u32, _u32, _u32, _u32, _u64, _P(HostGraphsC)]),
    "sigmo_default_options": (None, [_P(OptionsC)]),
    "sigmo_queue_create": (_i, [_i, _P(OptionsC), _P(_vp)]),
    "sigmo_queue_destroy": (_i, [_vp]),
    "sigmo_queue_wait": (_i, [_vp]),
    "sigmo_queue_stream": (_i, [_vp, _P(_vp)]),
    "sigmo_queue_last_stage_ms": (_i, [_vp, _P(_d)]),
    "sigmo_queue_device_info": (_i, [_vp, _P(_u64), ctypes.c_char_p, _sz]),
    "sigmo_queue_launch_count": (_i, [_vp, _P(_u64)]),
    "sigmo_graph_create": (_i, [_vp, _P(HostGraphsC), _P(_vp)]),
    "sigmo_graph_create_device": (_i, [_vp, _u32, _u64, _u64, _vp, _vp, _vp, _vp, _vp, _P(_vp)]),
    "sigmo_graph_destroy": (_i, [_vp]),
    "sigmo_graph_info": (_i, [_vp, _P(_u32), _P(_u64), _P(_u64), _P(_u32)]),
    "sigmo_graph_alloc_size": (_i, [_vp, _P(_u64)]),
    "sigmo_candidates_create": (_i, [_vp, _u64, _u64, _P(_vp)]),
    "sigmo_candidates_destroy": (_i, [_vp]),
    "sigmo_candidates_words_per_row": (_i, [_vp, _P(_u64)]),
    "sigmo_candidates_alloc_size": (_i, [_vp, _P(_u64)]),
    "sigmo_candidates_download": (_i, [_vp, _u64, _u64, _vp]),
    "sigmo_candidates_row_counts": (_i, [_vp, _vp]),
    "sigmo_candidates_digest": (_i, [_vp, _P(_u64)]),
    "sigmo_signature_create": (_i, [_vp, _u64, _u64, _P(_vp)]),
    "sigmo_signature_destroy": (_i, [_vp]),
    "sigmo_signature_generate": (_i, [_vp, _vp, _i]),
    "sigmo_signature_refine": (_i, [_vp, _vp, _i, _u32]),
    "sigmo_signature_download": (_i, [_vp, _i, _vp, _u64]),
    "sigmo_signature_alloc_size": (_i, [_vp, _i, _P(_u64)]),
    "sigmo_filter_candidates": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "sigmo_refine_candidates": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "sigmo_gmcr_create": (_i, [_vp, _P(_vp)]),
    "sigmo_gmcr_destroy": (_i, [_vp]),
    "sigmo_gmcr_generate": (_i, [_vp, _vp, _vp, _vp]),
    "sigmo_gmcr_total": (_i, [_vp, _P(_u64)]),
    "sigmo_gmcr_download": (_i, [_vp, _vp, _u64, _vp, _u64]),
    "sigmo_gmcr_generate_noalloc": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _u64, _P(_u64)]),
    "sigmo_join_candidates": (_i, [_vp, _vp, _vp, _vp, _vp, _P(_u64), _i, _vp]),
    "sigmo_join_wildcard_candidates": (_i, [_vp, _vp, _vp, _vp, _vp, _P(_u64), _i, _vp]),
    "sigmo_match_batched": (_i, [_vp, _vp, _vp, _u32, _i, _u32, _vp, _vp, _P(MatchResultC)]),
    "sigmo_queue_set_tuning": (_i, [_vp, _P(TuningC)]),
    "sigmo_queue_get_tuning": (_i, [_vp, _P(TuningC)]),
    "sigmo_queue_set_join_budget": (_i, [_vp, ctypes.c_uint64]),
    "sigmo_queue_get_join_budget": (_i, [_vp, _P(ctypes.c_uint64)]),
    "sigmo_autotune": (_i, [_vp, _vp, _vp, _u32, _i, _u32, _P(TuningC), _P(_d), _P(_d)]),
    "sigmo_server_default_options": (None, [_P(ServerOptionsC)]),
    "sigmo_server_create": (_i, [_i, _P(HostGraphsC), _vp, _P(ServerOptionsC), _P(_vp)]),
    "sigmo_server_submit": (_i, [_vp, _P(HostGraphsC), _u32, _P(_u64)]),
    "sigmo_server_wait": (_i, [_vp, _u64, ctypes.c_int64, _P(RequestResultC)]),
    "sigmo_server_query_totals": (_i, [_vp, _u64, _vp, _vp, _u32]),
    "sigmo_server_pairs": (_i, [_vp, _u64, _vp, _vp, _vp, _u64, _P(_u64)]),
    "sigmo_server_release": (_i, [_vp, _u64]),
    "sigmo_server_get_stats": (_i, [_vp, _P(ServerStatsC)]),
    "sigmo_server_destroy": (_i, [_vp]),
    "sigmo_match_download_counts": (_i, [_vp, _vp, _u64]),
}

_lib = None


def lib():
    """The loaded library.  Raises if it has not been built: there is no
    fallback implementation."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m sigmo_b200.build`")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    return (lib().sigmo_last_error() or b"").decode(errors="replace")


def check(rc: int):
    if rc != 0:
        raise SigmoError(rc, last_error())
