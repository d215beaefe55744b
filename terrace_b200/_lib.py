"""ctypes binding of libterrace_b200.so (the C ABI in include/terrace_b200.h).

There is no CPU fallback: if the library is missing, importing the package
raises, naming the build command.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libterrace_b200.so")

TRC_OK = 0
TRC_ERR_INVALID = 1
TRC_ERR_NOMEM = 2
TRC_ERR_CUDA = 3
TRC_ERR_TIMEOUT = 4
TRC_ERR_STATE = 5
TRC_ERR_NOT_BUILT = 6
TRC_ERR_IO = 7

TRC_DEVICE_PTR = 0x1
TRC_SYMMETRIZE = 0x2
TRC_DROP_SELF_LOOPS = 0x4
TRC_UNREACHED = 0xFFFFFFFF
TRC_NOALLOC_MAX_VERTICES = 1048576
TUNE_PUSH_PULL, TUNE_PAGERANK, TUNE_PMA = 1, 2, 4
REQ_INSERT, REQ_DELETE, REQ_BFS, REQ_DEGREE, REQ_NEIGHBORS, REQ_PAGERANK = range(6)
SERVE_FIFO, SERVE_BATCHED = 0, 1
RESULT_FULL, RESULT_SUMMARY = 0, 1


class TrcError(RuntimeError):
    """A non-OK trc_status; .status holds the code."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"[trc status {status}] {msg}")
        self.status = status


class trc_config(C.Structure):
    _fields_ = [("hub_threshold", C.c_uint32),
                ("pma_root_density", C.c_double),
                ("pma_build_density", C.c_double),
                ("hub_block_fill", C.c_double),
                ("push_pull_divisor", C.c_uint32),
                ("hub_stage_limit", C.c_uint32),
                ("cuda_graphs", C.c_uint32)]


class trc_device_view(C.Structure):
    _fields_ = [("n", C.c_uint32), ("inline_slots", C.c_uint32), ("hub_block", C.c_uint32),
                ("deg", C.c_void_p), ("inl", C.c_void_p), ("pbeg", C.c_void_p), ("pma", C.c_void_p),
                ("hub_of", C.c_void_p), ("hub_dir0", C.c_void_p), ("hub_nblk", C.c_void_p),
                ("hub_dir", C.c_void_p), ("hub_pre", C.c_void_p), ("hub_key", C.c_void_p),
                ("hslot", C.c_void_p), ("stream", C.c_void_p)]


class trc_tuning(C.Structure):
    _fields_ = [("push_pull_divisor", C.c_uint32), ("pr_group_cut", C.c_uint32),
                ("pr_group_lanes", C.c_uint32), ("pma_leaf_log", C.c_uint32),
                ("bfs_ms", C.c_double), ("pagerank_iter_ms", C.c_double),
                ("pma_insert_ms", C.c_double)]


class trc_server_config(C.Structure):
    _fields_ = [("mode", C.c_uint32), ("result_mode", C.c_uint32), ("symmetrize", C.c_uint32),
                ("max_bfs_group", C.c_uint32), ("max_round_edges", C.c_uint64)]


class trc_server_stats(C.Structure):
    _fields_ = [("completed", C.c_uint64), ("elapsed_s", C.c_double), ("p50_ms", C.c_double),
                ("p99_ms", C.c_double), ("mean_ms", C.c_double), ("max_ms", C.c_double),
                ("rounds", C.c_uint64), ("device_calls", C.c_uint64), ("rejected", C.c_uint64),
                ("version", C.c_uint64), ("worst_round_ms", C.c_double),
                ("worst_update_ms", C.c_double), ("worst_bfs_ms", C.c_double),
                ("worst_pagerank_ms", C.c_double), ("worst_round_requests", C.c_uint64),
                ("worst_round_rebuilds", C.c_uint64), ("pma_rebuilds", C.c_uint64)]


class trc_round_record(C.Structure):
    _fields_ = [("t_start_ms", C.c_double), ("ms", C.c_double), ("lookup_ms", C.c_double),
                ("update_ms", C.c_double), ("bfs_ms", C.c_double), ("pagerank_ms", C.c_double),
                ("lookups", C.c_uint32), ("updates", C.c_uint32), ("bfs", C.c_uint32),
                ("pageranks", C.c_uint32), ("update_pairs", C.c_uint64),
                ("bfs_groups", C.c_uint32), ("bfs_singles", C.c_uint32),
                ("rebuilds", C.c_uint32), ("pending_after", C.c_uint32)]


class trc_stats(C.Structure):
    _fields_ = [("n", C.c_uint32),
                ("num_edges", C.c_uint64),
                ("inline_edges", C.c_uint64),
                ("pma_edges", C.c_uint64),
                ("pma_capacity", C.c_uint64),
                ("hub_edges", C.c_uint64),
                ("num_hubs", C.c_uint32),
                ("hub_blocks_used", C.c_uint64),
                ("device_bytes", C.c_uint64),
                ("pma_rebuilds", C.c_uint64),
                ("pma_window_rebalances", C.c_uint64),
                ("last_keys", C.c_uint64),
                ("last_applied", C.c_uint64),
                ("last_touched", C.c_uint64),
                ("last_rewritten", C.c_uint64),
                ("last_gathered", C.c_uint64),
                ("last_written", C.c_uint64),
                ("last_windows", C.c_uint64),
                ("last_rebuild", C.c_uint64),
                ("last_hub_touched", C.c_uint64),
                ("last_hub_local", C.c_uint64),
                ("last_hub_rewritten", C.c_uint64),
                ("last_hub_blocks_written", C.c_uint64),
                ("last_hub_read", C.c_uint64),
                ("last_hub_written", C.c_uint64),
                ("hub_splits", C.c_uint64),
                ("hub_rewrites", C.c_uint64),
                ("hub_blocks_free", C.c_uint64),
                ("hub_absorbs", C.c_uint64), ("sort_retries", C.c_uint64)]


# (name, restype, argtypes) for every symbol the header declares
_vp = C.c_void_p
_u32, _u64, _i32, _int, _dbl = C.c_uint32, C.c_uint64, C.c_int32, C.c_int, C.c_double
SIGNATURES = [
    ("trc_config_default", None, [C.POINTER(trc_config)]),
    ("trc_status_string", C.c_char_p, [_int]),
    ("trc_last_error", C.c_char_p, []),
    ("trc_graph_create", _int, [_u32, _u64, C.POINTER(trc_config), C.POINTER(_vp)]),
    ("trc_graph_destroy", _int, [_vp]),
    ("trc_graph_set_stream", _int, [_vp, _vp]),
    ("trc_release_scratch", _int, [_vp]),
    ("trc_debug_sort_wait", _int, [_vp, _u32, _int]),
    ("trc_debug_sort_mode", _int, [_vp, _int]),
    ("trc_add_edge_batch", _int, [_vp, _vp, _vp, _u64, _u32, C.POINTER(_u64)]),
    ("trc_remove_edge_batch", _int, [_vp, _vp, _vp, _u64, _u32, C.POINTER(_u64)]),
    ("trc_is_edge", _int, [_vp, _vp, _vp, _u64, _vp, _u32]),
    ("trc_degree", _int, [_vp, _vp, _u64, _vp, _u32]),
    ("trc_neighbors", _int, [_vp, _u32, _vp, _u64, C.POINTER(_u64), _u32]),
    ("trc_count_common", _int, [_vp, _vp, _vp, _u64, _vp, _u32]),
    ("trc_num_vertices", _int, [_vp, C.POINTER(_u32)]),
    ("trc_num_edges", _int, [_vp, C.POINTER(_u64)]),
    ("trc_get_size", _int, [_vp, C.POINTER(_u64)]),
    ("trc_dump_csr", _int, [_vp, _vp, _vp, _u32]),
    ("trc_graph_load_adj", _int, [C.c_char_p, _u64, C.POINTER(trc_config), _u32, C.POINTER(_vp)]),
    ("trc_graph_save_adj", _int, [_vp, C.c_char_p]),
    ("trc_graph_load_csr", _int, [C.c_char_p, _u64, C.POINTER(trc_config), _u32, C.POINTER(_vp)]),
    ("trc_graph_save_csr", _int, [_vp, C.c_char_p]),
    ("trc_bfs", _int, [_vp, _u32, _vp, _vp, _u32]),
    ("trc_bfs_noalloc", _int, [_vp, _u32, _vp, _vp, _u32]),
    ("trc_msbfs", _int, [_vp, _vp, _u32, _vp, _u32]),
    ("trc_msbc", _int, [_vp, _vp, _u32, _vp, _u32]),
    ("trc_pagerank", _int, [_vp, _u32, _dbl, _vp, _u32]),
    ("trc_cc", _int, [_vp, _vp, _u32]),
    ("trc_bc", _int, [_vp, _u32, _vp, _u32]),
    ("trc_tc", _int, [_vp, C.POINTER(_u64)]),
    ("trc_rmat_generate", _int, [_u32, _u32, _dbl, _dbl, _dbl, _u64, _u64, _vp, _vp, _u32, _vp]),
    ("trc_get_stats", _int, [_vp, C.POINTER(trc_stats)]),
    ("trc_get_device_view", _int, [_vp, C.POINTER(trc_device_view)]),
    ("trc_check", _int, [_vp, C.POINTER(_u64)]),
    ("trc_profile_enable", _int, [_vp, _int]),
    ("trc_profile_reset", _int, [_vp]),
    ("trc_profile_get", _int, [_vp, C.c_char_p, C.POINTER(_dbl), C.POINTER(_u64)]),
    ("trc_profile_names", _int, [_vp, C.c_char_p, _u64]),
    ("trc_launch_count", _int, [_vp, C.POINTER(_u64)]),
    ("trc_autotune", _int, [_vp, _u32, _vp, _vp, _u64, _u32, C.POINTER(trc_tuning)]),
    ("trc_get_tuning", _int, [_vp, C.POINTER(trc_tuning)]),
    ("trc_set_tuning", _int, [_vp, C.POINTER(trc_tuning)]),
    ("trc_server_config_default", None, [C.POINTER(trc_server_config)]),
    ("trc_server_create", _int, [_vp, C.POINTER(trc_server_config), C.POINTER(_vp)]),
    ("trc_server_destroy", _int, [_vp]),
    ("trc_server_submit", _int, [_vp, _int, _vp, _vp, _u64, _u32, C.POINTER(_u64)]),
    ("trc_server_wait", _int, [_vp, _u64, C.c_int64]),
    ("trc_server_result", _int, [_vp, _u64, _vp, _u64, C.POINTER(_u64), C.POINTER(_dbl),
                                 C.POINTER(_u64), C.POINTER(_int)]),
    ("trc_server_release", _int, [_vp, _u64]),
    ("trc_server_get_stats", _int, [_vp, _int, C.POINTER(trc_server_stats)]),
    ("trc_server_reset_stats", _int, [_vp]),
    ("trc_server_hold", _int, [_vp, _int]),
    ("trc_server_rounds", _int, [_vp, C.POINTER(trc_round_record), _u64, C.POINTER(_u64)]),
]

_lib = None


def load(path: str = LIB_PATH):
    """Load the library and declare every signature.  Raises if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m terrace_b200.build` "
                          "(there is no CPU fallback)")
    L = C.CDLL(path)
    for name, res, args in SIGNATURES:
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(status: int):
    if status != TRC_OK:
        msg = load().trc_last_error().decode(errors="replace")
        raise TrcError(status, msg)
