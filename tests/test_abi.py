"""CPU checks of the C-ABI boundary: the library loads, exports every entry
point include/terrace_b200.h declares, the Python mirror binds them all, and
without a GPU the product fails loudly instead of falling back to the CPU."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER_DIR = os.path.join(ROOT, "include")


def declared_symbols():
    names = set()
    for fn in os.listdir(HEADER_DIR):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(HEADER_DIR, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(trc_\w+)\s*\(", text))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    from terrace_b200 import build, _lib
    if not os.path.exists(_lib.LIB_PATH):
        build.build()
    return ctypes.CDLL(_lib.LIB_PATH)


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ("trc_graph_create", "trc_add_edge_batch", "trc_remove_edge_batch", "trc_degree",
                 "trc_neighbors", "trc_bfs", "trc_pagerank", "trc_cc", "trc_bc", "trc_tc"):
        assert must in names


def test_library_exports_every_declared_symbol(lib):
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert missing == []


def test_python_binding_covers_header():
    from terrace_b200 import _lib
    bound = {name for name, _, _ in _lib.SIGNATURES}
    assert set(declared_symbols()) <= bound


def test_config_defaults_match_reference_constants(lib):
    from terrace_b200 import _lib
    L = _lib.load()
    cfg = _lib.trc_config()
    L.trc_config_default(ctypes.byref(cfg))
    assert cfg.hub_threshold == 1024          # MEDIUM_DEGREE, include/graph.h:39
    assert cfg.push_pull_divisor == 20        # edgeMap threshold, include/Map.cpp:65-74
    assert abs(cfg.pma_root_density - 0.75) < 1e-12
    assert abs(cfg.pma_build_density - 0.375) < 1e-12
    assert cfg.cuda_graphs == 1


def test_status_strings(lib):
    from terrace_b200 import _lib
    L = _lib.load()
    for s in range(7):
        assert L.trc_status_string(s)


def test_null_handle_is_invalid(lib):
    from terrace_b200 import _lib
    L = _lib.load()
    m = ctypes.c_uint64()
    assert L.trc_num_edges(None, ctypes.byref(m)) == _lib.TRC_ERR_INVALID
    assert b"null" in L.trc_last_error()


def test_no_cpu_fallback_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import terrace_b200 as T
    with pytest.raises(T.TrcError) as e:
        T.Graph(16)
    assert e.value.status == 3  # TRC_ERR_CUDA


def test_tuning_abi_without_gpu(lib):
    from terrace_b200 import _lib
    L = _lib.load()
    t = _lib.trc_tuning()
    assert L.trc_get_tuning(None, ctypes.byref(t)) == _lib.TRC_ERR_INVALID
    assert L.trc_set_tuning(None, ctypes.byref(t)) == _lib.TRC_ERR_INVALID
    assert L.trc_autotune(None, 1, None, None, 0, 0, ctypes.byref(t)) == _lib.TRC_ERR_INVALID


def test_server_abi_without_gpu(lib):
    """Server entry points validate their handles before any device work."""
    from terrace_b200 import _lib
    L = _lib.load()
    cfg = _lib.trc_server_config()
    L.trc_server_config_default(ctypes.byref(cfg))
    assert cfg.mode == _lib.SERVE_BATCHED and cfg.result_mode == _lib.RESULT_FULL
    assert cfg.max_bfs_group == 64 and cfg.symmetrize == 1
    h = ctypes.c_void_p()
    assert L.trc_server_create(None, ctypes.byref(cfg), ctypes.byref(h)) == _lib.TRC_ERR_INVALID
    rid = ctypes.c_uint64()
    assert L.trc_server_submit(None, _lib.REQ_BFS, None, None, 0, 0,
                               ctypes.byref(rid)) == _lib.TRC_ERR_INVALID
    assert L.trc_server_wait(None, 1, 0) == _lib.TRC_ERR_INVALID
    st = _lib.trc_server_stats()
    assert L.trc_server_get_stats(None, -1, ctypes.byref(st)) == _lib.TRC_ERR_INVALID
