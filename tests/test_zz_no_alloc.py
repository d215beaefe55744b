"""trc_bfs_noalloc: the BFS entry point that allocates no device memory.

It is for callers that cannot call cudaMalloc when they traverse (device
memory fixed at start-up, an allocator owned by another component, or a
request path that must not allocate); its scratch is a static device array.
The test calls it twice in a row through the C ABI on each graph and compares
each result with the oracle's BFS levels and with the existing trc_bfs:
levels must be identical and parents a valid BFS tree (parents are not
unique, as in the reference).  One graph has exactly TRC_NOALLOC_MAX_VERTICES
vertices with a frontier of all but one of them, so a queue fills to its
last slot.  It also checks the two limits: host output pointers and graphs
above TRC_NOALLOC_MAX_VERTICES are rejected with TRC_ERR_INVALID.  Named to
run last; it passes alone in a fresh process and after the other tests."""
import ctypes as C

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _noalloc_twice(T, _lib, L, g, off, tgt, src):
    import torch
    n = g.get_num_vertices()
    want = O.bfs_levels(off, tgt, src)
    par_ref, lv_ref = g.bfs(src)  # the existing (allocating) entry point
    assert np.array_equal(lv_ref, want)
    for _ in range(2):
        par = torch.full((n,), 7, dtype=torch.int32, device="cuda")
        lv = torch.full((n,), 7, dtype=torch.int32, device="cuda")
        st = L.trc_bfs_noalloc(g._h, src, C.c_void_p(par.data_ptr()), C.c_void_p(lv.data_ptr()),
                               _lib.TRC_DEVICE_PTR)
        assert st == _lib.TRC_OK, L.trc_last_error()
        lvh = lv.cpu().numpy().view(np.uint32)
        parh = par.cpu().numpy()
        assert np.array_equal(lvh, want)
        assert np.array_equal(lvh, lv_ref)
        assert O.bfs_check_parents(off, tgt, src, lvh, parh) == 0
    return par


def test_bfs_noalloc_matches_bfs():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    import terrace_b200 as T
    from terrace_b200 import _lib
    L = _lib.load()
    n = 1 << 16
    s, d = T.rmat_generate(n, 3, .5, .1, .1, 8 * n)
    g = T.Graph(n, hub_threshold=128)
    g.add_edge_batch(s, d, symmetrize=True, drop_self_loops=True)
    off, tgt = g.dump_csr()
    src = int(np.argmax(np.diff(off.astype(np.int64))))
    par = _noalloc_twice(T, _lib, L, g, off, tgt, src)
    # host outputs are refused (the call would need staging memory)
    hp = np.empty(n, np.int32)
    hl = np.empty(n, np.uint32)
    st = L.trc_bfs_noalloc(g._h, src, C.c_void_p(hp.ctypes.data), C.c_void_p(hl.ctypes.data), 0)
    assert st == _lib.TRC_ERR_INVALID
    g.close()
    # exactly the largest graph the static queues hold: a star on vertex 5
    # (level 1 = every other vertex but the tail, one queue filled to n - 2
    # entries) with a two-vertex tail 5 - 7 - (n-1) ... (level 2)
    nmax = _lib.TRC_NOALLOC_MAX_VERTICES
    leaves = np.setdiff1d(np.arange(nmax, dtype=np.uint32), np.array([5, nmax - 1], np.uint32))
    es = np.concatenate([np.full(len(leaves), 5, np.uint32), np.array([7], np.uint32)])
    ed = np.concatenate([leaves, np.array([nmax - 1], np.uint32)])
    big = T.Graph(nmax)
    big.add_edge_batch(es, ed, symmetrize=True, drop_self_loops=True)
    off, tgt = O.csr_from_keys(nmax, O.make_keys(es, ed, True, True))
    goff, gtgt = big.dump_csr()
    assert np.array_equal(goff, off) and np.array_equal(gtgt, tgt)
    for src in (5, nmax - 1):
        _noalloc_twice(T, _lib, L, big, off, tgt, src)
    big.close()
    # graphs above the static scratch size are refused before any device work
    over = T.Graph(nmax + 1)
    st = L.trc_bfs_noalloc(over._h, 0, C.c_void_p(par.data_ptr()), C.c_void_p(par.data_ptr()),
                           _lib.TRC_DEVICE_PTR)
    assert st == _lib.TRC_ERR_INVALID
    assert b"TRC_NOALLOC_MAX_VERTICES" in L.trc_last_error()
    over.close()
