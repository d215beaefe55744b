"""trc_bfs_noalloc: the BFS entry point that allocates no device memory.

It is for callers that cannot call cudaMalloc when they traverse (device
memory fixed at start-up, an allocator owned by another component, or a
request path that must not allocate); its scratch is a static device array.
The test calls it twice in a row through the C ABI and compares each result
with the existing trc_bfs: levels must be identical and parents a valid BFS
tree (parents are not unique, as in the reference).  It also checks the two
limits: host output pointers and graphs above TRC_NOALLOC_MAX_VERTICES are
rejected with TRC_ERR_INVALID.  Named to run last; it passes alone in a fresh
process and after the other tests."""
import ctypes as C

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


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
    par_ref, lv_ref = g.bfs(src)  # the existing (allocating) entry point
    for _ in range(2):
        par = torch.full((n,), 7, dtype=torch.int32, device="cuda")
        lv = torch.full((n,), 7, dtype=torch.int32, device="cuda")
        st = L.trc_bfs_noalloc(g._h, src, C.c_void_p(par.data_ptr()), C.c_void_p(lv.data_ptr()),
                               _lib.TRC_DEVICE_PTR)
        assert st == _lib.TRC_OK, L.trc_last_error()
        lvh = lv.cpu().numpy().view(np.uint32)
        parh = par.cpu().numpy()
        assert np.array_equal(lvh, lv_ref)
        assert O.bfs_check_parents(off, tgt, src, lvh, parh) == 0
    # host outputs are refused (the call would need staging memory)
    hp = np.empty(n, np.int32)
    hl = np.empty(n, np.uint32)
    st = L.trc_bfs_noalloc(g._h, src, C.c_void_p(hp.ctypes.data), C.c_void_p(hl.ctypes.data), 0)
    assert st == _lib.TRC_ERR_INVALID
    # graphs above the static scratch size are refused before any device work
    big = T.Graph(_lib.TRC_NOALLOC_MAX_VERTICES + 1)
    st = L.trc_bfs_noalloc(big._h, 0, C.c_void_p(par.data_ptr()), C.c_void_p(lv.data_ptr()),
                           _lib.TRC_DEVICE_PTR)
    assert st == _lib.TRC_ERR_INVALID
    assert b"TRC_NOALLOC_MAX_VERTICES" in L.trc_last_error()
