"""Failure paths of the device code, driven without a GPU fault.

The batch sort's scatter passes wait, per tile, for the digit counts of the
tiles before them (decoupled look-back).  That wait is bounded: after a set
number of polls the tile records ERR_TIMEOUT and returns, and the update
fails with TRC_ERR_TIMEOUT before anything in the graph is modified.  Here
the wait is made to run out on purpose with the library's test hook
(trc_debug_sort_wait: a few polls, and no tile 0 ever publishes -- a flag
that nothing sets), and the test checks the status, that the graph is
unchanged, and that the same handle works normally afterwards."""
import hashlib

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

SYM = dict(symmetrize=True, drop_self_loops=True)


@pytest.fixture(scope="module")
def T():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    import terrace_b200
    return terrace_b200


def csr_sha(off, tgt):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(off, "<u8").tobytes())
    h.update(np.ascontiguousarray(tgt, "<u4").tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("pairs", [1, 3000, 50000])
def test_sort_wait_runs_out_and_leaves_graph_unchanged(T, pairs):
    from terrace_b200 import _lib
    n = 1 << 12
    s, d = T.rmat_generate(n, 0, .5, .1, .1, 8 * n)
    g = T.Graph(n, hub_threshold=64)
    g.add_edge_batch(s, d, **SYM)
    keys = O.make_keys(s, d, True, True)
    h0 = csr_sha(*g.dump_csr())
    m0 = g.get_num_edges()
    bs, bd = T.rmat_generate(n, 5, .5, .1, .1, pairs)
    if pairs == 1:
        bs, bd = np.array([1], np.uint32), np.array([2], np.uint32)
    _lib.check(g._L.trc_debug_sort_wait(g._h, 32, 1))
    for op in (g.add_edge_batch, g.remove_edge_batch):
        with pytest.raises(T.TrcError) as e:
            op(bs, bd, **SYM)
        assert e.value.status == _lib.TRC_ERR_TIMEOUT
        assert "look-back" in str(e.value)
        assert g.get_num_edges() == m0
        assert csr_sha(*g.dump_csr()) == h0
        assert g.check() == 0
    # the defaults back: the same batch now applies, and matches the oracle
    _lib.check(g._L.trc_debug_sort_wait(g._h, 0, 0))
    g.add_edge_batch(bs, bd, **SYM)
    want = O.csr_from_keys(n, O.key_union(keys, O.make_keys(bs, bd, True, True)))
    off, tgt = g.dump_csr()
    assert np.array_equal(off, want[0]) and np.array_equal(tgt, want[1])
    assert g.check() == 0
    g.close()
