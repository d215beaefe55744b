"""GPU parity on the two large workloads, at their full sizes.

config 2: RMAT scale 22, edge factor 16 (a/b/c .5/.1/.1), the
LiveJournal-shaped streaming workload.  The bulk-loaded graph is pinned by
the SHA-256 of its CSR against the oracle (tests/golden/config_pins.json,
made by tests/golden/make_config_pins.py); then, for each batch size 1e1,
1e3, 1e5 and 1e6 (RMAT pairs of seed stream 1, symmetrized), the batch is
inserted and then deleted, and after each of the two steps the sorted
adjacency, BFS levels (exact, parents a valid tree), CC labels (exact),
PageRank 10 iterations (relative 1e-9) and the exact triangle count are
compared with the oracle.  The triangle count is carried from the pinned
count of the bulk load by the oracle's per-batch delta (triangles holding a
batch edge), so the whole graph is not recounted on the CPU.

config 3: RMAT scale 24, edge factor 32 (a/b/c .57/.19/.19), the skewed
graph whose maximum degree (~1e5) exercises the blocked tier.  Pinned the
same way; BFS levels and CC labels exact, BC from the maximum-degree vertex
within 1e-9 (NaN where unreached), PageRank 2 iterations within 1e-9; then a
1e6-pair batch (same skew) inserted and deleted, with the adjacency compared
with the oracle's set model after each.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
REL_TOL = 1e-9
SYM = dict(symmetrize=True, drop_self_loops=True)
SWEEP = (10, 1000, 100000, 1000000)


def pins():
    with open(os.path.join(GOLD, "config_pins.json")) as f:
        return json.load(f)


def rel_close(a, b, tol=REL_TOL):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if not np.array_equal(np.isnan(a), np.isnan(b)):
        return False
    f = ~np.isnan(a)
    scale = np.maximum(np.abs(a[f]), np.abs(b[f]))
    return bool(np.all(np.abs(a[f] - b[f]) <= tol * np.maximum(scale, 1e-300)))


def csr_sha(off, tgt):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(off, "<u8").tobytes())
    h.update(np.ascontiguousarray(tgt, "<u4").tobytes())
    return h.hexdigest()


@pytest.fixture(scope="module")
def T():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    import terrace_b200
    return terrace_b200


def sweep_batch(T, n, i, k):
    """Batch i of the sweep: k RMAT pairs of seed stream 1 (the benchmark's
    sweep uses the same batches for its first trial of each size)."""
    return T.rmat_generate(n, O.batch_seed(1, 1000 + 100 * i), .5, .1, .1, k)


def check_state(g, off, tgt, src, tc):
    goff, gtgt = g.dump_csr()
    assert np.array_equal(goff, off) and np.array_equal(gtgt, tgt)
    assert g.check() == 0
    par, lv = g.bfs(src)
    assert np.array_equal(lv, O.bfs_levels(off, tgt, src))
    assert O.bfs_check_parents(off, tgt, src, lv, par) == 0
    assert np.array_equal(g.cc(), O.cc(off, tgt))
    assert rel_close(g.pagerank(10), O.pagerank(off, tgt, 10))
    assert g.tc() == tc


def test_config2_update_sweep_with_analytics(T):
    p = pins()["config2"]
    n = p["n"]
    s, d = T.rmat_generate(n, 0, .5, .1, .1, 16 * n, device=True)
    g = T.Graph(n)
    g.add_edge_batch(s, d, **SYM)
    del s, d
    off, tgt = g.dump_csr()
    assert g.get_num_edges() == p["m"]
    assert csr_sha(off, tgt) == p["csr_sha256"]   # = the oracle's graph
    keys = O.csr_keys(off, tgt)
    src = p["argmax_degree"]
    tc = p["tc_exact"]
    assert g.tc() == tc
    for i, k in enumerate(SWEEP):
        bs, bd = sweep_batch(T, n, i, k)
        bk = O.make_keys(bs, bd, True, True)
        new = O.key_difference(bk, keys)
        assert g.add_edge_batch(bs, bd, **SYM) == len(new)
        keys = O.key_union(keys, new)
        off, tgt = O.csr_from_keys(n, keys)
        tc += O.tc_touching(off, tgt, new)
        check_state(g, off, tgt, src, tc)
        gone = O.key_intersection(keys, bk)
        assert g.remove_edge_batch(bs, bd, **SYM) == len(gone)
        tc -= O.tc_touching(off, tgt, gone)
        keys = O.key_difference(keys, gone)
        off, tgt = O.csr_from_keys(n, keys)
        check_state(g, off, tgt, src, tc)
    g.close()


def test_config3_skewed_graph_analytics_and_updates(T):
    import torch
    p = pins()["config3"]
    n = p["n"]
    s, d = T.rmat_generate(n, 0, .57, .19, .19, 32 * n, device=True)
    g = T.Graph(n)
    g.add_edge_batch(s, d, **SYM)
    del s, d
    torch.cuda.empty_cache()
    off, tgt = g.dump_csr()
    assert g.get_num_edges() == p["m"]
    assert csr_sha(off, tgt) == p["csr_sha256"]   # = the oracle's graph
    st = g.stats()
    assert st["num_hubs"] > 0 and st["hub_edges"] > 0
    src = p["argmax_degree"]
    assert g.degree(src) == p["max_degree"]
    par, lv = g.bfs(src)
    assert np.array_equal(lv, O.bfs_levels(off, tgt, src))
    assert O.bfs_check_parents(off, tgt, src, lv, par) == 0
    del par, lv
    assert np.array_equal(g.cc(), O.cc(off, tgt))
    assert rel_close(g.bc(src), O.bc(off, tgt, src))
    assert rel_close(g.pagerank(2), O.pagerank(off, tgt, 2))
    # a 1e6-pair batch of the same skew: touches the largest hubs
    keys = O.csr_keys(off, tgt)
    del off, tgt
    bs, bd = T.rmat_generate(n, O.batch_seed(1, 0), .57, .19, .19, 1000000)
    bk = O.make_keys(bs, bd, True, True)
    new = O.key_difference(bk, keys)
    assert g.add_edge_batch(bs, bd, **SYM) == len(new)
    after = O.key_union(keys, new)
    goff, gtgt = g.dump_csr()
    woff, wtgt = O.csr_from_keys(n, after)
    assert np.array_equal(goff, woff) and np.array_equal(gtgt, wtgt)
    del goff, gtgt, woff, wtgt, after
    assert g.check() == 0
    assert g.remove_edge_batch(bs, bd, **SYM) == len(bk)   # every batch edge is present now
    goff, gtgt = g.dump_csr()
    woff, wtgt = O.csr_from_keys(n, O.key_difference(keys, bk))
    assert np.array_equal(goff, woff) and np.array_equal(gtgt, wtgt)
    assert g.check() == 0
    g.close()
