"""Batching layer: CUDA-graph replay of the PageRank iteration loop.

The replayed loop must give bit-identical ranks to direct launches (same
kernels, same order), across graph updates (the captured graph is patched
or re-captured when the class lists change), and the oracle's ranks within
1e-9 relative."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")


def test_pagerank_graph_replay_bit_identical():
    _gpu()
    import terrace_b200 as T
    n = 1 << 14
    s, d = O.rmat(n, 0, .5, .1, .1, 8 * n)
    gs = [T.Graph(n, hub_threshold=64, cuda_graphs=cg) for cg in (True, False)]
    for g in gs:
        g.add_edge_batch(s, d, symmetrize=True, drop_self_loops=True)
    for step in range(4):
        iters = (10, 10, 3, 10)[step]
        r = [g.pagerank(iters) for g in gs]
        assert np.array_equal(r[0], r[1]), step
        off, tgt = gs[0].dump_csr()
        ref = O.pagerank(off, tgt, iters)
        assert np.allclose(r[0], ref, rtol=1e-9, atol=0)
        # launches are counted for replays too: 1 init + 4 per iteration at most
        c0 = gs[0].launch_count()
        gs[0].pagerank(iters, device=True)
        assert 1 <= gs[0].launch_count() - c0 <= 1 + 4 * iters
        bs, bd = O.rmat(n, 100 + step, .5, .1, .1, 2000)
        for g in gs:
            g.add_edge_batch(bs, bd, symmetrize=True, drop_self_loops=True)


def test_autotuner_keeps_results_exact():
    """trc_autotune picks from its candidate sets, leaves the edge set and
    the structure invariants unchanged (the PMA trial inserts and removes the
    sample's absent edges), and later BFS / PageRank still match the oracle."""
    _gpu()
    import terrace_b200 as T
    n = 1 << 14
    s, d = O.rmat(n, 0, .5, .1, .1, 8 * n)
    g = T.Graph(n, hub_threshold=64)
    g.add_edge_batch(s, d, symmetrize=True, drop_self_loops=True)
    off0, tgt0 = g.dump_csr()
    src = int(np.argmax(np.diff(off0.astype(np.int64))))
    bs, bd = O.rmat(n, 77, .5, .1, .1, 4000)
    t = g.autotune(sample=(bs, bd))
    assert t["push_pull_divisor"] in (4, 8, 12, 16, 20, 32, 64)
    assert t["pr_group_lanes"] in (4, 8, 16) and t["pr_group_cut"] in (32, 64, 128)
    assert 1 <= t["pma_leaf_log"] <= 5
    assert t["bfs_ms"] > 0 and t["pagerank_iter_ms"] > 0 and t["pma_insert_ms"] > 0
    assert g.get_tuning()["pma_leaf_log"] == t["pma_leaf_log"]
    off1, tgt1 = g.dump_csr()
    assert np.array_equal(off0, off1) and np.array_equal(tgt0, tgt1)
    assert g.check() == 0
    _, lv = g.bfs(src)
    assert np.array_equal(lv, O.bfs_levels(off0, tgt0, src))
    ref = O.pagerank(off0, tgt0, 5)
    assert np.allclose(g.pagerank(5), ref, rtol=1e-9, atol=0)
    for lanes, cut in ((4, 32), (16, 128), (8, 64)):
        g.set_tuning(pr_group_lanes=lanes, pr_group_cut=cut, push_pull_divisor=7, pma_leaf_log=3)
        assert np.allclose(g.pagerank(5), ref, rtol=1e-9, atol=0)
        _, lv = g.bfs(src)
        assert np.array_equal(lv, O.bfs_levels(off0, tgt0, src))
    # inserts with a wider leaf keep the structure valid
    g.add_edge_batch(bs, bd, symmetrize=True, drop_self_loops=True)
    assert g.check() == 0
    with pytest.raises(T.TrcError) as e:
        g.set_tuning(pr_group_lanes=5)
    assert e.value.status == 1
