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
