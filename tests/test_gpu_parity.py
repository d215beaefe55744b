"""GPU parity of the sm_100a library (through the C ABI) against the golden
fixtures recorded from the reference and against the CPU oracle.

Tolerances: lists, levels, labels and counts are compared exactly; PageRank
and BC are FP64 sums whose order differs (warp reductions here, atomics /
sequential sums in the reference), compared at relative 1e-9 (REL_TOL)."""
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


def load(name):
    return np.load(os.path.join(GOLD, name))


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


def graph_from_csr(T, off, tgt, **kw):
    n = len(off) - 1
    g = T.Graph(n, **kw)
    src = np.repeat(np.arange(n, dtype=np.uint32), np.diff(off.astype(np.int64)))
    g.add_edge_batch(src, tgt)
    return g


def assert_same_csr(g, off, tgt):
    goff, gtgt = g.dump_csr()
    assert np.array_equal(goff, off)
    assert np.array_equal(gtgt, tgt)
    assert g.check() == 0


def check_algorithms(g, off, tgt, rec=None, prefix=""):
    """BFS levels/parents, PR(5,10), CC, BC, TC against oracle (+ fixture)."""
    deg = np.diff(off.astype(np.int64))
    src = int(rec[prefix + "bfs_src"]) if rec is not None else int(deg.argmax())
    par, lv = g.bfs(src)
    want_lv = O.bfs_levels(off, tgt, src)
    assert np.array_equal(lv, want_lv)
    if rec is not None:
        assert np.array_equal(lv, rec[prefix + "bfs_levels"])
    assert O.bfs_check_parents(off, tgt, src, lv, par) == 0
    for it in (5, 10):
        pr = g.pagerank(it)
        assert rel_close(pr, O.pagerank(off, tgt, it))
        if rec is not None:
            assert rel_close(pr, rec[prefix + f"pr{it}"])
    assert rel_close(g.pagerank(7, damping=0.85), O.pagerank(off, tgt, 7, 0.85))
    cc = g.cc()
    assert np.array_equal(cc, O.cc(off, tgt))
    if rec is not None:
        assert np.array_equal(cc, rec[prefix + "cc"])
    bc = g.bc(src)
    assert rel_close(bc, O.bc(off, tgt, src))
    if rec is not None:
        assert rel_close(bc, rec[prefix + "bc"])
    assert g.tc() == O.tc(off, tgt)


def test_rmat_device_generator_bitexact(T):
    z = load("rmat_pin.npz")
    for i in range(3):
        n, seed, a, b, c = z[f"p{i}_params"]
        s, d = T.rmat_generate(int(n), int(seed), a, b, c, 4096, first=1000)
        assert np.array_equal(s, z[f"p{i}_src"]) and np.array_equal(d, z[f"p{i}_dst"])
    s, d = T.rmat_generate(1 << 20, 77, .57, .19, .19, 200000, first=123456789)
    os_, od = O.rmat(1 << 20, 77, .57, .19, .19, 200000, first=123456789)
    assert np.array_equal(s, os_) and np.array_equal(d, od)


@pytest.mark.parametrize("name", ["s12_updates.npz", "s12_skew.npz"])
@pytest.mark.parametrize("hub_threshold,stage", [(1024, 49152), (64, 49152), (64, 100)])
def test_update_sequence_matches_reference(T, name, hub_threshold, stage):
    """Bulk load, then every insert/delete batch of the fixture; the sorted
    adjacency must equal the reference's after each step.  stage=100 sends a
    hub block receiving more than 100 batch edges through the whole-hub
    rewrite instead of the block-local merge."""
    z = load(name)
    n = int(z["n"])
    g = graph_from_csr(T, z["s0_off"], z["s0_tgt"], hub_threshold=hub_threshold,
                       hub_stage_limit=stage)
    assert_same_csr(g, z["s0_off"], z["s0_tgt"])
    step, j = 1, 0
    while f"batch{j}_src" in z.files:
        bs, bd = z[f"batch{j}_src"], z[f"batch{j}_dst"]
        g.add_edge_batch(bs, bd, **SYM)
        assert_same_csr(g, z[f"s{step}_off"], z[f"s{step}_tgt"])
        g.remove_edge_batch(bs, bd, **SYM)
        assert_same_csr(g, z[f"s{step + 1}_off"], z[f"s{step + 1}_tgt"])
        step += 2
        j += 1
    assert g.get_num_vertices() == n


@pytest.mark.parametrize("name", ["s12_updates.npz", "s12_skew.npz"])
def test_algorithms_match_reference(T, name):
    z = load(name)
    g = graph_from_csr(T, z["s0_off"], z["s0_tgt"])
    check_algorithms(g, z["s0_off"], z["s0_tgt"], z, "s0_")
    last = int(z["steps"]) - 1
    g2 = graph_from_csr(T, z[f"s{last}_off"], z[f"s{last}_tgt"], hub_threshold=64)
    check_algorithms(g2, z[f"s{last}_off"], z[f"s{last}_tgt"], z, "final_")


def test_tc_matches_reference_exact_path(T):
    z = load("low_degree_tc.npz")
    off, tgt = O.csr_from_keys(int(z["n"]), z["keys"])
    g = graph_from_csr(T, off, tgt)
    assert g.tc() == int(z["ref_tc"]) == 12000


def test_static_workload_rmat17(T):
    """RMAT scale 17 ef 8 seed 0 (bulk load + BFS from 9 and from the
    max-degree vertex, PR 5, CC, BC, TC) against the reference summary."""
    with open(os.path.join(GOLD, "config1_summary.json")) as f:
        s = json.load(f)
    n = 1 << 17
    src, dst = T.rmat_generate(n, 0, .5, .1, .1, 8 * n)
    g = T.Graph(n)
    g.add_edge_batch(src, dst, **SYM)
    assert g.get_num_edges() == s["m"]
    off, tgt = g.dump_csr()
    assert csr_sha(off, tgt) == s["csr_sha256"]
    assert g.check() == 0
    for v in (9, s["argmax_degree"]):
        par, lv = g.bfs(v)
        assert hashlib.sha256(lv.astype("<u4").tobytes()).hexdigest() == s[f"bfs{v}_levels_sha256"]
        assert O.bfs_check_parents(off, tgt, v, lv, par) == 0
    sample = np.array(s["sample"])
    pr = g.pagerank(5)
    assert rel_close(pr[sample], np.array(s["pr5_sample"]))
    assert abs(pr.sum() - s["pr5_sum"]) <= 1e-9 * s["pr5_sum"]
    cc = g.cc()
    assert hashlib.sha256(cc.astype("<u4").tobytes()).hexdigest() == s["cc_sha256"]
    bc = g.bc(s["bc_src"])
    ref = np.array([np.nan if x is None else x for x in s["bc_sample"]])
    assert rel_close(bc[sample], ref)
    assert g.tc() == s["tc_exact_rmat17"] == 758730


def test_set_semantics_edge_cases(T):
    g = T.Graph(100, hub_threshold=20)
    assert g.add_edge_batch(np.array([], np.uint32), np.array([], np.uint32)) == 0
    # duplicates and both directions
    assert g.add_edge_batch([1, 1, 2, 1], [5, 5, 1, 5]) == 2
    assert g.degree(1) == 1 and g.degree(2) == 1
    assert list(g.neighbors(1)) == [5]
    assert g.add_edge(1, 5) == -1 and g.add_edge(5, 1) == 0
    # self loops kept unless dropped
    assert g.add_edge_batch([7], [7]) == 1
    assert g.add_edge_batch([8], [8], drop_self_loops=True) == 0
    # removing absent edges is a no-op (the reference would drop a neighbour)
    assert g.remove_edge_batch([1, 3], [6, 4]) == 0
    assert g.remove_edge(1, 5) == 0 and g.remove_edge(1, 5) == -1
    # out-of-range ids fail with TRC_ERR_INVALID and leave the graph unchanged
    m = g.get_num_edges()
    with pytest.raises(T.TrcError) as e:
        g.add_edge_batch([1, 200], [2, 3])
    assert e.value.status == 1
    assert g.get_num_edges() == m
    with pytest.raises(T.TrcError):
        g.degree(100)
    # grow a vertex through every tier: inline -> PMA -> hub, then shrink
    nb = np.arange(30, 100, dtype=np.uint32)
    g.add_edge_batch(np.full(len(nb), 0, np.uint32), nb, symmetrize=True)
    assert list(g.neighbors(0)) == list(nb)
    assert g.stats()["num_hubs"] >= 1
    assert g.check() == 0
    g.remove_edge_batch(np.full(60, 0, np.uint32), nb[:60], symmetrize=True)
    assert list(g.neighbors(0)) == list(nb[60:])
    assert g.check() == 0
    assert g.is_edge(0, 99) == 1 and g.is_edge(0, 30) == 0
    assert g.count_common(0, 95) == 0


def test_random_updates_against_set_model(T):
    """Random inserts/deletes with small tier thresholds, checked against the
    oracle's set model after every batch (exercises window rebalances, PMA
    rebuilds, hub promotion and hub region growth)."""
    rng = np.random.default_rng(1)
    n = 3000
    g = T.Graph(n, hub_threshold=48, hub_stage_limit=400)
    cur = np.zeros(0, np.uint64)
    for step in range(14):
        k = int(rng.integers(1, 20000))
        s = rng.integers(0, n, k).astype(np.uint32)
        # skew: a few vertices get many edges
        s[: k // 3] = rng.integers(0, 20, k // 3).astype(np.uint32)
        d = rng.integers(0, n, k).astype(np.uint32)
        bk = O.make_keys(s, d, True, True)
        if step % 3 == 2:
            g.remove_edge_batch(s, d, **SYM)
            cur = O.key_difference(cur, bk)
        else:
            g.add_edge_batch(s, d, **SYM)
            cur = O.key_union(cur, bk)
        off, tgt = O.csr_from_keys(n, cur)
        assert_same_csr(g, off, tgt)
    st = g.stats()
    assert st["num_hubs"] > 0 and st["pma_rebuilds"] >= 1
    check_algorithms(g, off, tgt)
    # queries
    qs = rng.integers(0, n, 5000).astype(np.uint32)
    qd = rng.integers(0, n, 5000).astype(np.uint32)
    want = np.isin((qs.astype(np.uint64) << np.uint64(32)) | qd.astype(np.uint64), cur)
    assert np.array_equal(g.is_edge(qs, qd).astype(bool), want)
    assert np.array_equal(g.degree(qs), np.diff(off.astype(np.int64))[qs].astype(np.uint32))
    cc_q = g.count_common(qs[:500], qd[:500])
    for a, b, c in zip(qs[:500], qd[:500], cc_q):
        na = set(tgt[off[a]:off[a + 1]].tolist())
        nb = set(tgt[off[b]:off[b + 1]].tolist())
        assert c == sum(1 for w in na & nb if w < min(a, b))


def test_back_to_back_batches_defer_their_tails(T):
    """Batch calls return with their last kernels still queued, and a host
    batch that follows at once copies its input on a second stream while
    they run.  Graph A takes batches back to back from two reused host
    arrays (overwritten right after each call returns) and device tensors;
    graph B takes the same batches with a query after each (every query
    waits for the tail).  Both must equal the oracle's set model, and their
    counters (tier-3 free list, splits, the last batch's rewrite counts)
    must agree."""
    import torch
    rng = np.random.default_rng(5)
    n = 3000
    kw = dict(hub_threshold=48, hub_stage_limit=400)
    ga, gb = T.Graph(n, **kw), T.Graph(n, **kw)
    sizes = [20000, 5000, 19000, 1, 700, 15000, 20000, 300, 12000, 20000, 9000, 4, 18000, 20000]
    hs = np.zeros(max(sizes), np.uint32)
    hd = np.zeros(max(sizes), np.uint32)
    cur = np.zeros(0, np.uint64)
    for step, k in enumerate(sizes):
        s = rng.integers(0, n, k).astype(np.uint32)
        s[: k // 3] = rng.integers(0, 20, k // 3).astype(np.uint32)
        d = rng.integers(0, n, k).astype(np.uint32)
        bk = O.make_keys(s, d, True, True)
        ins = step % 3 != 2
        hs[:k], hd[:k] = s, d
        if step % 4 == 3:  # device input
            ts_, td_ = torch.from_numpy(s.view(np.int32)).cuda(), torch.from_numpy(d.view(np.int32)).cuda()
            torch.cuda.synchronize()  # the graph's own stream does not wait for torch's
            ta = ga.add_edge_batch if ins else ga.remove_edge_batch
            ca = ta(ts_, td_, **SYM)
        else:
            ta = ga.add_edge_batch if ins else ga.remove_edge_batch
            ca = ta(hs[:k], hd[:k], **SYM)
            hs[:k] = 7  # the caller may reuse its arrays at once
            hd[:k] = 9
        tb = gb.add_edge_batch if ins else gb.remove_edge_batch
        cb = tb(s, d, **SYM)
        gb.get_num_edges()
        cur = O.key_union(cur, bk) if ins else O.key_difference(cur, bk)
        assert ca == cb
    off, tgt = O.csr_from_keys(n, cur)
    sa, sb = ga.stats(), gb.stats()
    sa.pop("device_bytes")
    sb.pop("device_bytes")
    assert sa == sb
    assert sa["num_hubs"] > 0 and sa["last_rewritten"] > 0
    assert_same_csr(ga, off, tgt)
    assert_same_csr(gb, off, tgt)
    # a batch straight after another, then an analytic: the analytic waits
    ga.add_edge_batch(s, d, **SYM)
    ga.remove_edge_batch(s, d, **SYM)
    cur = O.key_difference(cur, bk)
    off, tgt = O.csr_from_keys(n, cur)
    assert np.array_equal(ga.bfs(int(s[0]))[1], O.bfs_levels(off, tgt, int(s[0])))
    assert_same_csr(ga, off, tgt)


@pytest.mark.parametrize("mode", [1, 2])
def test_batch_sort_modes_agree_with_oracle(T, mode):
    """The bucket sort (mode 2: every batch) and the radix sort (mode 1) give
    the same graph as the oracle's set model over batches of 1..2e5 keys
    (empty buckets, dropped self loops, buckets of every size tier); a batch
    with a source of more than 16384 keys goes back to the radix sort before
    the graph is modified (sort_retries counts it)."""
    from terrace_b200 import _lib
    rng = np.random.default_rng(7 + mode)
    n = 40000
    g = T.Graph(n, hub_threshold=64)
    _lib.check(g._L.trc_debug_sort_mode(g._h, mode))
    cur = np.zeros(0, np.uint64)
    sizes = [1, 2, 17, 33, 300, 1025, 4096, 20000, 100000]
    for step, k in enumerate(sizes):
        s = rng.integers(0, n, k).astype(np.uint32)
        d = rng.integers(0, n, k).astype(np.uint32)
        if k >= 300:  # skew: runs of equal sources of every bucket tier
            a, b = min(k // 4, 6000), min(k // 8, 12000)
            s[:a] = rng.integers(0, 8, a).astype(np.uint32)
            s[a:a + b] = 12345
        bk = O.make_keys(s, d, True, True)
        if step % 4 == 3:
            g.remove_edge_batch(s, d, **SYM)
            cur = O.key_difference(cur, bk)
        else:
            g.add_edge_batch(s, d, **SYM)
            cur = O.key_union(cur, bk)
        assert_same_csr(g, *O.csr_from_keys(n, cur))
    assert g.stats()["sort_retries"] == 0
    # one source with 20000 distinct neighbours in one batch: its bucket is
    # above the bucket sort's limit
    d = rng.permutation(n)[:20000].astype(np.uint32)
    s = np.full(20000, 77, np.uint32)
    g.add_edge_batch(s, d, **SYM)
    cur = O.key_union(cur, O.make_keys(s, d, True, True))
    assert_same_csr(g, *O.csr_from_keys(n, cur))
    assert g.stats()["sort_retries"] == (1 if mode == 2 else 0)
    assert g.check() == 0
    g.close()


@pytest.mark.parametrize("n", [1, 3, 70])
def test_batch_sort_tiny_graphs_large_batches(T, n):
    """Batches of 10,000-60,000 pairs on graphs of 1, 3 and 70 vertices
    (every bucket holds thousands of duplicates, self loops dropped, one
    vertex: every key invalid), in every sort mode: the oracle's edge set
    after each batch."""
    from terrace_b200 import _lib
    rng = np.random.default_rng(n)
    for mode in (0, 1, 2):
        g = T.Graph(n)
        _lib.check(g._L.trc_debug_sort_mode(g._h, mode))
        cur = np.zeros(0, np.uint64)
        for step, k in enumerate((10000, 60000, 30000)):
            s = rng.integers(0, n, k).astype(np.uint32)
            d = rng.integers(0, n, k).astype(np.uint32)
            bk = O.make_keys(s, d, True, True)
            if step == 2:
                g.remove_edge_batch(s[: k // 2], d[: k // 2], **SYM)
                cur = O.key_difference(cur, O.make_keys(s[: k // 2], d[: k // 2], True, True))
            else:
                g.add_edge_batch(s, d, **SYM)
                cur = O.key_union(cur, bk)
            assert_same_csr(g, *O.csr_from_keys(n, cur))
        assert g.check() == 0
        g.close()


def test_streaming_rmat22_roundtrip_and_parity(T):
    """LiveJournal-shaped RMAT scale 22 ef 16: bulk load and one 1e6-pair
    insert + delete batch.  Parity with the oracle's set model by CSR hash,
    plus the size-independent round trip (insert then delete of a fresh
    batch restores the original hash)."""
    n = 1 << 22
    s, d = T.rmat_generate(n, 0, .5, .1, .1, 16 * n)
    g = T.Graph(n)
    g.add_edge_batch(s, d, **SYM)
    n_, keys = O.rmat_graph_keys(22, 16, .5, .1, .1, 0)
    off, tgt = g.dump_csr()
    woff, wtgt = O.csr_from_keys(n, keys)
    assert np.array_equal(off, woff) and np.array_equal(tgt, wtgt)
    h0 = csr_sha(off, tgt)
    bs, bd = T.rmat_generate(n, O.batch_seed(1, 0), .5, .1, .1, 1000000)
    bk = O.make_keys(bs, bd, True, True)
    fresh = O.key_difference(bk, keys)
    fs, fd = O.keys_to_pairs(fresh)
    assert g.add_edge_batch(fs, fd) == len(fresh)
    off1, tgt1 = g.dump_csr()
    w1off, w1tgt = O.csr_from_keys(n, O.key_union(keys, bk))
    assert np.array_equal(off1, w1off) and np.array_equal(tgt1, w1tgt)
    assert g.check() == 0
    assert g.remove_edge_batch(fs, fd) == len(fresh)
    assert csr_sha(*g.dump_csr()) == h0
    assert g.check() == 0


def test_bfs_into_unaligned_device_arrays(T):
    """trc_bfs writing into caller device arrays that start 4 bytes past a
    16-byte boundary (the initialisation then takes its scalar path) gives
    the same parents and levels as into its own arrays."""
    import ctypes as C
    import torch
    from terrace_b200 import _lib
    n = 1 << 12
    s, d = T.rmat_generate(n, 3, .5, .1, .1, 8 * n)
    g = T.Graph(n, hub_threshold=64)
    g.add_edge_batch(s, d, **SYM)
    par0, lv0 = g.bfs(0)
    par = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    lv = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    _lib.check(g._L.trc_bfs(g._h, 0, C.c_void_p(par.data_ptr() + 4), C.c_void_p(lv.data_ptr() + 4),
                            _lib.TRC_DEVICE_PTR))
    torch.cuda.synchronize()
    assert np.array_equal(lv[1:].cpu().numpy().view(np.uint32), lv0)
    p = par[1:].cpu().numpy()
    assert np.array_equal(p >= 0, par0 >= 0)
    g.close()


def test_large_graph_pagerank_bfs_cc(T):
    """RMAT scale 23 (8.4M vertices, rank vector 67 MB): PageRank, CC, and
    BFS through several dense steps with candidate compaction."""
    n = 1 << 23
    s, d = T.rmat_generate(n, 5, .57, .19, .19, 4 * n)
    g = T.Graph(n)
    g.add_edge_batch(s, d, **SYM)
    keys = O.make_keys(s, d, True, True)
    off, tgt = O.csr_from_keys(n, keys)
    goff, gtgt = g.dump_csr()
    assert np.array_equal(goff, off) and np.array_equal(gtgt, tgt)
    assert rel_close(g.pagerank(3), O.pagerank(off, tgt, 3))
    assert rel_close(g.pagerank(2, damping=0.85), O.pagerank(off, tgt, 2, 0.85))
    src = int(np.diff(off.astype(np.int64)).argmax())
    par, lv = g.bfs(src)
    assert np.array_equal(lv, O.bfs_levels(off, tgt, src))
    assert O.bfs_check_parents(off, tgt, src, lv, par) == 0
    assert np.array_equal(g.cc(), O.cc(off, tgt))


@pytest.mark.parametrize("n_log,k", [(10, 5), (16, 64), (20, 33)])
def test_msbfs_equals_single_source_bfs(T, n_log, k):
    """Multi-source BFS (k sources as bits of one 64-bit mask per vertex)
    gives, for every source, exactly the levels of a single-source BFS;
    the small graph exercises pull steps, the large ones push then pull."""
    n = 1 << n_log
    s, d = T.rmat_generate(n, 11, .57, .19, .19, 8 * n)
    g = T.Graph(n, hub_threshold=64)
    g.add_edge_batch(s, d, **SYM)
    off, tgt = g.dump_csr()
    rng = np.random.default_rng(n_log)
    deg = np.diff(off.astype(np.int64))
    cand = np.nonzero(deg > 0)[0]
    srcs = rng.choice(cand, k, replace=False).astype(np.uint32)
    srcs[0] = 0 if deg[0] == 0 else srcs[0]   # an isolated source when vertex 0 is isolated
    lv = g.msbfs(srcs)
    assert lv.shape == (k, n)
    for i in range(k):
        assert np.array_equal(lv[i], O.bfs_levels(off, tgt, int(srcs[i]))), i


@pytest.mark.parametrize("n_log,k", [(10, 5), (14, 64), (17, 40)])
def test_msbc_equals_single_source_bc(T, n_log, k):
    """Multi-source BC (k sources in one traversal) gives, for every source,
    the oracle's BC (the reference's Brandes variant) within 1e-9 relative,
    NaN exactly where the source does not reach; sources include a repeated
    vertex and, when present, an isolated one."""
    n = 1 << n_log
    s, d = T.rmat_generate(n, 13, .57, .19, .19, 8 * n)
    g = T.Graph(n, hub_threshold=64)
    g.add_edge_batch(s, d, **SYM)
    off, tgt = g.dump_csr()
    rng = np.random.default_rng(n_log + 100)
    deg = np.diff(off.astype(np.int64))
    cand = np.nonzero(deg > 0)[0]
    srcs = rng.choice(cand, k, replace=False).astype(np.uint32)
    if k > 2:
        srcs[1] = srcs[0]                       # the same source twice
    iso = np.nonzero(deg == 0)[0]
    if len(iso) and k > 3:
        srcs[2] = iso[0]
    out = g.msbc(srcs)
    assert out.shape == (k, n)
    for i in range(k):
        want = O.bc(off, tgt, int(srcs[i]))
        nan = np.isnan(want)
        assert np.array_equal(np.isnan(out[i]), nan), i
        assert rel_close(out[i][~nan], want[~nan]), i


@pytest.mark.parametrize("stage", [49152, 100])
def test_blocked_tier_block_local_updates(T, stage):
    """A hub of degree 100,000 (blocked tier, the reference's per-vertex
    B-tree) under small and concentrated batches, every step matching the
    oracle's set model: deletes that leave every other block under-full merge
    those blocks with their untouched successors; scattered inserts land in
    the touched blocks only (elements written scale with the blocks touched,
    not with the hub's degree); a dense insert into one key range splits
    blocks; deletes of a run empty whole blocks; deletes of the smallest
    neighbours refill the inline row from the blocks; the hub shrinks into
    its inline row and grows back.  stage=100 sends groups of more than 100
    keys through the whole-hub rewrite instead."""
    rng = np.random.default_rng(7)
    n = 1 << 18
    hub = 7
    nb = np.sort(rng.choice(np.arange(1000, n, dtype=np.uint32), 100000, replace=False))
    s, d = T.rmat_generate(n, 3, .5, .1, .1, 4 * n)
    s, d = s[(s != hub) & (d != hub)], d[(s != hub) & (d != hub)]   # the hub's edges: nb only
    g = T.Graph(n, hub_stage_limit=stage)
    g.add_edge_batch(np.concatenate([s, np.full(len(nb), hub, np.uint32)]),
                     np.concatenate([d, nb]), **SYM)
    cur = O.key_union(O.make_keys(s, d, True, True),
                      O.make_keys(np.full(len(nb), hub, np.uint32), nb, True, True))
    assert g.degree(hub) == len(nb)

    def hub_list():
        off, tgt = O.csr_from_keys(n, cur)
        return tgt[off[hub]:off[hub + 1]].copy()

    def step(dst, insert):
        nonlocal cur
        src = np.full(len(dst), hub, np.uint32)
        bk = O.make_keys(src, np.asarray(dst, np.uint32), True, True)
        if insert:
            g.add_edge_batch(src, dst, **SYM)
            cur = O.key_union(cur, bk)
        else:
            g.remove_edge_batch(src, dst, **SYM)
            cur = O.key_difference(cur, bk)
        off, tgt = O.csr_from_keys(n, cur)
        assert_same_csr(g, off, tgt)
        return g.stats(), off, tgt

    # 1. the bulk load filled blocks of `per` elements: empty most of every
    # other block (30 left), whose untouched successor then joins it
    rest = len(nb) - 16
    per = -(-rest // -(-rest // 192))
    hl = hub_list()
    ranks = np.concatenate([np.arange(j * per + 10, j * per + per - 20)
                            for j in range(0, rest // per - 1, 2)]) + 16
    st, _, _ = step(hl[ranks], False)
    if stage > 100:
        assert st["last_hub_local"] == 1 and st["hub_absorbs"] > 100
    # 2. fifty scattered new neighbours: block-local, few blocks written
    hl = hub_list()
    absent = np.setdiff1d(np.arange(1000, n, dtype=np.uint32), hl)
    new = rng.choice(absent, 50, replace=False).astype(np.uint32)
    st, _, _ = step(new, True)
    assert st["last_hub_touched"] >= 1
    if stage > 100:
        assert st["last_hub_local"] >= 1
        assert st["last_hub_written"] < 50 * 300 + 5000   # not the hub's ~75,000
    # 3. a dense range of 3,000 new neighbours: splits (stage=100: a rewrite)
    hl = hub_list()
    lo = int(hl[len(hl) // 2])
    dense = np.setdiff1d(np.arange(lo, lo + 40000, dtype=np.uint32), hl)[:3000]
    splits0 = st["hub_splits"]
    st, _, _ = step(dense, True)
    if stage > 100:
        assert st["hub_splits"] > splits0 and st["last_hub_rewritten"] == 0
    else:
        assert st["last_hub_rewritten"] >= 1
    # 4. delete a run of 2,000 consecutive neighbours: whole blocks emptied
    hl = hub_list()
    free0 = st["hub_blocks_free"]
    st, _, _ = step(hl[30000:32000], False)
    if stage > 100:
        assert st["hub_blocks_free"] > free0
    # 5. delete the 300 smallest neighbours: the inline row refills
    hl = hub_list()
    st, off, tgt = step(hl[:300], False)
    assert g.check() == 0
    check_algorithms(g, off, tgt)
    # 6. the hub shrinks into its inline row and grows back
    hl = hub_list()
    st, _, _ = step(hl[:-10], False)
    assert g.degree(hub) == 10
    st, off, tgt = step(hl, True)
    assert g.check() == 0
    g.close()


def test_bc_and_bfs_from_isolated_and_leaf_sources(T):
    """Single-source BC (and BFS) from an isolated vertex and from a vertex of
    degree one, against the oracle: the reference's backward step adds
    1/sigma to every vertex of every level, the source included, so an
    isolated source ends at 0 and every other vertex at NaN."""
    n = 1 << 12
    s, d = T.rmat_generate(n, 0, .5, .1, .1, 4 * n)
    g = T.Graph(n, hub_threshold=64)
    g.add_edge_batch(s, d, **SYM)
    off, tgt = g.dump_csr()
    deg = np.diff(off.astype(np.int64))
    for src in (int(np.flatnonzero(deg == 0)[0]), int(np.flatnonzero(deg == 1)[0]),
                int(deg.argmax())):
        assert rel_close(g.bc(src), O.bc(off, tgt, src)), src
        par, lv = g.bfs(src)
        assert np.array_equal(lv, O.bfs_levels(off, tgt, src))
        assert O.bfs_check_parents(off, tgt, src, lv, par) == 0
    g.close()


def test_blocked_tier_random_batches(T):
    """Three hubs of 12,000-40,000 neighbours (block-local path) under forty
    random insert and delete batches of 1..5,000 edges each, some spread over
    the whole list and some packed into one key range, compared with the
    oracle's set model after every batch."""
    rng = np.random.default_rng(11)
    n = 1 << 17
    hubs = np.array([3, 70000, 131000], np.uint32)
    s, d = T.rmat_generate(n, 9, .5, .1, .1, 2 * n)
    keep = ~np.isin(s, hubs) & ~np.isin(d, hubs)
    s, d = s[keep], d[keep]
    hs = np.concatenate([np.full(k, h, np.uint32) for h, k in zip(hubs, (12000, 25000, 40000))])
    hd = np.concatenate([rng.choice(n, k, replace=False).astype(np.uint32)
                         for k in (12000, 25000, 40000)])
    g = T.Graph(n)
    g.add_edge_batch(np.concatenate([s, hs]), np.concatenate([d, hd]), **SYM)
    cur = O.make_keys(np.concatenate([s, hs]), np.concatenate([d, hd]), True, True)
    local = 0
    for step in range(40):
        h = hubs[rng.integers(0, 3)]
        k = int(rng.integers(1, 5000))
        if rng.random() < 0.5:
            dst = rng.integers(0, n, k).astype(np.uint32)
        else:
            lo = int(rng.integers(0, n - 4000))
            dst = rng.integers(lo, lo + 4000, k).astype(np.uint32)
        src = np.full(k, h, np.uint32)
        bk = O.make_keys(src, dst, True, True)
        if step % 2:
            g.remove_edge_batch(src, dst, **SYM)
            cur = O.key_difference(cur, bk)
        else:
            g.add_edge_batch(src, dst, **SYM)
            cur = O.key_union(cur, bk)
        local += g.stats()["last_hub_local"]
        off, tgt = O.csr_from_keys(n, cur)
        assert_same_csr(g, off, tgt)
    assert local > 10
    check_algorithms(g, off, tgt)
    g.close()
