"""Serving layer: every result served in a mix equals the same request run
alone on the snapshot it recorded.

A random stream of interleaved inserts, deletes (sizes from 1 to 2,000
pairs), BFS, degree, neighbour-list and PageRank requests is submitted to a
trc_server; requests arriving while a round runs on the GPU join the next
round (continuous batching: BFS packed into multi-source launches, updates
of a round merged into one net change).  Replay: a fresh graph gets the
same initial edges, then the update requests one by one in arrival order;
after the updates of version v every query that recorded version v runs
alone through the plain Graph calls.  BFS levels, degrees and neighbour
lists must be identical; PageRank within 1e-9 relative (FP64).  The replay
also keeps the oracle's edge set: the first served BFS of every version
must equal the oracle's levels on it, and the replayed graph must equal it
at the end."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

N_SCALE = 13


def _gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")


def _initial(T, n, seed=5):
    s, d = O.rmat(n, seed, .5, .1, .1, 6 * n)
    g = T.Graph(n, hub_threshold=64, hub_stage_limit=400)
    g.add_edge_batch(s, d, symmetrize=True, drop_self_loops=True)
    return g, (s, d)


def _stream(n, count, seed):
    rng = np.random.default_rng(seed)
    reqs = []
    for _ in range(count):
        x = rng.random()
        if x < 0.55:
            k = int(np.exp(rng.uniform(0, np.log(2000))))
            src = rng.integers(0, n, k, dtype=np.uint32)
            # half of the pairs land among low ids so requests overlap
            dst = rng.integers(0, n if rng.random() < .5 else 64, k, dtype=np.uint32)
            reqs.append(("ins" if rng.random() < .5 else "del", src, dst))
        elif x < 0.80:
            reqs.append(("bfs", int(rng.integers(0, n)), None))
        elif x < 0.88:
            reqs.append(("deg", rng.integers(0, n, int(rng.integers(1, 50)), dtype=np.uint32), None))
        elif x < 0.95:
            reqs.append(("nbr", int(rng.integers(0, 64)), None))
        else:
            reqs.append(("pr", int(rng.integers(1, 4)), None))
    return reqs


def _serve(T, server, reqs):
    ids = []
    for kind, a, b in reqs:
        if kind == "ins":
            ids.append(server.insert(a, b))
        elif kind == "del":
            ids.append(server.delete(a, b))
        elif kind == "bfs":
            ids.append(server.bfs(a))
        elif kind == "deg":
            ids.append(server.degree(a))
        elif kind == "nbr":
            ids.append(server.neighbors(a))
        else:
            ids.append(server.pagerank(a))
    out = []
    for (kind, _, _), rid in zip(reqs, ids):
        server.wait(rid, 60000)
        dt = np.float64 if kind == "pr" else np.uint32
        arr, lat, ver, st = server.result(rid, dt)
        out.append((arr.copy(), ver, st))
        server.release(rid)
    return out


def _replay_and_check(T, n, reqs, served, summary=False):
    g, (s0, d0) = _initial(T, n)
    keys = O.make_keys(s0, d0, True, True)  # the oracle's edge set, replayed alongside
    by_version = {}
    for i, (kind, _, _) in enumerate(reqs):
        if kind not in ("ins", "del"):
            by_version.setdefault(served[i][1], []).append(i)
    upd = [i for i, (k, _, _) in enumerate(reqs) if k in ("ins", "del")]
    versions = sorted(set(by_version) | {served[i][1] for i in upd})
    checked = 0
    ui = 0
    for v in versions:
        while ui < len(upd) and served[upd[ui]][1] <= v:
            kind, a, b = reqs[upd[ui]]
            assert served[upd[ui]][2] == 0
            if kind == "ins":
                g.add_edge_batch(a, b, symmetrize=True, drop_self_loops=True)
                keys = O.key_union(keys, O.make_keys(a, b, True, True))
            else:
                g.remove_edge_batch(a, b, symmetrize=True, drop_self_loops=True)
                keys = O.key_difference(keys, O.make_keys(a, b, True, True))
            ui += 1
        # the replayed graph and the served BFS levels pinned to the oracle
        # too (the first BFS of each version), not only to the library
        off, tgt = O.csr_from_keys(n, keys)
        bfs_here = [i for i in by_version.get(v, []) if reqs[i][0] == "bfs"]
        if bfs_here and not summary:
            i = bfs_here[0]
            assert np.array_equal(served[i][0], O.bfs_levels(off, tgt, reqs[i][1])), (i, v)
        for i in by_version.get(v, []):
            kind, a, _ = reqs[i]
            arr, _, st = served[i]
            assert st == 0, (i, kind, st)
            if kind == "bfs":
                _, lv = g.bfs(a)
                if summary:
                    r = lv != T.TRC_UNREACHED
                    assert arr.tolist() == [int(r.sum()), int(lv[r].max())], (i, v)
                else:
                    assert np.array_equal(arr, lv), (i, v)
            elif kind == "deg":
                assert np.array_equal(arr, g.degree(a)), (i, v)
            elif kind == "nbr":
                assert np.array_equal(arr, g.neighbors(a)), (i, v)
            else:
                x = g.pagerank(a)
                if summary:
                    ref = np.array([x.sum(), x.max()])
                else:
                    ref = x
                assert np.allclose(arr, ref, rtol=1e-9, atol=0), (i, v)
            checked += 1
    assert ui == len(upd)
    off, tgt = O.csr_from_keys(n, keys)
    goff, gtgt = g.dump_csr()
    assert np.array_equal(goff, off) and np.array_equal(gtgt, tgt)
    return checked


@pytest.mark.parametrize("batched,summary", [(True, False), (True, True), (False, False)])
def test_served_results_equal_alone(batched, summary):
    _gpu()
    import terrace_b200 as T
    n = 1 << N_SCALE
    reqs = _stream(n, 400 if batched else 150, seed=11 + batched + 2 * summary)
    g, _ = _initial(T, n)
    srv = T.Server(g, batched=batched, summary=summary)
    served = _serve(T, srv, reqs)
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(reqs)
    if batched:
        assert st["rounds"] < len(reqs)  # requests were served together
    else:
        assert st["rounds"] == len(reqs)
    checked = _replay_and_check(T, n, reqs, served, summary=summary)
    assert checked > 0


def test_server_admission_and_errors():
    _gpu()
    import terrace_b200 as T
    from terrace_b200 import _lib
    n = 1 << 12
    s, d = O.rmat(n, 5, .5, .1, .1, 4 * n)
    g = T.Graph(n, hbm_budget=96 << 20, hub_threshold=64)
    g.add_edge_batch(s, d, symmetrize=True, drop_self_loops=True)
    m0 = g.get_num_edges()
    srv = T.Server(g, batched=True)
    rng = np.random.default_rng(1)
    big = rng.integers(0, n, 4 << 20, dtype=np.uint32)
    r_big = srv.insert(big, big[::-1].copy())   # beyond the HBM budget
    r_bad = srv.bfs(n + 5)                      # invalid source
    r_ok = srv.degree(np.arange(16, dtype=np.uint32))
    for r in (r_big, r_bad, r_ok):
        srv.wait(r, 60000)
    _, _, _, st_big = srv.result(r_big)
    _, _, _, st_bad = srv.result(r_bad)
    deg, _, ver, st_ok = srv.result(r_ok)
    assert st_big == _lib.TRC_ERR_NOMEM
    assert st_bad == _lib.TRC_ERR_INVALID
    assert st_ok == 0 and ver == 0
    stats = srv.stats()
    assert stats["rejected"] >= 1
    srv.close()
    assert g.get_num_edges() == m0
    assert np.array_equal(deg, g.degree(np.arange(16, dtype=np.uint32)))


def test_large_round_wide_vertex_ids():
    """A round of 300 update requests on a graph with 25-bit vertex ids: the
    round's tagged sort key (src, dst, arrival rank, op) needs all of its
    bits; the net change must equal the requests applied one by one."""
    _gpu()
    import terrace_b200 as T
    n = 1 << 25
    g = T.Graph(n)
    rng = np.random.default_rng(7)
    srv = T.Server(g, batched=True)
    srv.hold(True)
    reqs, ids = [], []
    for i in range(300):
        k = int(rng.integers(1, 40))
        # overlapping endpoints across requests (low ids), plus high ids
        a = rng.integers(0, 4096, k, dtype=np.uint32)
        b = np.where(rng.random(k) < .5, rng.integers(0, 4096, k), rng.integers(n - 4096, n, k))
        b = b.astype(np.uint32)
        op = "ins" if (i < 20 or rng.random() < .6) else "del"
        reqs.append((op, a, b))
        ids.append(srv.insert(a, b) if op == "ins" else srv.delete(a, b))
    srv.hold(False)
    for rid in ids:
        srv.wait(rid, 120000)
        _, _, ver, st = srv.result(rid)
        assert st == 0
        assert ver == 1  # one round, one net change
        srv.release(rid)
    assert srv.stats()["rounds"] == 1
    tr = srv.rounds()
    assert len(tr) == 1 and tr[0]["updates"] == 300 and tr[0]["bfs"] == 0
    assert tr[0]["update_pairs"] == sum(len(a) for _, a, _ in reqs)
    assert tr[0]["ms"] >= tr[0]["update_ms"] > 0
    srv.close()
    keys = np.zeros(0, np.uint64)
    for op, a, b in reqs:
        kk = O.make_keys(a, b, True, True)
        keys = O.key_union(keys, kk) if op == "ins" else O.key_difference(keys, kk)
    assert g.get_num_edges() == len(keys)
    us = np.unique((keys >> np.uint64(32)).astype(np.uint32))
    for u in us[:: max(1, len(us) // 200)]:
        want = (keys[(keys >> np.uint64(32)) == u] & np.uint64(0xFFFFFFFF)).astype(np.uint32)
        assert np.array_equal(g.neighbors(int(u)), want), u
    g.close()
