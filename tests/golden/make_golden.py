"""Generate the golden fixtures in tests/golden/ by running the UNMODIFIED
reference Terrace (oracle/_ref/libterrace_ref.so, built by oracle/build_ref.sh
from the reference sources) on seeded RMAT graphs and update batches.

Run from the repository root after oracle/build_ref.sh:

    python tests/golden/make_golden.py

The reference runs with ONE OpenMP thread: its parallel remove_edge races on
the last vertex (observed: 1 failed remove out of 115,598 with 8 threads on an
RMAT scale-14 graph, none with 1 thread), and its neighbour iterator can
return the last vertex's list out of order (a PMA edge case), so every list
is sorted per vertex before it is recorded.

Fixtures:
  rmat_pin.npz         first edges of the reference rMat generator for three
                       parameter sets (pins the oracle's and the GPU generator)
  s12_updates.npz      scale-12 ef-8 graph: bulk load, then insert/delete
                       batches; per-step sorted adjacency and algorithm outputs
  s12_skew.npz         scale-12 ef-8 a=.57 b=.19 c=.19 plus six star hubs above
                       the reference's 1024 B-tree threshold: same records
  low_degree_tc.npz    a graph whose degrees stay <= 13, where the reference TC
                       runs only its in-place intersection and is exact
  config1_summary.json RMAT scale 17 ef 8 seed 0 (the static workload):
                       hashes and samples of every output
  adj_pin.npz          AdjacencyGraph texts and the reference reader's
                       (n, edges) for each (python tests/golden/make_golden.py
                       --adj-only regenerates only this one)
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def csr_sha(off, tgt) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(off, "<u8").tobytes())
    h.update(np.ascontiguousarray(tgt, "<u4").tobytes())
    return h.hexdigest()


def arr_sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def sorted_ref_csr(R: O.RefGraph):
    off, tgt = R.csr()
    out = tgt.copy()
    for v in range(R.n):
        a, b = int(off[v]), int(off[v + 1])
        out[a:b] = np.sort(tgt[a:b])
    return off, out


def ref_outputs(R: O.RefGraph, src: int, pr_iters=(5, 10)):
    parents = R.bfs(src)
    rec = {
        "bfs_src": np.uint32(src),
        "bfs_levels": O.levels_from_parents(parents, src),
        "bfs_parents": parents,
        "cc": R.cc(),
        "bc": R.bc(src),
        "ref_tc": np.uint64(R.tc()),
    }
    for it in pr_iters:
        rec[f"pr{it}"] = R.pagerank(it)
    return rec


def fresh_ref(n, keys):
    R = O.RefGraph(n)
    R.add_keys(keys, 0)
    return R


def rmat_batches(n, a, b, c, sizes, stream):
    return [O.rmat(n, O.batch_seed(stream, j), a, b, c, size) for j, size in enumerate(sizes)]


def hub_graph_and_batches():
    """RMAT scale 12 ef 8 (a=.57 b=.19 c=.19) plus six seeded star hubs of
    degree 1100..2500, above the reference's 1024 B-tree threshold
    (include/graph.h:39); batches mix RMAT edges with hub edges."""
    n = 1 << 12
    rng = np.random.default_rng(12)
    s, d = O.rmat(n, 0, .57, .19, .19, 8 * n)
    hubs = [1, 100, 2000, 3000, 4000, 4095]
    hs, hd = [s], [d]
    for h in hubs:
        nb = rng.choice(n, int(rng.integers(1100, 2500)), replace=False).astype(np.uint32)
        hs.append(np.full(len(nb), h, np.uint32))
        hd.append(nb)
    keys = O.make_keys(np.concatenate(hs), np.concatenate(hd), True, True)
    batches = []
    for j, size in enumerate([100, 5000]):
        bs, bd = O.rmat(n, O.batch_seed(1, j), .57, .19, .19, size)
        xs = rng.choice(hubs, size // 2).astype(np.uint32)
        xd = rng.integers(0, n, size // 2).astype(np.uint32)
        batches.append((np.concatenate([bs, xs]), np.concatenate([bd, xd])))
    return n, keys, batches


def run_sequence(name, n, keys, batches, params):
    """Bulk load, then insert and delete each batch.  The update sequence runs
    on a reference Graph with one extra, never-touched vertex n: the
    reference's PMA mishandles its LAST vertex (its list can come back out of
    order and binary-search removes then fail: 8 failed removes on vertex
    4095 in this sequence without the padding).  Algorithm outputs come from
    fresh n-vertex reference graphs bulk-loaded with the same edge set."""
    R = O.RefGraph(n + 1)
    R.add_keys(keys, 0)
    cur = keys
    rec = {"n": np.uint32(n), "params": np.array(params, np.float64)}

    def snap(step):
        off, tgt = sorted_ref_csr(R)
        assert off[n] == off[n + 1]  # the padding vertex stays empty
        rec[f"s{step}_off"], rec[f"s{step}_tgt"] = off[:n + 1].copy(), tgt
        return off[:n + 1], tgt

    off, tgt = snap(0)
    deg = np.diff(off.astype(np.int64))
    F = fresh_ref(n, cur)
    for k, v in ref_outputs(F, int(deg.argmax())).items():
        rec["s0_" + k] = v
    F.close()
    step = 1
    for j, (bs, bd) in enumerate(batches):
        rec[f"batch{j}_src"], rec[f"batch{j}_dst"] = bs, bd
        bk = O.make_keys(bs, bd, symmetrize=True, drop_self=True)
        R.add_keys(O.key_difference(bk, cur), perm_seed=j + 1)
        cur = O.key_union(cur, bk)
        snap(step)
        step += 1
        gone = O.key_intersection(bk, cur)
        fails = R.remove_keys(gone)
        assert fails == 0, (name, j, fails)
        cur = O.key_difference(cur, gone)
        off, tgt = snap(step)
        step += 1
    deg = np.diff(off.astype(np.int64))
    F = fresh_ref(n, cur)
    for k, v in ref_outputs(F, int(deg.argmax())).items():
        rec["final_" + k] = v
    F.close()
    rec["steps"] = np.uint32(step)
    np.savez_compressed(os.path.join(OUT, name), **rec)
    print(name, "n", n, "m0", len(keys), "steps", step, "maxdeg", int(deg.max()))


def adj_texts():
    """AdjacencyGraph texts for the reader pins: mixed white space (tabs,
    carriage returns, runs of blanks, a NUL), empty lists, a last vertex with
    edges, a directed graph, and a seeded RMAT graph one number per line."""
    yield (b"AdjacencyGraph\n5\n7\n0\n2\n2\n5\n6\n1\n4\n0\n3\n4\n0\n1\n")
    yield (b"  AdjacencyGraph\r\n4 \t 5\r\n0  1\t1 3\r\n\r\n3 0 2\x00 1\t\t0 ")
    yield b"AdjacencyGraph 3 0 0 0 0"
    n, keys = O.rmat_graph_keys(10, 4, .57, .19, .19, 3)
    off, tgt = O.csr_from_keys(n, keys)
    yield O.format_adj(off, tgt)


def adj_pin():
    """adj_pin.npz: each text and the reference reader's (n, src, dst)."""
    rec = {}
    path = os.path.join(OUT, "_adj_tmp.adj")
    for i, text in enumerate(adj_texts()):
        with open(path, "wb") as f:
            f.write(text)
        n, src, dst = O.ref_read_adj(path)
        rec[f"t{i}_text"] = np.frombuffer(text, np.uint8)
        rec[f"t{i}_n"] = np.uint32(n)
        rec[f"t{i}_src"], rec[f"t{i}_dst"] = src, dst
        print("adj text", i, "n", n, "m", len(src))
    os.remove(path)
    np.savez_compressed(os.path.join(OUT, "adj_pin.npz"), **rec)


def main():
    if not O.ref_available():
        raise SystemExit("build oracle/_ref first: oracle/build_ref.sh")
    O.ref_lib().ref_set_threads(1)
    adj_pin()
    if "--adj-only" in sys.argv:
        return

    pins = {}
    for i, (n, seed, a, b, c) in enumerate([(1 << 17, 0, .5, .1, .1),
                                           (1 << 24, 0, .57, .19, .19),
                                           (1 << 22, 0x9E3779B9, .5, .1, .1)]):
        s, d = O.ref_rmat(n, seed, a, b, c, 4096, first=1000)
        pins[f"p{i}_params"] = np.array([n, seed, a, b, c], np.float64)
        pins[f"p{i}_src"], pins[f"p{i}_dst"] = s, d
    np.savez_compressed(os.path.join(OUT, "rmat_pin.npz"), **pins)
    print("rmat_pin.npz")

    n, keys = O.rmat_graph_keys(12, 8, .5, .1, .1, 0)
    run_sequence("s12_updates.npz", n, keys, rmat_batches(n, .5, .1, .1, [10, 1000, 20000], 1),
                 [12, 8, .5, .1, .1, 0])
    n, keys, batches = hub_graph_and_batches()
    run_sequence("s12_skew.npz", n, keys, batches, [12, 8, .57, .19, .19, 0])

    # Low-degree graph: 600 disjoint 6-cliques (degree 5) plus a seeded
    # random matching; every degree stays <= 13, so the reference TC runs
    # only its in-place intersection (include/graph.h:900-921) and is exact.
    n = 1 << 12
    rng = np.random.default_rng(7)
    perm = rng.permutation(n).astype(np.uint32)
    ss, dd = [], []
    for q in range(600):
        grp = perm[6 * q:6 * q + 6]
        for x in range(6):
            for y in range(x + 1, 6):
                ss.append(grp[x]); dd.append(grp[y])
    m2 = rng.permutation(n).astype(np.uint32)
    ss += list(m2[0::2]); dd += list(m2[1::2])
    keys = O.make_keys(np.array(ss, np.uint32), np.array(dd, np.uint32), True, True)
    R = O.RefGraph(n)
    R.add_keys(keys, 0)
    off, tgt = sorted_ref_csr(R)
    assert np.diff(off.astype(np.int64)).max() <= 13
    np.savez_compressed(os.path.join(OUT, "low_degree_tc.npz"), n=np.uint32(n), keys=keys,
                        ref_tc=np.uint64(R.tc()))
    print("low_degree_tc.npz ref_tc", R.tc())

    # Static workload summary (RMAT scale 17, ef 8, seed 0).
    n, keys = O.rmat_graph_keys(17, 8, .5, .1, .1, 0)
    R = O.RefGraph(n)
    R.add_keys(keys, 0)
    off, tgt = sorted_ref_csr(R)
    deg = np.diff(off.astype(np.int64))
    rng = np.random.default_rng(0)
    sample = np.sort(rng.choice(n, 256, replace=False)).astype(np.int64)
    summ = {"n": n, "m": int(len(keys)), "max_degree": int(deg.max()),
            "argmax_degree": int(deg.argmax()), "isolated": int((deg == 0).sum()),
            "csr_sha256": csr_sha(off, tgt), "sample": sample.tolist(),
            "tc_exact_rmat17": 758730}
    for src in (9, int(deg.argmax())):
        p = R.bfs(src)
        lv = O.levels_from_parents(p, src)
        summ[f"bfs{src}_levels_sha256"] = arr_sha(lv.astype("<u4"))
        summ[f"bfs{src}_reached"] = int((lv != O.UNREACHED).sum())
        summ[f"bfs{src}_max_level"] = int(lv[lv != O.UNREACHED].max())
    pr = R.pagerank(5)
    summ["pr5_sum"] = float(np.sum(pr))
    summ["pr5_sample"] = pr[sample].tolist()
    cc = R.cc()
    summ["cc_sha256"] = arr_sha(cc.astype("<u4"))
    summ["cc_components"] = int(len(np.unique(cc)))
    bcv = R.bc(int(deg.argmax()))
    fin = np.isfinite(bcv)
    summ["bc_src"] = int(deg.argmax())
    summ["bc_finite"] = int(fin.sum())
    summ["bc_sum_finite"] = float(np.sum(bcv[fin]))
    summ["bc_sample"] = [None if not np.isfinite(x) else float(x) for x in bcv[sample]]
    summ["ref_tc_layout_dependent"] = int(R.tc())
    with open(os.path.join(OUT, "config1_summary.json"), "w") as f:
        json.dump(summ, f, indent=1)
    print("config1_summary.json", {k: v for k, v in summ.items() if "sample" not in k})


if __name__ == "__main__":
    main()
