"""Pin the CPU oracle (oracle/oracle.c) against the golden fixtures recorded
from the unmodified reference Terrace (tests/golden/make_golden.py)."""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# PageRank / BC are FP64 sums; atomics and iteration order in the reference
# may reorder them, so they are compared within this relative tolerance.
REL_TOL = 1e-9


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


def test_rmat_generator_pinned():
    z = load("rmat_pin.npz")
    for i in range(3):
        n, seed, a, b, c = z[f"p{i}_params"]
        s, d = O.rmat(int(n), int(seed), a, b, c, 4096, first=1000)
        assert np.array_equal(s, z[f"p{i}_src"])
        assert np.array_equal(d, z[f"p{i}_dst"])


def replay(z):
    """Set-model replay of a fixture's update sequence; yields (step, keys)."""
    n = int(z["n"])
    off, tgt = z["s0_off"], z["s0_tgt"]
    cur = (np.repeat(np.arange(n, dtype=np.uint64), np.diff(off.astype(np.int64))) << np.uint64(32)) \
        | tgt.astype(np.uint64)
    yield 0, cur
    step = 1
    j = 0
    while f"batch{j}_src" in z.files:
        bk = O.make_keys(z[f"batch{j}_src"], z[f"batch{j}_dst"], True, True)
        cur = O.key_union(cur, bk)
        yield step, cur
        step += 1
        cur = O.key_difference(cur, bk)
        yield step, cur
        step += 1
        j += 1


@pytest.mark.parametrize("name", ["s12_updates.npz", "s12_skew.npz"])
def test_update_sequence_matches_reference(name):
    z = load(name)
    n = int(z["n"])
    steps = 0
    for step, keys in replay(z):
        off, tgt = O.csr_from_keys(n, keys)
        assert np.array_equal(off, z[f"s{step}_off"]), step
        assert np.array_equal(tgt, z[f"s{step}_tgt"]), step
        steps += 1
    assert steps == int(z["steps"])


@pytest.mark.parametrize("name", ["s12_updates.npz", "s12_skew.npz"])
@pytest.mark.parametrize("when", ["s0", "final"])
def test_algorithms_match_reference(name, when):
    z = load(name)
    last = int(z["steps"]) - 1
    idx = 0 if when == "s0" else last
    off, tgt = z[f"s{idx}_off"], z[f"s{idx}_tgt"]
    src = int(z[f"{when}_bfs_src"])
    lv = O.bfs_levels(off, tgt, src)
    assert np.array_equal(lv, z[f"{when}_bfs_levels"])
    assert O.bfs_check_parents(off, tgt, src, lv, z[f"{when}_bfs_parents"]) == 0
    for it in (5, 10):
        assert rel_close(O.pagerank(off, tgt, it), z[f"{when}_pr{it}"])
    assert np.array_equal(O.cc(off, tgt), z[f"{when}_cc"])
    assert rel_close(O.bc(off, tgt, src), z[f"{when}_bc"])


def test_tc_matches_reference_exact_path():
    z = load("low_degree_tc.npz")
    off, tgt = O.csr_from_keys(int(z["n"]), z["keys"])
    assert O.tc(off, tgt) == int(z["ref_tc"]) == 12000


def test_config1_summary():
    with open(os.path.join(GOLD, "config1_summary.json")) as f:
        s = json.load(f)
    n, keys = O.rmat_graph_keys(17, 8, .5, .1, .1, 0)
    assert n == s["n"] and len(keys) == s["m"]
    off, tgt = O.csr_from_keys(n, keys)
    assert csr_sha(off, tgt) == s["csr_sha256"]
    deg = np.diff(off.astype(np.int64))
    assert int(deg.max()) == s["max_degree"] and int((deg == 0).sum()) == s["isolated"]
    for src in (9, s["argmax_degree"]):
        lv = O.bfs_levels(off, tgt, src)
        assert hashlib.sha256(lv.astype("<u4").tobytes()).hexdigest() == s[f"bfs{src}_levels_sha256"]
    sample = np.array(s["sample"])
    pr = O.pagerank(off, tgt, 5)
    assert rel_close(pr[sample], np.array(s["pr5_sample"]))
    assert abs(pr.sum() - s["pr5_sum"]) <= 1e-9 * abs(s["pr5_sum"])
    cc = O.cc(off, tgt)
    assert hashlib.sha256(cc.astype("<u4").tobytes()).hexdigest() == s["cc_sha256"]
    bc = O.bc(off, tgt, s["bc_src"])
    ref = np.array([np.nan if x is None else x for x in s["bc_sample"]])
    assert rel_close(bc[sample], ref)
    assert O.tc(off, tgt) == s["tc_exact_rmat17"] == 758730


def test_adj_reader_pinned_to_reference():
    """The oracle's AdjacencyGraph parser gives exactly the reference
    reader's (n, edges) on every pinned text (mixed white space, empty
    lists, a NUL separator, a one-number-per-line RMAT graph), and the
    oracle's formatter writes text that parses back to the same CSR."""
    z = np.load(os.path.join(GOLD, "adj_pin.npz"))
    i = 0
    while f"t{i}_text" in z:
        n, s, d = O.parse_adj(z[f"t{i}_text"].tobytes())
        assert n == int(z[f"t{i}_n"])
        assert np.array_equal(s, z[f"t{i}_src"]) and np.array_equal(d, z[f"t{i}_dst"])
        i += 1
    assert i >= 4
    n, keys = O.rmat_graph_keys(9, 4, .5, .1, .1, 1)
    off, tgt = O.csr_from_keys(n, keys)
    n2, s2, d2 = O.parse_adj(O.format_adj(off, tgt))
    off2, tgt2 = O.csr_from_keys(n2, O.make_keys(s2, d2, False, False))
    assert n2 == n and np.array_equal(off2, off) and np.array_equal(tgt2, tgt)
    for bad in (b"AdjGraph 1 0 0", b"AdjacencyGraph 2 1 0 1", b"AdjacencyGraph 2 1 0 x 1",
                b"AdjacencyGraph 2 1 1 0 1"):
        with pytest.raises(ValueError):
            O.parse_adj(bad)


def test_tc_touching_equals_recount():
    """The oracle's triangle delta (triangles that hold at least one edge of a
    batch) against full recounts before and after inserting and removing
    batches, on a skewed graph whose batches share edges with it and with
    each other."""
    n = 1 << 11
    rng = np.random.default_rng(4)
    s, d = O.rmat(n, 21, .57, .19, .19, 12 * n)
    keys = O.make_keys(s, d, True, True)
    t0 = O.tc(*O.csr_from_keys(n, keys))
    for j in range(4):
        bs, bd = O.rmat(n, 100 + j, .57, .19, .19, int(rng.integers(1, 4000)))
        bk = O.make_keys(bs, bd, True, True)
        new = O.key_difference(bk, keys)
        g1 = O.key_union(keys, bk)
        t1 = O.tc(*O.csr_from_keys(n, g1))
        assert t1 - t0 == O.tc_touching(*O.csr_from_keys(n, g1), new)
        h = len(bs) // 2
        gone = O.key_intersection(g1, O.make_keys(bs[:h], bd[:h], True, True))
        g2 = O.key_difference(g1, gone)
        t2 = O.tc(*O.csr_from_keys(n, g2))
        assert t1 - t2 == O.tc_touching(*O.csr_from_keys(n, g1), gone)
        keys, t0 = g2, t2
    assert O.tc_touching(*O.csr_from_keys(n, keys), np.zeros(0, np.uint64)) == 0
