"""Graph files: the reference's AdjacencyGraph text (include/io_util.h:
112-145), parsed and written on the GPU, and the binary CSR file.

Every pinned text (tests/golden/adj_pin.npz, with the reference reader's
output) loads to exactly the reference's edge set; a saved graph's text is
byte-identical to the oracle's formatter and loads back to the same CSR;
malformed files fail with TRC_ERR_INVALID and missing ones with TRC_ERR_IO,
leaving no graph behind."""
import os

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def T():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    import terrace_b200 as T
    return T


def _csr(n, s, d, sym=False):
    return O.csr_from_keys(n, O.make_keys(s, d, sym, False))


def test_load_pinned_adj_texts(T, tmp_path):
    z = np.load(os.path.join(GOLD, "adj_pin.npz"))
    i = 0
    while f"t{i}_text" in z:
        p = tmp_path / f"t{i}.adj"
        p.write_bytes(z[f"t{i}_text"].tobytes())
        n = int(z[f"t{i}_n"])
        g = T.Graph.load_adj(p, hub_threshold=64)
        assert g.n == n
        off, tgt = _csr(n, z[f"t{i}_src"], z[f"t{i}_dst"])
        goff, gtgt = g.dump_csr()
        assert np.array_equal(goff, off) and np.array_equal(gtgt, tgt), i
        g.close()
        gs = T.Graph.load_adj(p, symmetrize=True)
        off, tgt = _csr(n, z[f"t{i}_src"], z[f"t{i}_dst"], sym=True)
        goff, gtgt = gs.dump_csr()
        assert np.array_equal(goff, off) and np.array_equal(gtgt, tgt), i
        gs.close()
        i += 1


def test_save_and_reload_adj_and_csr(T, tmp_path):
    n = 1 << 13
    s, d = T.rmat_generate(n, 21, .57, .19, .19, 8 * n)
    g = T.Graph(n, hub_threshold=64)
    g.add_edge_batch(s, d, symmetrize=True, drop_self_loops=True)
    off, tgt = g.dump_csr()
    pa = tmp_path / "g.adj"
    g.save_adj(pa)
    assert pa.read_bytes() == O.format_adj(off, tgt)
    g2 = T.Graph.load_adj(pa, hub_threshold=64)
    o2, t2 = g2.dump_csr()
    assert np.array_equal(o2, off) and np.array_equal(t2, tgt)
    assert g2.check() == 0
    pc = tmp_path / "g.csr"
    g.save_csr(pc)
    assert pc.stat().st_size == 24 + 8 * (n + 1) + 4 * len(tgt)
    g3 = T.Graph.load_csr(pc)
    o3, t3 = g3.dump_csr()
    assert np.array_equal(o3, off) and np.array_equal(t3, tgt)
    # the loaded graph is a normal graph: analytics agree with the original
    src = int(np.diff(off.astype(np.int64)).argmax())
    assert np.array_equal(g3.bfs(src)[1], g.bfs(src)[1])
    for x in (g, g2, g3):
        x.close()


@pytest.mark.parametrize("text", [
    b"AdjGraph\n2\n1\n0\n1\n1\n",             # header
    b"AdjacencyGraph\n2\n1\n0\n1\n",          # n + m + 2 numbers expected
    b"AdjacencyGraph\n2\n1\n0\n1\n1\n7\n",    # one too many
    b"AdjacencyGraph\n2\n1\n0\n1\n1x\n",      # not a number
    b"AdjacencyGraph\n2\n1\n1\n0\n1\n",       # offsets do not start at 0
    b"AdjacencyGraph\n3\n1\n0\n1\n0\n1\n",    # offsets fall
    b"AdjacencyGraph\n2\n1\n0\n1\n2\n",       # target >= n
    b"AdjacencyGraph\n0\n0\n",                # no vertices
])
def test_malformed_adj_rejected(T, tmp_path, text):
    from terrace_b200 import _lib
    p = tmp_path / "bad.adj"
    p.write_bytes(text)
    with pytest.raises(_lib.TrcError) as e:
        T.Graph.load_adj(p)
    assert e.value.status == _lib.TRC_ERR_INVALID


def test_file_errors(T, tmp_path):
    from terrace_b200 import _lib
    with pytest.raises(_lib.TrcError) as e:
        T.Graph.load_adj(tmp_path / "missing.adj")
    assert e.value.status == _lib.TRC_ERR_IO
    p = tmp_path / "bad.csr"
    p.write_bytes(b"NOTACSR0" + bytes(16))
    with pytest.raises(_lib.TrcError) as e:
        T.Graph.load_csr(p)
    assert e.value.status == _lib.TRC_ERR_INVALID
    g = T.Graph(64)
    g.add_edge_batch([1, 2], [2, 3], symmetrize=True)
    g.save_csr(p)
    data = p.read_bytes()
    p.write_bytes(data[:-4])                      # truncated
    with pytest.raises(_lib.TrcError) as e:
        T.Graph.load_csr(p)
    assert e.value.status == _lib.TRC_ERR_INVALID
    with pytest.raises(_lib.TrcError) as e:
        g.save_adj(tmp_path / "no_such_dir" / "g.adj")
    assert e.value.status == _lib.TRC_ERR_IO
    g.close()
