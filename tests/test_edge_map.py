"""The public C++ surface: the facade header (include/terrace_b200.hpp) and
the generic edgeMap / vertexMap layer (include/terrace_b200_edge_map.cuh).

CPU: both compile (g++ for the facade driver, nvcc for sm_100a device
functors) and link against libterrace_b200.so.
GPU: the reference's BFS, CC and PageRank written with the reference's
functors on the generic layer agree with trc_bfs / trc_cc / trc_pagerank and
with the oracle; the facade driver's numbers agree with the oracle."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TESTS = os.path.join(ROOT, "tests")
BUILD = os.path.join(TESTS, "_build")
INC = os.path.join(ROOT, "include")
LIBDIR = os.path.join(ROOT, "terrace_b200")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def _lib_built():
    from terrace_b200 import build
    build.build()


def build_edge_map_lib():
    _lib_built()
    os.makedirs(BUILD, exist_ok=True)
    out = os.path.join(BUILD, "libedge_map_check.so")
    src = os.path.join(TESTS, "edge_map_check.cu")
    hdr = os.path.join(INC, "terrace_b200_edge_map.cuh")
    if not os.path.exists(out) or os.path.getmtime(out) < max(os.path.getmtime(src),
                                                               os.path.getmtime(hdr)):
        subprocess.check_call([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O2",
                               "-std=c++17", "-shared", "-Xcompiler", "-fPIC", "-I" + INC, src,
                               "-L" + LIBDIR, "-lterrace_b200", "-Xlinker", "-rpath=" + LIBDIR,
                               "-o", out])
    return out


def build_facade_exe():
    _lib_built()
    os.makedirs(BUILD, exist_ok=True)
    out = os.path.join(BUILD, "cxx_facade_check")
    src = os.path.join(TESTS, "cxx_facade_check.cc")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-Wall", "-I" + INC, src, "-L" + LIBDIR,
                           "-lterrace_b200", "-Wl,-rpath," + LIBDIR, "-o", out])
    return out


def test_public_headers_compile():
    assert os.path.exists(build_edge_map_lib())
    assert os.path.exists(build_facade_exe())


@pytest.mark.gpu
def test_generic_edge_map_matches_builtin():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    import terrace_b200 as T
    E = C.CDLL(build_edge_map_lib())
    for f in (E.em_bfs, E.em_cc, E.em_pagerank):
        f.restype = C.c_int
    n = 1 << 14
    s, d = T.rmat_generate(n, 4, .57, .19, .19, 16 * n)
    g = T.Graph(n, hub_threshold=200)
    g.add_edge_batch(s, d, symmetrize=True, drop_self_loops=True)
    off, tgt = g.dump_csr()
    src = int(np.diff(off.astype(np.int64)).argmax())
    par = np.empty(n, np.int32)
    lv = np.empty(n, np.uint32)
    assert E.em_bfs(g._h, src, par.ctypes.data_as(C.c_void_p), lv.ctypes.data_as(C.c_void_p)) == 0
    _, blv = g.bfs(src)
    assert np.array_equal(lv, blv)
    assert np.array_equal(lv, O.bfs_levels(off, tgt, src))
    assert O.bfs_check_parents(off, tgt, src, lv, par) == 0
    lab = np.empty(n, np.uint32)
    assert E.em_cc(g._h, lab.ctypes.data_as(C.c_void_p)) == 0
    assert np.array_equal(lab, g.cc())
    pr = np.empty(n, np.float64)
    assert E.em_pagerank(g._h, 5, pr.ctypes.data_as(C.c_void_p)) == 0
    want = O.pagerank(off, tgt, 5)
    # the dense "all" edgeMap sums each list sequentially in sorted order,
    # as the reference and the oracle do: bit-exact here
    assert np.array_equal(pr, want)
    assert np.allclose(g.pagerank(5), want, rtol=1e-9, atol=0)


@pytest.mark.gpu
def test_cxx_facade_driver():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    exe = build_facade_exe()
    out = subprocess.check_output([exe], text=True).split()
    n, m, best, reached, prsum, comps, tri, nb, dup, ise = out
    n = int(n)
    s, d = O.rmat(n, 0, .5, .1, .1, 8 * n)
    keys = O.make_keys(s, d, True, True)
    off, tgt = O.csr_from_keys(n, keys)
    deg = np.diff(off.astype(np.int64))
    assert int(m) == len(keys)
    assert int(best) == int(deg.argmax())
    lv = O.bfs_levels(off, tgt, int(best))
    assert int(reached) == int((lv != O.UNREACHED).sum())
    assert abs(float(prsum) - O.pagerank(off, tgt, 5).sum()) <= 1e-9 * float(prsum)
    assert int(comps) == len(np.unique(O.cc(off, tgt)))
    assert int(tri) == O.tc(off, tgt)
    assert int(nb) == deg[int(best)]
    assert int(dup) == -1 and int(ise) == 1
