"""CPU oracle for the Terrace hot path -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this package; the product (``terrace_b200``) never does.

Two checkers live here:

* ``liboracle.so`` -- oracle/oracle.c, a C restatement of the reference's
  algorithms over sorted neighbour lists (each function cites the reference
  file:line it follows);
* ``_ref/libterrace_ref.so`` -- the UNMODIFIED reference Terrace compiled from
  its own sources by oracle/build_ref.sh, driven through oracle/ref_driver.cc.
  It is optional at run time (``ref_available()``).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_ORACLE_SO = os.path.join(_HERE, "liboracle.so")
_REF_SO = os.path.join(_HERE, "_ref", "libterrace_ref.so")

UNREACHED = 0xFFFFFFFF

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def build_oracle(force: bool = False) -> str:
    """Compile oracle/oracle.c into oracle/liboracle.so (gcc)."""
    src = os.path.join(_HERE, "oracle.c")
    if force or not os.path.exists(_ORACLE_SO) or os.path.getmtime(src) > os.path.getmtime(_ORACLE_SO):
        subprocess.check_call(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", src,
                               "-o", _ORACLE_SO, "-lm"])
    return _ORACLE_SO


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_ORACLE_SO):
            build_oracle()
        L = C.CDLL(_ORACLE_SO)
        L.orc_hash32.restype = C.c_uint32
        L.orc_hash32.argtypes = [C.c_uint32]
        L.orc_hash64.restype = C.c_uint64
        L.orc_hash64.argtypes = [C.c_uint64]
        L.orc_rmat.restype = None
        L.orc_rmat.argtypes = [C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_double,
                               C.c_uint64, C.c_uint64, _u32p, _u32p]
        L.orc_make_keys.restype = C.c_uint64
        L.orc_make_keys.argtypes = [_u32p, _u32p, C.c_uint64, C.c_int, C.c_int, _u64p]
        for name in ("orc_key_union", "orc_key_difference", "orc_key_intersection"):
            f = getattr(L, name)
            f.restype = C.c_uint64
            f.argtypes = [_u64p, C.c_uint64, _u64p, C.c_uint64, _u64p]
        L.orc_csr_from_keys.restype = None
        L.orc_csr_from_keys.argtypes = [C.c_uint32, _u64p, C.c_uint64, _u64p, _u32p]
        L.orc_bfs_levels.restype = None
        L.orc_bfs_levels.argtypes = [C.c_uint32, _u64p, _u32p, C.c_uint32, _u32p]
        L.orc_bfs_check_parents.restype = C.c_uint64
        L.orc_bfs_check_parents.argtypes = [C.c_uint32, _u64p, _u32p, C.c_uint32, _u32p, _i32p]
        L.orc_pagerank.restype = None
        L.orc_pagerank.argtypes = [C.c_uint32, _u64p, _u32p, C.c_uint32, C.c_double, _f64p]
        L.orc_cc.restype = None
        L.orc_cc.argtypes = [C.c_uint32, _u64p, _u32p, _u32p]
        L.orc_bc.restype = None
        L.orc_bc.argtypes = [C.c_uint32, _u64p, _u32p, C.c_uint32, _f64p]
        L.orc_tc.restype = C.c_uint64
        L.orc_tc.argtypes = [C.c_uint32, _u64p, _u32p]
        L.orc_tc_touching.restype = C.c_uint64
        L.orc_tc_touching.argtypes = [C.c_uint32, _u64p, _u32p, _u64p, C.c_uint64]
        _lib = L
    return _lib


# ---------------------------------------------------------------- generators

def hash32(x: int) -> int:
    return int(lib().orc_hash32(x & 0xFFFFFFFF))


def hash64(x: int) -> int:
    return int(lib().orc_hash64(x & 0xFFFFFFFFFFFFFFFF))


def rmat(n: int, seed: int, a: float, b: float, c: float, count: int, first: int = 0):
    """Edges first..first+count-1 of rMat<uint32_t>(n, seed, a, b, c)
    (include/rmat_util.h:81-115)."""
    src = np.empty(count, np.uint32)
    dst = np.empty(count, np.uint32)
    lib().orc_rmat(n, seed & 0xFFFFFFFF, a, b, c, first, count, src, dst)
    return src, dst


def make_keys(src, dst, symmetrize: bool = True, drop_self: bool = True) -> np.ndarray:
    src = np.ascontiguousarray(src, np.uint32)
    dst = np.ascontiguousarray(dst, np.uint32)
    out = np.empty(max(1, 2 * len(src)), np.uint64)
    m = lib().orc_make_keys(src, dst, len(src), int(symmetrize), int(drop_self), out)
    return out[:m].copy()


def _setop(fn, A, B):
    A = np.ascontiguousarray(A, np.uint64)
    B = np.ascontiguousarray(B, np.uint64)
    out = np.empty(max(1, len(A) + len(B)), np.uint64)
    m = fn(A if len(A) else np.zeros(1, np.uint64), len(A),
           B if len(B) else np.zeros(1, np.uint64), len(B), out)
    return out[:m].copy()


def key_union(A, B):
    return _setop(lib().orc_key_union, A, B)


def key_difference(A, B):
    return _setop(lib().orc_key_difference, A, B)


def key_intersection(A, B):
    return _setop(lib().orc_key_intersection, A, B)


def keys_to_pairs(keys):
    keys = np.asarray(keys, np.uint64)
    return (keys >> np.uint64(32)).astype(np.uint32), (keys & np.uint64(0xFFFFFFFF)).astype(np.uint32)


def csr_from_keys(n: int, keys):
    keys = np.ascontiguousarray(keys, np.uint64)
    off = np.empty(n + 1, np.uint64)
    tgt = np.empty(max(1, len(keys)), np.uint32)
    lib().orc_csr_from_keys(n, keys if len(keys) else np.zeros(1, np.uint64), len(keys), off, tgt)
    return off, tgt[:len(keys)]


def rmat_graph_keys(scale: int, edge_factor: int, a: float, b: float, c: float, seed: int):
    """Workload graph: ef*n RMAT edges (reference generator), self-loops
    dropped, symmetrized and deduplicated."""
    n = 1 << scale
    src, dst = rmat(n, seed, a, b, c, edge_factor * n)
    return n, make_keys(src, dst, symmetrize=True, drop_self=True)


def batch_seed(seed: int, j: int) -> int:
    """Seed of update batch j drawn from stream `seed`: hash32(seed) ^ j."""
    return hash32(seed) ^ (j & 0xFFFFFFFF)


# ---------------------------------------------------------------- algorithms

def _csr(off, tgt):
    off = np.ascontiguousarray(off, np.uint64)
    tgt = np.ascontiguousarray(tgt, np.uint32)
    if len(tgt) == 0:
        tgt = np.zeros(1, np.uint32)
    return off, tgt


def bfs_levels(off, tgt, src: int):
    n = len(off) - 1
    off, tgt = _csr(off, tgt)
    lv = np.empty(n, np.uint32)
    lib().orc_bfs_levels(n, off, tgt, src, lv)
    return lv


def bfs_check_parents(off, tgt, src: int, levels, parents) -> int:
    n = len(off) - 1
    off, tgt = _csr(off, tgt)
    return int(lib().orc_bfs_check_parents(n, off, tgt, src,
                                           np.ascontiguousarray(levels, np.uint32),
                                           np.ascontiguousarray(parents, np.int32)))


def pagerank(off, tgt, iters: int, damping: float = 0.0):
    n = len(off) - 1
    off, tgt = _csr(off, tgt)
    out = np.empty(n, np.float64)
    lib().orc_pagerank(n, off, tgt, iters, damping, out)
    return out


def cc(off, tgt):
    n = len(off) - 1
    off, tgt = _csr(off, tgt)
    out = np.empty(n, np.uint32)
    lib().orc_cc(n, off, tgt, out)
    return out


def bc(off, tgt, src: int):
    n = len(off) - 1
    off, tgt = _csr(off, tgt)
    out = np.empty(n, np.float64)
    lib().orc_bc(n, off, tgt, src, out)
    return out


def tc(off, tgt) -> int:
    n = len(off) - 1
    off, tgt = _csr(off, tgt)
    return int(lib().orc_tc(n, off, tgt))


def tc_touching(off, tgt, bkeys) -> int:
    """Triangles of the graph that contain at least one edge of bkeys (sorted
    unique directed keys, both directions of every edge): the change of the
    triangle count when those edges are added to (or removed from) it."""
    n = len(off) - 1
    off, tgt = _csr(off, tgt)
    bk = np.ascontiguousarray(bkeys, np.uint64)
    if len(bk) == 0:
        return 0
    return int(lib().orc_tc_touching(n, off, tgt, bk, len(bk)))


def csr_keys(off, tgt):
    """Sorted directed keys (src<<32|dst) of a CSR."""
    off = np.asarray(off, np.uint64)
    n = len(off) - 1
    src = np.repeat(np.arange(n, dtype=np.uint64), np.diff(off.astype(np.int64)))
    return (src << np.uint64(32)) | np.asarray(tgt, np.uint64)


# ------------------------------------------------------- reference library

_ref = None


def ref_available() -> bool:
    return os.path.exists(_REF_SO)


def ref_lib():
    global _ref
    if _ref is None:
        if not ref_available():
            raise RuntimeError("oracle/_ref/libterrace_ref.so is not built (oracle/build_ref.sh)")
        L = C.CDLL(_REF_SO)
        vp = C.c_void_p
        L.ref_set_threads.argtypes = [C.c_int]
        L.ref_set_threads.restype = None
        L.ref_get_threads.restype = C.c_int
        L.ref_graph_new.restype = vp
        L.ref_graph_new.argtypes = [C.c_uint32]
        L.ref_graph_free.argtypes = [vp]
        L.ref_graph_free.restype = None
        L.ref_add_edge_batch.argtypes = [vp, _u32p, _u32p, C.c_uint32, C.c_uint32]
        L.ref_add_edge_batch.restype = None
        L.ref_remove_edges.argtypes = [vp, _u32p, _u32p, C.c_uint32]
        L.ref_remove_edges.restype = C.c_int64
        L.ref_degree.argtypes = [vp, C.c_uint32]
        L.ref_degree.restype = C.c_uint32
        L.ref_is_edge.argtypes = [vp, C.c_uint32, C.c_uint32]
        L.ref_is_edge.restype = C.c_uint32
        L.ref_num_edges.argtypes = [vp]
        L.ref_num_edges.restype = C.c_uint64
        L.ref_dump_csr.argtypes = [vp, _u64p, _u32p]
        L.ref_dump_csr.restype = None
        L.ref_bfs.argtypes = [vp, C.c_uint32, _i32p]
        L.ref_bfs.restype = None
        L.ref_pagerank.argtypes = [vp, C.c_uint32, _f64p]
        L.ref_pagerank.restype = None
        L.ref_cc.argtypes = [vp, _u32p]
        L.ref_cc.restype = None
        L.ref_bc.argtypes = [vp, C.c_uint32, _f64p]
        L.ref_bc.restype = None
        L.ref_tc.argtypes = [vp]
        L.ref_tc.restype = C.c_uint64
        L.ref_rmat.argtypes = [C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_double,
                               C.c_uint64, C.c_uint64, _u32p, _u32p]
        L.ref_rmat.restype = None
        L.ref_read_adj.argtypes = [C.c_char_p, C.POINTER(C.c_uint32), _u32p, _u32p, C.c_uint64]
        L.ref_read_adj.restype = C.c_uint64
        _ref = L
    return _ref


def ref_rmat(n: int, seed: int, a: float, b: float, c: float, count: int, first: int = 0):
    """The reference's own rMat<uint32_t> generator (pins ``rmat``)."""
    src = np.empty(count, np.uint32)
    dst = np.empty(count, np.uint32)
    ref_lib().ref_rmat(n, seed & 0xFFFFFFFF, a, b, c, first, count, src, dst)
    return src, dst


def ref_read_adj(path: str):
    """The reference's AdjacencyGraph reader on a well-formed file:
    (n, src, dst) in file order."""
    n = C.c_uint32()
    probe = np.empty(1, np.uint32)
    m = ref_lib().ref_read_adj(path.encode(), C.byref(n), probe, probe, 0)
    src = np.empty(max(m, 1), np.uint32)
    dst = np.empty(max(m, 1), np.uint32)
    ref_lib().ref_read_adj(path.encode(), C.byref(n), src, dst, m)
    return int(n.value), src[:m], dst[:m]


# --------------------------------------------------------------------------
# AdjacencyGraph text (include/io_util.h:112-145): words separated by space,
# tab, newline, carriage return or NUL (isSpace, include/io_util.h:27-36);
# "AdjacencyGraph", n, m, n offsets, m targets; vertex i's edges are
# targets [off[i], off[i+1]), the last vertex's ending at m.

_ADJ_SPACE = b" \t\n\r\0"


def parse_adj(data: bytes):
    """(n, src, dst) of an AdjacencyGraph text, edges in file order; raises
    ValueError where the reference would stop (missing header, word count
    other than n + m + 2) and on words that are not decimal numbers or
    offsets that do not rise from 0 (the reference's atol accepts those
    silently)."""
    import re
    words = re.split(b"[ \t\n\r\x00]+", data.strip(_ADJ_SPACE))
    if not words or words[0] != b"AdjacencyGraph":
        raise ValueError("missing header AdjacencyGraph")
    nums = words[1:]
    if any(not w.isdigit() for w in nums):
        raise ValueError("a word is not a number")
    vals = np.array([int(w) for w in nums], dtype=np.uint64)
    if len(vals) < 2:
        raise ValueError("missing n and m")
    n, m = int(vals[0]), int(vals[1])
    if len(vals) != n + m + 2:
        raise ValueError("length != n + m + 2")
    off = vals[2:2 + n]
    if n and (off[0] != 0 or np.any(np.diff(off.astype(np.int64)) < 0) or np.any(off > m)):
        raise ValueError("offsets not monotone from 0")
    ends = np.append(off[1:], np.uint64(m)) if n else off
    src = np.repeat(np.arange(n, dtype=np.uint32), (ends - off).astype(np.int64))
    dst = vals[2 + n:].astype(np.uint32)
    return n, src, dst


def format_adj(off, tgt) -> bytes:
    """AdjacencyGraph text of a CSR: one number per line after the header."""
    n = len(off) - 1
    nums = [n, int(off[n])] + [int(x) for x in off[:n]] + [int(x) for x in tgt]
    return b"AdjacencyGraph\n" + b"".join(b"%d\n" % x for x in nums)


class RefGraph:
    """The unmodified reference graphstore::Graph, through ref_driver.cc."""

    def __init__(self, n: int):
        self.n = n
        self.L = ref_lib()
        self.h = self.L.ref_graph_new(n)

    def close(self):
        if self.h:
            self.L.ref_graph_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_keys(self, keys, perm_seed: int = 0):
        """keys: sorted unique uint64 (src<<32|dst), none already present."""
        s, d = keys_to_pairs(keys)
        if len(s):
            self.L.ref_add_edge_batch(self.h, s, d, len(s), perm_seed)

    def remove_keys(self, keys) -> int:
        """keys: existing edges only.  Returns the number of failed removes."""
        s, d = keys_to_pairs(keys)
        if not len(s):
            return 0
        return int(self.L.ref_remove_edges(self.h, s, d, len(s)))

    def num_edges(self) -> int:
        return int(self.L.ref_num_edges(self.h))

    def degree(self, v: int) -> int:
        return int(self.L.ref_degree(self.h, v))

    def csr(self):
        off = np.empty(self.n + 1, np.uint64)
        m = self.num_edges()
        tgt = np.empty(max(1, m), np.uint32)
        self.L.ref_dump_csr(self.h, off, tgt)
        return off, tgt[:m]

    def bfs(self, src: int):
        p = np.empty(self.n, np.int32)
        self.L.ref_bfs(self.h, src, p)
        return p

    def pagerank(self, iters: int):
        out = np.empty(self.n, np.float64)
        self.L.ref_pagerank(self.h, iters, out)
        return out

    def cc(self):
        out = np.empty(self.n, np.uint32)
        self.L.ref_cc(self.h, out)
        return out

    def bc(self, src: int):
        out = np.empty(self.n, np.float64)
        self.L.ref_bc(self.h, src, out)
        return out

    def tc(self) -> int:
        return int(self.L.ref_tc(self.h))


def levels_from_parents(parents, src: int):
    """Depth of every vertex by walking parent pointers (the reference's
    VERIFY dump, include/BFS.h:60-82); UNREACHED where parent is -1."""
    parents = np.asarray(parents, np.int64)
    n = len(parents)
    lv = np.full(n, UNREACHED, np.uint64)
    lv[src] = 0
    reached = parents >= 0
    # iterate pointer jumping: depth via repeated squaring of the parent map
    depth = np.where(reached, 1, 0).astype(np.int64)
    depth[src] = 0
    par = np.where(reached, parents, np.arange(n))
    for _ in range(64):
        nxt = par[par]
        add = depth[par]
        if np.array_equal(nxt, par):
            break
        depth = depth + add
        par = nxt
    lv = np.where(reached, depth, UNREACHED).astype(np.uint64)
    return lv.astype(np.uint32)
