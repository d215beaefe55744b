"""Python mirror of the reference Graph API over the C ABI.

Method names follow graphstore::Graph (include/graph.h:73-230) and the
algorithm entry points of the reference (include/BFS.h, Pagerank.h,
Components.h, BC.h, TC.h).  Arrays may be numpy arrays (host) or CUDA torch
tensors (device; passed with TRC_DEVICE_PTR, no copy).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L


def _is_cuda_tensor(x) -> bool:
    return type(x).__module__.startswith("torch") and getattr(x, "is_cuda", False)


def _arr(x, dtype):
    """Returns (pointer, length, device_flag, keepalive)."""
    if _is_cuda_tensor(x):
        import torch
        want = {np.uint32: torch.int32, np.int32: torch.int32, np.uint64: torch.int64,
                np.float64: torch.float64, np.uint8: torch.uint8}[dtype]
        if x.dtype not in (want,) and not (dtype == np.uint32 and x.dtype == torch.int32):
            x = x.to(want)
        x = x.contiguous()
        return x.data_ptr(), x.numel(), L.TRC_DEVICE_PTR, x
    a = np.ascontiguousarray(x, dtype=dtype)
    return a.ctypes.data, a.size, 0, a


def _config(hub_threshold: int = 1024, pma_root_density: float = 0.75,
            pma_build_density: float = 0.375, hub_block_fill: float = 0.75,
            push_pull_divisor: int = 20, hub_stage_limit: int = 49152,
            cuda_graphs: bool = True):
    lib = L.load()
    cfg = L.trc_config()
    lib.trc_config_default(C.byref(cfg))
    cfg.hub_threshold = hub_threshold
    cfg.pma_root_density = pma_root_density
    cfg.pma_build_density = pma_build_density
    cfg.hub_block_fill = hub_block_fill
    cfg.push_pull_divisor = push_pull_divisor
    cfg.hub_stage_limit = hub_stage_limit
    cfg.cuda_graphs = int(cuda_graphs)
    return cfg


class Graph:
    """B200-resident Terrace graph: inline rows, PMA segments, hub blocks."""

    def __init__(self, n: int, hbm_budget: int = 0, *, _handle=None, **config):
        self._L = L.load()
        if _handle is None:
            cfg = _config(**config)
            h = C.c_void_p()
            L.check(self._L.trc_graph_create(n, hbm_budget, C.byref(cfg), C.byref(h)))
            _handle = h
        self._h = _handle
        self.n = n

    @classmethod
    def load_adj(cls, path: str, hbm_budget: int = 0, symmetrize: bool = False,
                 drop_self_loops: bool = False, **config) -> "Graph":
        """A graph from an AdjacencyGraph text file (the reference's input
        format, include/io_util.h:112-145), parsed on the GPU."""
        return cls._load(L.load().trc_graph_load_adj, path, hbm_budget, symmetrize,
                         drop_self_loops, config)

    @classmethod
    def load_csr(cls, path: str, hbm_budget: int = 0, symmetrize: bool = False,
                 drop_self_loops: bool = False, **config) -> "Graph":
        """A graph from a binary CSR file written by save_csr."""
        return cls._load(L.load().trc_graph_load_csr, path, hbm_budget, symmetrize,
                         drop_self_loops, config)

    @classmethod
    def _load(cls, fn, path, hbm_budget, sym, drop, config):
        cfg = _config(**config)
        flags = (L.TRC_SYMMETRIZE if sym else 0) | (L.TRC_DROP_SELF_LOOPS if drop else 0)
        h = C.c_void_p()
        L.check(fn(str(path).encode(), hbm_budget, C.byref(cfg), flags, C.byref(h)))
        n = C.c_uint32()
        L.check(L.load().trc_num_vertices(h, C.byref(n)))
        return cls(int(n.value), _handle=h)

    def save_adj(self, path: str):
        """Writes the graph as an AdjacencyGraph text file (formatted on the GPU)."""
        L.check(self._L.trc_graph_save_adj(self._h, str(path).encode()))

    def save_csr(self, path: str):
        """Writes the graph as a binary CSR file ("TRCCSR01", n, m, offsets, targets)."""
        L.check(self._L.trc_graph_save_csr(self._h, str(path).encode()))

    # ---------------------------------------------------------------- lifetime
    def close(self):
        if getattr(self, "_h", None):
            L.check(self._L.trc_graph_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_stream(self, stream):
        """Bind to a CUDA stream (torch.cuda.Stream, raw handle or None).
        None and handle 0 (torch's default stream) select the graph's own
        stream; bind a non-default stream to order the graph's work with other
        work on it (a batch call returns with its last kernels still queued)."""
        ptr = getattr(stream, "cuda_stream", stream)
        L.check(self._L.trc_graph_set_stream(self._h, C.c_void_p(ptr or 0)))

    def release_scratch(self):
        """Free temporary device buffers kept between calls."""
        L.check(self._L.trc_release_scratch(self._h))

    # ---------------------------------------------------------------- updates
    def add_edge_batch(self, srcs, dests, symmetrize: bool = False,
                       drop_self_loops: bool = False) -> int:
        """Insert edges (set semantics); returns directed edges inserted."""
        return self._batch(self._L.trc_add_edge_batch, srcs, dests, symmetrize, drop_self_loops)

    def remove_edge_batch(self, srcs, dests, symmetrize: bool = False,
                          drop_self_loops: bool = False) -> int:
        """Remove edges (absent ones ignored); returns directed edges removed."""
        return self._batch(self._L.trc_remove_edge_batch, srcs, dests, symmetrize, drop_self_loops)

    def _batch(self, fn, srcs, dests, sym, drop):
        ps, ns, fs, ks = _arr(srcs, np.uint32)
        pd, nd, fd, kd = _arr(dests, np.uint32)
        if ns != nd:
            raise ValueError("srcs and dests differ in length")
        if fs != fd:
            raise ValueError("srcs and dests must both be host or both be device arrays")
        flags = fs | (L.TRC_SYMMETRIZE if sym else 0) | (L.TRC_DROP_SELF_LOOPS if drop else 0)
        out = C.c_uint64()
        L.check(fn(self._h, C.c_void_p(ps), C.c_void_p(pd), ns, flags, C.byref(out)))
        return int(out.value)

    def add_edge(self, s: int, d: int) -> int:
        """Graph::add_edge: 0 if inserted, -1 if it already existed."""
        return 0 if self.add_edge_batch([s], [d]) == 1 else -1

    def remove_edge(self, s: int, d: int) -> int:
        """Graph::remove_edge: 0 if removed, -1 if absent."""
        return 0 if self.remove_edge_batch([s], [d]) == 1 else -1

    # ---------------------------------------------------------------- queries
    def is_edge(self, s, d):
        scalar = np.isscalar(s)
        ps, ns, fs, ks = _arr(np.atleast_1d(s) if scalar else s, np.uint32)
        pd, nd, fd, kd = _arr(np.atleast_1d(d) if scalar else d, np.uint32)
        if fs:
            import torch
            out = torch.empty(ns, dtype=torch.uint8, device=ks.device)
            optr = out.data_ptr()
        else:
            out = np.empty(ns, np.uint8)
            optr = out.ctypes.data
        L.check(self._L.trc_is_edge(self._h, C.c_void_p(ps), C.c_void_p(pd), ns, C.c_void_p(optr), fs))
        return int(out[0]) if scalar else out

    def degree(self, v):
        scalar = np.isscalar(v)
        pv, nv, fv, kv = _arr(np.atleast_1d(v) if scalar else v, np.uint32)
        if fv:
            import torch
            out = torch.empty(nv, dtype=torch.int32, device=kv.device)
            optr = out.data_ptr()
        else:
            out = np.empty(nv, np.uint32)
            optr = out.ctypes.data
        L.check(self._L.trc_degree(self._h, C.c_void_p(pv), nv, C.c_void_p(optr), fv))
        return int(out[0]) if scalar else out

    def neighbors(self, v: int) -> np.ndarray:
        """Sorted neighbour list (the reference's NeighborIterator order)."""
        ln = C.c_uint64()
        L.check(self._L.trc_neighbors(self._h, v, None, 0, C.byref(ln), 0))
        out = np.empty(max(1, ln.value), np.uint32)
        L.check(self._L.trc_neighbors(self._h, v, C.c_void_p(out.ctypes.data), ln.value,
                                      C.byref(ln), 0))
        return out[:ln.value]

    def map_neighbors(self, v: int, f):
        """Call f(v, w) for every neighbour w in sorted order."""
        for w in self.neighbors(v):
            f(v, int(w))

    def count_common(self, s, d):
        scalar = np.isscalar(s)
        ps, ns, fs, ks = _arr(np.atleast_1d(s) if scalar else s, np.uint32)
        pd, nd, fd, kd = _arr(np.atleast_1d(d) if scalar else d, np.uint32)
        out = np.empty(ns, np.uint32)
        L.check(self._L.trc_count_common(self._h, C.c_void_p(ps), C.c_void_p(pd), ns,
                                         C.c_void_p(out.ctypes.data), 0))
        return int(out[0]) if scalar else out

    def get_num_vertices(self) -> int:
        x = C.c_uint32()
        L.check(self._L.trc_num_vertices(self._h, C.byref(x)))
        return int(x.value)

    def get_num_edges(self) -> int:
        x = C.c_uint64()
        L.check(self._L.trc_num_edges(self._h, C.byref(x)))
        return int(x.value)

    def get_size(self) -> int:
        x = C.c_uint64()
        L.check(self._L.trc_get_size(self._h, C.byref(x)))
        return int(x.value)

    def dump_csr(self):
        """(offsets uint64[n+1], targets uint32[m]) of the sorted lists."""
        m = self.get_num_edges()
        off = np.empty(self.n + 1, np.uint64)
        tgt = np.empty(max(1, m), np.uint32)
        L.check(self._L.trc_dump_csr(self._h, C.c_void_p(off.ctypes.data),
                                     C.c_void_p(tgt.ctypes.data), 0))
        return off, tgt[:m]

    # ---------------------------------------------------------------- analytics
    def _out(self, device, dtype, n):
        if device:
            import torch
            tdt = {np.int32: torch.int32, np.uint32: torch.int32, np.float64: torch.float64}[dtype]
            t = torch.empty(n, dtype=tdt, device="cuda")
            return t, t.data_ptr(), L.TRC_DEVICE_PTR
        a = np.empty(n, dtype)
        return a, a.ctypes.data, 0

    def bfs(self, src: int, device: bool = False):
        """(parents int32[n], levels uint32[n]); BFS_with_edge_map."""
        par, pp, f = self._out(device, np.int32, self.n)
        lv, pl, _ = self._out(device, np.uint32, self.n)
        L.check(self._L.trc_bfs(self._h, src, C.c_void_p(pp), C.c_void_p(pl), f))
        return par, lv

    def msbfs(self, sources, device: bool = False):
        """Levels of up to 64 BFS at once: array (k, n), TRC_UNREACHED if
        unreached (one traversal, one bit per source per vertex)."""
        src, ps, keep = self._sources(sources, device)
        k = len(src)
        out, po, f = self._out(device, np.uint32, k * self.n)
        L.check(self._L.trc_msbfs(self._h, C.c_void_p(ps), k, C.c_void_p(po), f))
        return out.reshape(k, self.n)

    @staticmethod
    def _sources(sources, device):
        """Host sources as (array, pointer, keepalive); on the device when the
        outputs are (one flag covers every array argument)."""
        src = np.ascontiguousarray(sources, np.uint32)
        if not device:
            return src, src.ctypes.data, src
        import torch
        t = torch.as_tensor(src.view(np.int32)).to("cuda")
        return src, t.data_ptr(), t

    def msbc(self, sources, device: bool = False):
        """BC of up to 64 sources at once: array (k, n), row i = bc(sources[i])
        (one traversal, one bit per source per vertex)."""
        src, ps, keep = self._sources(sources, device)
        k = len(src)
        out, po, f = self._out(device, np.float64, k * self.n)
        L.check(self._L.trc_msbc(self._h, C.c_void_p(ps), k, C.c_void_p(po), f))
        return out.reshape(k, self.n)

    def pagerank(self, iters: int, damping: float = 0.0, device: bool = False):
        """PR_S<double>; damping 0 = the reference's undamped iteration."""
        out, po, f = self._out(device, np.float64, self.n)
        L.check(self._L.trc_pagerank(self._h, iters, damping, C.c_void_p(po), f))
        return out

    def cc(self, device: bool = False):
        out, po, f = self._out(device, np.uint32, self.n)
        L.check(self._L.trc_cc(self._h, C.c_void_p(po), f))
        return out

    def bc(self, src: int, device: bool = False):
        out, po, f = self._out(device, np.float64, self.n)
        L.check(self._L.trc_bc(self._h, src, C.c_void_p(po), f))
        return out

    def tc(self) -> int:
        x = C.c_uint64()
        L.check(self._L.trc_tc(self._h, C.byref(x)))
        return int(x.value)

    # ---------------------------------------------------------------- diagnostics
    # ---------------------------------------------------------------- tuning
    def autotune(self, push_pull: bool = True, pagerank: bool = True, sample=None,
                 symmetrize: bool = True) -> dict:
        """trc_autotune: times candidate choices on this graph and keeps the
        fastest.  `sample` = (srcs, dests) tunes the PMA leaf (inserted and
        removed again; the edge set is unchanged)."""
        what = (L.TUNE_PUSH_PULL if push_pull else 0) | (L.TUNE_PAGERANK if pagerank else 0)
        ps = pd = None
        k = 0
        flags = L.TRC_SYMMETRIZE if symmetrize else 0
        keep = ()
        if sample is not None:
            what |= L.TUNE_PMA
            a, na, fa, ka = _arr(sample[0], np.uint32)
            b, nb, fb, kb = _arr(sample[1], np.uint32)
            if na != nb or fa != fb:
                raise ValueError("sample arrays differ in length or location")
            ps, pd, k, keep = C.c_void_p(a), C.c_void_p(b), na, (ka, kb)
            flags |= fa
        t = L.trc_tuning()
        L.check(self._L.trc_autotune(self._h, what, ps, pd, k, flags, C.byref(t)))
        del keep
        return {k: getattr(t, k) for k, _ in L.trc_tuning._fields_}

    def get_tuning(self) -> dict:
        t = L.trc_tuning()
        L.check(self._L.trc_get_tuning(self._h, C.byref(t)))
        return {k: getattr(t, k) for k, _ in L.trc_tuning._fields_}

    def set_tuning(self, **kw):
        t = L.trc_tuning()
        L.check(self._L.trc_get_tuning(self._h, C.byref(t)))
        for k, v in kw.items():
            setattr(t, k, v)
        L.check(self._L.trc_set_tuning(self._h, C.byref(t)))

    def stats(self) -> dict:
        s = L.trc_stats()
        L.check(self._L.trc_get_stats(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in L.trc_stats._fields_}

    def check(self) -> int:
        x = C.c_uint64()
        L.check(self._L.trc_check(self._h, C.byref(x)))
        return int(x.value)

    def profile(self, on: bool = True):
        L.check(self._L.trc_profile_enable(self._h, int(on)))

    def profile_reset(self):
        L.check(self._L.trc_profile_reset(self._h))

    def profile_get(self, name: str | None = None):
        ms = C.c_double()
        cnt = C.c_uint64()
        L.check(self._L.trc_profile_get(self._h, name.encode() if name else None,
                                        C.byref(ms), C.byref(cnt)))
        return ms.value, int(cnt.value)

    def launch_count(self) -> int:
        x = C.c_uint64()
        L.check(self._L.trc_launch_count(self._h, C.byref(x)))
        return int(x.value)

    def profile_names(self):
        buf = C.create_string_buffer(1 << 16)
        L.check(self._L.trc_profile_names(self._h, buf, len(buf)))
        return [s for s in buf.value.decode().split("\n") if s]


def rmat_generate(n: int, seed: int, a: float, b: float, c: float, count: int, first: int = 0,
                  device: bool = False, stream=None):
    """Device RMAT generator, bit-exact with rMat<uint32_t>."""
    lib = L.load()
    sp = getattr(stream, "cuda_stream", stream) or 0
    if device:
        import torch
        s = torch.empty(count, dtype=torch.int32, device="cuda")
        d = torch.empty(count, dtype=torch.int32, device="cuda")
        L.check(lib.trc_rmat_generate(n, seed & 0xFFFFFFFF, a, b, c, first, count,
                                      C.c_void_p(s.data_ptr()), C.c_void_p(d.data_ptr()),
                                      L.TRC_DEVICE_PTR, C.c_void_p(sp)))
        return s, d
    s = np.empty(max(1, count), np.uint32)
    d = np.empty(max(1, count), np.uint32)
    L.check(lib.trc_rmat_generate(n, seed & 0xFFFFFFFF, a, b, c, first, count,
                                  C.c_void_p(s.ctypes.data), C.c_void_p(d.ctypes.data), 0,
                                  C.c_void_p(sp)))
    return s[:count], d[:count]
