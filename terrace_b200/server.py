"""Python mirror of the serving layer (trc_server_* in include/terrace_b200.h)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L


class Server:
    """Continuous-batching request server over a Graph (see trc_server_create).

    While it runs, use the graph only through the server."""

    def __init__(self, graph, batched: bool = True, summary: bool = False, symmetrize: bool = True,
                 max_bfs_group: int = 64, max_round_edges: int = 1 << 24):
        self._L = L.load()
        cfg = L.trc_server_config()
        self._L.trc_server_config_default(C.byref(cfg))
        cfg.mode = L.SERVE_BATCHED if batched else L.SERVE_FIFO
        cfg.result_mode = L.RESULT_SUMMARY if summary else L.RESULT_FULL
        cfg.symmetrize = int(symmetrize)
        cfg.max_bfs_group = max_bfs_group
        cfg.max_round_edges = max_round_edges
        h = C.c_void_p()
        L.check(self._L.trc_server_create(graph._h, C.byref(cfg), C.byref(h)))
        self._h = h
        self.graph = graph

    def close(self):
        if getattr(self, "_h", None):
            L.check(self._L.trc_server_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, kind: int, a=None, b=None, param: int = 0) -> int:
        keep = []
        pa = pb = None
        k = 0
        if a is not None:
            a = np.ascontiguousarray(a, np.uint32)
            keep.append(a)
            pa = C.c_void_p(a.ctypes.data)
            k = len(a)
        if b is not None:
            b = np.ascontiguousarray(b, np.uint32)
            keep.append(b)
            pb = C.c_void_p(b.ctypes.data)
        rid = C.c_uint64()
        L.check(self._L.trc_server_submit(self._h, kind, pa, pb, k, param, C.byref(rid)))
        return int(rid.value)

    def insert(self, src, dst):
        return self.submit(L.REQ_INSERT, src, dst)

    def delete(self, src, dst):
        return self.submit(L.REQ_DELETE, src, dst)

    def bfs(self, src: int):
        return self.submit(L.REQ_BFS, param=src)

    def degree(self, vertices):
        return self.submit(L.REQ_DEGREE, vertices)

    def neighbors(self, v: int):
        return self.submit(L.REQ_NEIGHBORS, param=v)

    def pagerank(self, iters: int):
        return self.submit(L.REQ_PAGERANK, param=iters)

    def wait(self, rid: int, timeout_ms: int = -1):
        L.check(self._L.trc_server_wait(self._h, rid, timeout_ms))

    def result(self, rid: int, dtype=np.uint32):
        """(array, latency_ms, version, status) of a finished request."""
        nb = C.c_uint64()
        lat = C.c_double()
        ver = C.c_uint64()
        st = C.c_int()
        L.check(self._L.trc_server_result(self._h, rid, None, 0, C.byref(nb), C.byref(lat),
                                          C.byref(ver), C.byref(st)))
        out = np.empty(max(1, nb.value), np.uint8)
        L.check(self._L.trc_server_result(self._h, rid, C.c_void_p(out.ctypes.data), nb.value,
                                          C.byref(nb), C.byref(lat), C.byref(ver), C.byref(st)))
        return out[:nb.value].view(dtype), lat.value, int(ver.value), int(st.value)

    def release(self, rid: int):
        L.check(self._L.trc_server_release(self._h, rid))

    def stats(self, kind: int = -1) -> dict:
        s = L.trc_server_stats()
        L.check(self._L.trc_server_get_stats(self._h, kind, C.byref(s)))
        return {k: getattr(s, k) for k, _ in L.trc_server_stats._fields_}

    def rounds(self) -> list:
        """The per-round trace (trc_server_rounds), oldest first, as dicts."""
        cnt = C.c_uint64()
        L.check(self._L.trc_server_rounds(self._h, None, 0, C.byref(cnt)))
        buf = (L.trc_round_record * max(cnt.value, 1))()
        L.check(self._L.trc_server_rounds(self._h, buf, cnt.value, C.byref(cnt)))
        return [{k: getattr(r, k) for k, _ in L.trc_round_record._fields_}
                for r in buf[:cnt.value]]

    def reset_stats(self):
        L.check(self._L.trc_server_reset_stats(self._h))

    def hold(self, on: bool = True):
        """While held no new round starts; release (hold(False)) to serve
        everything queued meanwhile as one round."""
        L.check(self._L.trc_server_hold(self._h, 1 if on else 0))
