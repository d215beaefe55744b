"""Small, self-contained runs of single hot kernels, sized for ncu captures.

    python -m terrace_b200.profile_case pagerank --scale 24 --ef 8 --iters 3
    python -m terrace_b200.profile_case bfs --scale 24 --ef 8
    python -m terrace_b200.profile_case insert --scale 22 --ef 16 --batches 3

Each case builds an RMAT graph on the device (the reference generator,
a=.57 b=.19 c=.19 for PageRank/BFS, a=.5 b=.1 c=.1 for inserts), frees the
build's temporaries, then runs the named operation a few times inside an
NVTX range "timed" (insert: the benchmark's batches of seed stream 1, after
one untimed batch).  The
profiles/ summaries name the exact command line they were made with.
"""
from __future__ import annotations

import argparse
import time

import numpy as np


def _range(name):
    """NVTX range around the measured part (ncu --nvtx --nvtx-include name/)."""
    import torch
    try:
        torch.cuda.nvtx.range_push(name)
        return lambda: torch.cuda.nvtx.range_pop()
    except Exception:
        return lambda: None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["pagerank", "bfs", "insert", "bc", "cc"])
    ap.add_argument("--scale", type=int, default=22)
    ap.add_argument("--ef", type=int, default=16)
    ap.add_argument("--iters", type=int, default=3)
    ap.add_argument("--batches", type=int, default=3)
    ap.add_argument("--batch", type=int, default=1_000_000)
    args = ap.parse_args()
    import torch
    import terrace_b200 as T
    from terrace_b200.workload import batch_seed

    n = 1 << args.scale
    abc = (.5, .1, .1) if args.case == "insert" else (.57, .19, .19)
    s, d = T.rmat_generate(n, 0, *abc, args.ef * n, device=True)
    g = T.Graph(n)
    m = g.add_edge_batch(s, d, symmetrize=True, drop_self_loops=True)
    del s, d
    g.release_scratch()
    torch.cuda.empty_cache()
    deg = g.degree(np.arange(n, dtype=np.uint32))
    src = int(np.argmax(deg))
    if args.case == "insert":  # one untimed batch first (buffers sized)
        bs, bd = T.rmat_generate(n, batch_seed(1, 0), *abc, args.batch, device=True)
        g.add_edge_batch(bs, bd, symmetrize=True, drop_self_loops=True)
    else:  # degree-class lists built outside the range
        g.pagerank(1, device=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    end = _range("timed")
    if args.case == "pagerank":
        g.pagerank(args.iters, device=True)
    elif args.case == "bfs":
        for _ in range(args.iters):
            g.bfs(src, device=True)
    elif args.case == "bc":
        g.bc(src, device=True)
    elif args.case == "cc":
        for _ in range(args.iters):
            g.cc(device=True)
    else:
        for j in range(1, args.batches + 1):
            bs, bd = T.rmat_generate(n, batch_seed(1, j), *abc, args.batch, device=True)
            g.add_edge_batch(bs, bd, symmetrize=True, drop_self_loops=True)
    torch.cuda.synchronize()
    end()
    print(f"{args.case} scale {args.scale} ef {args.ef}: m={m} {time.perf_counter() - t0:.3f}s")


if __name__ == "__main__":
    main()
