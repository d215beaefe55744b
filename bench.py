#!/usr/bin/env python
"""Benchmark of the Terrace hot path on B200.

Workload (N=1 line): streaming updates on a LiveJournal-shaped RMAT graph --
scale 22 (4,194,304 vertices), edge factor 16, a=.5 b=.1 c=.1, seed 0,
symmetrized, self-loops dropped (the reference's RMAT generator, bit-exact).
One step = one batch of 1,000,000 RMAT (src,dst) pairs (seed stream 1,
symmetrized) inserted through the library.  value = directed edges inserted
per second over the K timed steps, batches already resident in HBM.

Also measured (extra keys): deletes of the same batches, BFS / PageRank /
CC / BC / TC on the scale-22 graph, and BFS / PageRank GTEPS with their HBM
roofline on the scale-24 RMAT graph (ef 32, a=.57 b=.19 c=.19).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

--impl reference times the reference Terrace CPU build
(oracle/_ref/libterrace_ref.so, compiled from the reference sources) on the
host cores, same workload and metric.  Under torchrun each rank is an
independent replica (the path does not shard: "replicas only").
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SCALE, EF, A, B, C = 22, 16, 0.5, 0.1, 0.1
BATCH = 1_000_000
BATCH_STREAM = 1
S24 = (24, 32, 0.57, 0.19, 0.19)


def hash32(a: int) -> int:
    a &= 0xFFFFFFFF
    a = ((a + 0x7ED55D16) + (a << 12)) & 0xFFFFFFFF
    a = ((a ^ 0xC761C23C) ^ (a >> 19)) & 0xFFFFFFFF
    a = ((a + 0x165667B1) + (a << 5)) & 0xFFFFFFFF
    a = ((a + 0xD3A2646C) ^ (a << 9)) & 0xFFFFFFFF
    a = ((a + 0xFD7046C5) + (a << 3)) & 0xFFFFFFFF
    a = ((a ^ 0xB55A4F09) ^ (a >> 16)) & 0xFFFFFFFF
    return a


def batch_seed(stream: int, j: int) -> int:
    return hash32(stream) ^ j


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# --------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_{os.getpid()}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader",
                                          "-i", str(self.idx), "-lms", "100"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        self.f.close()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        try:
            os.remove(self.path)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}

        def mhz(s):
            try:
                return float(s.split()[0])
            except Exception:
                return None
        sm = [mhz(r[1]) for r in rows if mhz(r[1])]
        mx = max((mhz(r[2]) or 0) for r in rows)
        reasons = set()
        for r in rows:
            for name, val in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                                  "sw_power_cap"), r[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        loaded = [x for x in sm if x > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(rows)}


# ------------------------------------------------------------- our GPU arm
def run_ours(args, rank, world):
    import torch
    import terrace_b200 as T
    from terrace_b200 import build as TB
    if not os.path.exists(T.LIB_PATH):
        TB.build()
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream()
    hbm_gbs, peak_kind = load_peaks()
    n = 1 << SCALE

    # ---- setup (untimed): graph and batches resident in HBM
    s, d = T.rmat_generate(n, 0, A, B, C, EF * n, device=True)
    g = T.Graph(n)
    g.set_stream(stream)
    t0 = time.perf_counter()
    m0 = g.add_edge_batch(s, d, symmetrize=True, drop_self_loops=True)
    torch.cuda.synchronize()
    bulk_s = time.perf_counter() - t0
    del s, d
    nb = args.warmup + 2 * args.steps
    batches = [T.rmat_generate(n, batch_seed(BATCH_STREAM, j), A, B, C, BATCH, device=True)
               for j in range(nb)]
    torch.cuda.synchronize()

    def timed(fn, K, flush=False):
        """Max over ranks of device time of K calls of fn(i) (ms/step)."""
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        out = [fn(i) for i in range(K)]
        ev1.record(stream)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        ms = ev0.elapsed_time(ev1)
        if world > 1:
            t = torch.tensor([ms], device=dev)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            ms = float(t.item())
        return ms, out

    # ---- warm-up inserts (W), then K timed inserts, then deletes of all
    for j in range(args.warmup):
        g.add_edge_batch(*batches[j], symmetrize=True, drop_self_loops=True)
    l0 = g.launch_count()
    clk = ClockSampler(dev.index)
    clk.start()
    ins_ms, ins = timed(lambda i: g.add_edge_batch(*batches[args.warmup + i], symmetrize=True,
                                                   drop_self_loops=True), args.steps)
    clocks = clk.stop()
    launches = g.launch_count() - l0
    inserted = sum(ins)
    value = inserted * world / (ins_ms / 1e3)
    pairs_per_s = BATCH * args.steps * world / (ins_ms / 1e3)
    del_ms, dels = timed(lambda i: g.remove_edge_batch(*batches[args.warmup + i], symmetrize=True,
                                                       drop_self_loops=True), args.steps)
    deleted = sum(dels)

    # ---- profiled pass (separate from the timed region): K fresh batches of
    # the same stream, CUDA events around every kernel, per-batch sizes
    g.profile(True)
    g.profile_reset()
    sizes = []
    pb = batches[args.warmup + args.steps:]
    for bs_, bd_ in pb:
        g.add_edge_batch(bs_, bd_, symmetrize=True, drop_self_loops=True)
        sizes.append(g.stats())
    allk = {name: g.profile_get(name) for name in g.profile_names()}
    kernel_ms = {k: v for k, v in allk.items() if not k.startswith("host:")}
    host_ms = {k[5:]: v[0] / len(pb) for k, v in allk.items() if k.startswith("host:")}
    g.profile(False)
    for bs_, bd_ in pb:
        g.remove_edge_batch(bs_, bd_, symmetrize=True, drop_self_loops=True)
    for j in range(args.warmup):
        g.remove_edge_batch(*batches[j], symmetrize=True, drop_self_loops=True)

    # ---- e2e: same metric through the public API with pinned HOST buffers
    host = []
    for j in range(args.steps):
        hs = torch.empty(BATCH, dtype=torch.int32, pin_memory=True)
        hd = torch.empty(BATCH, dtype=torch.int32, pin_memory=True)
        hs.copy_(batches[args.warmup + j][0].cpu())
        hd.copy_(batches[args.warmup + j][1].cpu())
        host.append((hs.numpy().view(np.uint32), hd.numpy().view(np.uint32)))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_cnt = [g.add_edge_batch(hs, hd, symmetrize=True, drop_self_loops=True) for hs, hd in host]
    e2e_s = time.perf_counter() - t0
    for hs, hd in host:
        g.remove_edge_batch(hs, hd, symmetrize=True, drop_self_loops=True)
    e2e_val = sum(e2e_cnt) * world / e2e_s

    # ---- analytics on the scale-22 graph (device outputs)
    st = g.stats()
    off_deg = g.degree(np.arange(n, dtype=np.uint32))
    src = int(np.argmax(off_deg))
    reached_deg = 0

    def t_call(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        t = []
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = fn()
            e1.record(stream)
            torch.cuda.synchronize()
            t.append(e0.elapsed_time(e1))
        return min(t), r

    bfs_ms, (par, lv) = t_call(lambda: g.bfs(src, device=True))
    lvh = lv.cpu().numpy().view(np.uint32)
    reached_deg = int(off_deg[lvh != 0xFFFFFFFF].astype(np.int64).sum())
    pr_ms, _ = t_call(lambda: g.pagerank(10, device=True))
    cc_ms, _ = t_call(lambda: g.cc(device=True))
    bc_ms, _ = t_call(lambda: g.bc(src, device=True), reps=2)
    tc_ms, tcount = t_call(lambda: g.tc(), reps=1)
    m22 = g.get_num_edges()
    analytics22 = {
        "graph": f"rmat{SCALE} ef{EF}", "m": m22,
        "bfs_ms": bfs_ms, "bfs_gteps": reached_deg / 2 / (bfs_ms / 1e3) / 1e9,
        "pagerank10_ms": pr_ms, "pagerank_gteps": 10 * m22 / (pr_ms / 1e3) / 1e9,
        "cc_ms": cc_ms, "bc_ms": bc_ms, "tc_ms": tc_ms, "triangles": tcount,
    }

    # ---- roofline of the dominant kernel of the timed insert steps
    dom = max(kernel_ms.items(), key=lambda kv: kv[1][0])
    roof = roofline_for(dom[0], dom[1], sizes, hbm_gbs, peak_kind)
    total_kernel_ms = sum(v[0] for v in kernel_ms.values())

    g.close()
    del batches
    torch.cuda.empty_cache()

    # ---- scale-24 static analytics (BFS / PageRank roofline target)
    s24 = {} if args.skip_scale24 else scale24(T, torch, stream, hbm_gbs, peak_kind)

    res = {
        "metric": "insert edges/s (batch 1e6 pairs, symmetrized)",
        "value": value, "unit": "edges/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ins_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (RMAT generator of the reference, bit-exact; seeded)",
        "config": {"workload": f"streaming updates: RMAT scale {SCALE} ef {EF} a={A} b={B} c={C} seed 0 "
                               f"symmetrized ({m0} directed edges), batches of {BATCH} pairs (seed stream "
                               f"{BATCH_STREAM}) inserted, inputs resident in HBM",
                   "batch_pairs": BATCH, "graph_edges": m0, "l2": "working set > L2 (graph ~0.9 GB)",
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "pairs_per_s": pairs_per_s,
        "delete_edges_per_s": deleted * world / (del_ms / 1e3),
        "bulk_load_edges_per_s": m0 / bulk_s,
        "e2e": {"value": e2e_val, "unit": "edges/s", "h2d_bytes_per_step": 8 * BATCH,
                "d2h_bytes_per_step": 8},
        "gpu_launches": launches,
        "clocks": clocks,
        "roofline": roof,
        "host_phase_ms_per_batch": {k: round(v, 3) for k, v in host_ms.items()},
        "kernel_ms_per_batch": round(total_kernel_ms / args.steps, 3),
        "kernel_share": {k: round(v[0] / total_kernel_ms, 4) for k, v in
                         sorted(kernel_ms.items(), key=lambda kv: -kv[1][0])[:12]},
        "analytics_rmat22": analytics22,
        "analytics_rmat24": s24,
        "tiers": {k: st[k] for k in ("inline_edges", "pma_edges", "hub_edges", "num_hubs",
                                     "pma_capacity", "pma_rebuilds", "pma_window_rebalances")},
    }
    return res


def kernel_bytes(name, sz):
    """Algorithmic bytes of one launch of an update-pipeline kernel for a
    batch with sizes `sz` (trc_stats last_*): the bytes the kernel must move
    (DESIGN.md lists the formulas)."""
    k2, kb, nr = sz["last_keys"], sz["last_applied"], sz["last_rewritten"]
    so, sn = sz["last_gathered"], sz["last_written"]
    if name == "upd_merge_small":  # old list in (4 B), batch keys in (8 B), new list out (4 B)
        return 4 * so + 8 * kb + 4 * sn + 40 * nr
    if name == "upd_gather":      # old lists (4 B) -> 64-bit keys; per-vertex metadata
        return 12 * so + 28 * nr
    if name == "merge":           # two sorted key streams in, one out
        return 8 * (so + kb) + 8 * sn
    if name == "upd_scatter":     # keys in, 4-byte lists out; per-vertex metadata
        return 12 * sn + 28 * nr
    if name == "radix_scatter":   # read + write one key per pass
        return 16 * k2
    if name == "radix_hist":
        return 8 * k2
    return None


def roofline_for(name, ms_cnt, sizes, hbm_gbs, peak_kind):
    """Algorithmic bytes per launch of the dominant insert kernel divided by
    its mean CUDA-event duration (profiled pass of the same batches)."""
    ms, cnt = ms_cnt
    per_launch_ms = ms / max(cnt, 1)
    per = [kernel_bytes(name, sz) for sz in sizes]
    if any(b is None for b in per):
        return {"bound": "hbm", "kernel": name, "achieved": None, "peak": hbm_gbs, "unit": "GB/s",
                "frac": None, "traffic": None, "peak_kind": peak_kind,
                "note": "no byte formula for this kernel", "launch_ms": per_launch_ms}
    bytes_per = sum(per) / len(per)
    achieved = bytes_per / (per_launch_ms / 1e3) / 1e9
    return {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": hbm_gbs, "unit": "GB/s",
            "frac": achieved / hbm_gbs, "traffic": None, "peak_kind": peak_kind,
            "bytes_per_launch": bytes_per, "launch_ms": per_launch_ms}


def scale24(T, torch, stream, hbm_gbs, peak_kind):
    sc, ef, a, b, c = S24
    n = 1 << sc
    s, d = T.rmat_generate(n, 0, a, b, c, ef * n, device=True)
    g = T.Graph(n)
    g.set_stream(stream)
    t0 = time.perf_counter()
    m = g.add_edge_batch(s, d, symmetrize=True, drop_self_loops=True)
    torch.cuda.synchronize()
    load_s = time.perf_counter() - t0
    del s, d
    torch.cuda.empty_cache()
    deg = g.degree(np.arange(n, dtype=np.uint32))
    src = int(np.argmax(deg))
    g.profile(True)

    def best(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        out = []
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = fn()
            e1.record(stream)
            torch.cuda.synchronize()
            out.append(e0.elapsed_time(e1))
        return min(out), r

    g.profile_reset()
    bfs_ms, (par, lv) = best(lambda: g.bfs(src, device=True))
    bfs_prof = {k: g.profile_get(k) for k in g.profile_names()}
    lvh = lv.cpu().numpy().view(np.uint32)
    reached = lvh != 0xFFFFFFFF
    rdeg = int(deg[reached].astype(np.int64).sum())
    g.profile_reset()
    pr_ms, _ = best(lambda: g.pagerank(10, device=True))
    pr_prof = {k: g.profile_get(k) for k in g.profile_names()}
    st = g.stats()
    g.close()
    # algorithmic bytes: BFS 4*sum_R deg + 12 n; PR per iteration 4 m + 28 n
    bfs_bytes = 4 * rdeg + 12 * n
    pr_bytes_it = 4 * m + 28 * n
    pr_kernel_ms = sum(v[0] for k, v in pr_prof.items() if k.startswith("pr_")) / 4  # 4 runs
    pr_gbs = pr_bytes_it * 10 / (pr_kernel_ms / 1e3) / 1e9
    return {
        "graph": f"rmat{sc} ef{ef} a={a} b={b} c={c}", "n": n, "m": m, "bulk_load_s": load_s,
        "bulk_load_edges_per_s": m / load_s,
        "bfs_src": src, "bfs_ms": bfs_ms, "bfs_reached": int(reached.sum()),
        "bfs_gteps": rdeg / 2 / (bfs_ms / 1e3) / 1e9,
        "bfs_hbm_gbs": bfs_bytes / (bfs_ms / 1e3) / 1e9,
        "bfs_roofline_frac": bfs_bytes / (bfs_ms / 1e3) / 1e9 / hbm_gbs,
        "pagerank10_ms": pr_ms, "pagerank_gteps": 10 * m / (pr_ms / 1e3) / 1e9,
        "pagerank_kernel_ms_per_iter": pr_kernel_ms / 10,
        "pagerank_hbm_gbs": pr_gbs, "pagerank_roofline_frac": pr_gbs / hbm_gbs,
        "peak_gbs": hbm_gbs, "peak_kind": peak_kind,
        "pr_kernels": {k: v for k, v in pr_prof.items()},
        "bfs_kernels": {k: v for k, v in bfs_prof.items()},
        "tiers": {k: st[k] for k in ("inline_edges", "pma_edges", "hub_edges", "num_hubs")},
    }


# ------------------------------------------------------------ CPU baselines
def reference_insert_run(steps, warmup, threads, scale=SCALE, sample_note=None):
    """Reference Terrace (oracle/_ref) on the host: bulk load (untimed), then
    `steps` timed add_edge_batch calls of 1e6-pair batches (sorted, deduped,
    only new edges -- the reference's preconditions, prepared untimed as
    src/graph_bm.cc:343-355 does)."""
    import oracle as O
    O.ref_lib().ref_set_threads(threads)
    n = 1 << scale
    _, keys = O.rmat_graph_keys(scale, EF, A, B, C, 0)
    R = O.RefGraph(n + 1)  # spare last vertex: see tests/golden/make_golden.py
    R.add_keys(keys, 0)
    cur = keys
    times, counts = [], []
    for j in range(warmup + steps):
        bs, bd = O.rmat(n, batch_seed(BATCH_STREAM, j), A, B, C, BATCH)
        bk = O.make_keys(bs, bd, True, True)
        new = O.key_difference(bk, cur)
        cur = O.key_union(cur, bk)
        t0 = time.perf_counter()
        R.add_keys(new, perm_seed=j + 1)
        dt = time.perf_counter() - t0
        if j >= warmup:
            times.append(dt)
            counts.append(len(new))
    R.close()
    return sum(counts) / sum(times), sum(times), len(keys)


def run_reference_arm(args, rank, world):
    import oracle as O
    if rank != 0:
        return None
    if not O.ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libterrace_ref.so not built "
                "(oracle/build_ref.sh needs the reference sources)"}
    threads = os.cpu_count() or 1
    val, tsum, m = reference_insert_run(args.steps, args.warmup, threads)
    return {
        "impl": "reference", "metric": "insert edges/s (batch 1e6 pairs, symmetrized)",
        "value": val, "unit": "edges/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * tsum / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (RMAT generator of the reference; seeded)",
        "config": {"workload": f"streaming updates: RMAT scale {SCALE} ef {EF} a={A} b={B} c={C} seed 0 "
                               f"symmetrized ({m} directed edges), batches of {BATCH} pairs inserted",
                   "batch_pairs": BATCH, "graph_edges": m},
        "cpu_baseline": {"value": val, "unit": "edges/s", "cores": threads, "kind": "reference",
                         "sample": f"{args.steps} timed add_edge_batch calls of 1e6-pair batches "
                                   "(reference OpenMP build, g++ -Ofast, all host threads)"},
        "e2e": {"value": val, "unit": "edges/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def cpu_baseline_for_ours():
    """The reference on the host, bounded sample: 3 timed 1e6-pair batches
    into the same scale-22 graph (bulk load untimed)."""
    import oracle as O
    if not O.ref_available():
        # the port: sorted-set union of a batch into the edge set
        n = 1 << SCALE
        _, keys = O.rmat_graph_keys(SCALE, EF, A, B, C, 0)
        bs, bd = O.rmat(n, batch_seed(BATCH_STREAM, 0), A, B, C, BATCH)
        t0 = time.perf_counter()
        bk = O.make_keys(bs, bd, True, True)
        new = O.key_difference(bk, keys)
        O.key_union(keys, bk)
        dt = time.perf_counter() - t0
        return {"value": len(new) / dt, "unit": "edges/s", "cores": 1, "kind": "port",
                "sample": "one 1e6-pair batch merged into the scale-22 edge set (oracle set model)"}
    threads = os.cpu_count() or 1
    val, tsum, m = reference_insert_run(3, 0, threads)
    return {"value": val, "unit": "edges/s", "cores": threads, "kind": "reference",
            "sample": f"3 add_edge_batch calls of 1e6-pair batches into the scale-22 graph "
                      f"({m} edges, bulk load untimed), {tsum:.2f} s timed"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--skip-scale24", action="store_true")
    ap.add_argument("--skip-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        res = run_reference_arm(args, rank, world)
        if res is not None:
            print(json.dumps(res), flush=True)
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    res = run_ours(args, rank, world)
    if rank == 0:
        if not args.skip_cpu_baseline:
            res["cpu_baseline"] = cpu_baseline_for_ours()
        print(json.dumps(res), flush=True)
    if world > 1:
        import torch
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
