"""Pins of the two large workload graphs, computed by the CPU oracle
(oracle/oracle.c: the reference's rMat generator, self-loops dropped,
symmetrized, sorted and deduplicated) so that the GPU tests at these sizes
need not rebuild them on the CPU:

  config2  RMAT scale 22, edge factor 16, a/b/c .5/.1/.1, seed 0 -- the
           LiveJournal-shaped streaming workload: vertex and edge counts,
           SHA-256 of the CSR (offsets as little-endian u64, then targets as
           u32), the exact triangle count and the maximum-degree vertex
  config3  RMAT scale 24, edge factor 32, a/b/c .57/.19/.19, seed 0 -- the
           skewed workload of the blocked tier: counts, CSR SHA-256, the
           maximum-degree vertex and its degree

    python tests/golden/make_config_pins.py   # writes tests/golden/config_pins.json

Scale 24 needs about 25 GB of host memory and a few minutes.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import oracle as O  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "config_pins.json")


def csr_sha(off, tgt) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(off, "<u8").tobytes())
    h.update(np.ascontiguousarray(tgt, "<u4").tobytes())
    return h.hexdigest()


def pin(scale, ef, a, b, c, tc=False):
    t0 = time.time()
    n, keys = O.rmat_graph_keys(scale, ef, a, b, c, 0)
    off, tgt = O.csr_from_keys(n, keys)
    del keys
    deg = np.diff(off.astype(np.int64))
    rec = {"scale": scale, "edge_factor": ef, "a": a, "b": b, "c": c, "seed": 0,
           "n": n, "m": int(off[-1]), "csr_sha256": csr_sha(off, tgt),
           "argmax_degree": int(deg.argmax()), "max_degree": int(deg.max())}
    if tc:
        rec["tc_exact"] = O.tc(off, tgt)
    rec["seconds"] = round(time.time() - t0, 1)
    print(rec, flush=True)
    return rec


def main():
    pins = {"config2": pin(22, 16, .5, .1, .1, tc=True),
            "config3": pin(24, 32, .57, .19, .19)}
    with open(OUT, "w") as f:
        json.dump(pins, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
