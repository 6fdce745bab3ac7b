#!/usr/bin/env python
"""Write a benchmark graph as a reference `.bin`, in the engine's vertex order.

TEST INFRASTRUCTURE: bench.py's reference arm runs this as a separate process
before it times the reference, so the timed process loads only the reference
build.  The pairs come from the engine's host generators (CPU code, identical
for any thread count); the oracle orders them with its restatement of the
engine's round-synchronous peel (og_sort_gpu_rounds) and writes the `.bin`
container (src/graph.cc:154-176 layout).  The reference then loads it in
stored order (main.cc:26 sorts only non-.bin input), so edge root r means the
same edge (v0 < v1) for the reference and the engine.

    python oracle/ordered_bin.py rmat20 OUT.bin
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))

GRAPHS = {"rmat20": (20, 16, 2), "rmat14": (14, 16, 1), "rmat16": (16, 16, 1)}


def main():
    if len(sys.argv) != 3 or sys.argv[1] not in GRAPHS:
        print(f"usage: {sys.argv[0]} {'|'.join(GRAPHS)} OUT.bin", file=sys.stderr)
        return 2
    import oracle
    import rdmce_b200 as mce

    scale, ef, seed = GRAPHS[sys.argv[1]]
    u, v = mce.gen_rmat(scale, ef, seed)
    g = oracle.Graph.from_pairs(u, v).sort_gpu_rounds()
    g.store_bin(sys.argv[2])
    off, adj, lab = g.export()
    h = hashlib.sha256()
    for a in (off.astype("<u4"), adj.astype("<u4"), lab.astype("<u4")):
        h.update(np.ascontiguousarray(a).tobytes())
    print(f"n {g.n} m {g.m} degeneracy {g.degeneracy} csr_sha256 {h.hexdigest()}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
