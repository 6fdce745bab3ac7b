#!/usr/bin/env python
"""Generate the sampled-root parity fixtures under tests/golden/samples/.

The bench's workloads hold far more maximal cliques than any solver can
enumerate in full (R-MAT scale 20 holds about 1.9e14), so a step enumerates
every maximal clique under a seeded sample of edge roots.  These fixtures pin
that sample's answer with the CPU oracle, so the GPU tests and bench.py can
check the headline numbers bit-exactly.

The oracle orders the graph with its restatement of the engine's
round-synchronous peel (oracle.c og_sort_gpu_rounds), which yields the engine's
exact CSR; a root id r is then the r-th edge (v0 < v1) of that CSR on both
sides.  The fixture records a digest of the CSR, so a test first checks that
the engine built the same ordered graph, then compares per-root counts and
checksums, the totals and the clique-size histogram.

    python tests/golden/make_samples.py rmat20      # bench headline sample
    python tests/golden/make_samples.py rmat24      # R-MAT 24 + planted, stratified roots
    python tests/golden/make_samples.py batch       # 10,000 many-instance members
    python tests/golden/make_samples.py serve       # the serving loop's requests

Inputs come from the engine's host generators (rdmce_b200.gen_*), which run
on the CPU and give the same pairs for any thread count.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
OUT = os.path.join(HERE, "samples")

# R-MAT scale 20, edge factor 16, seed 2: the bench headline graph
RMAT20 = dict(scale=20, edge_factor=16, seed=2)
RMAT20_SAMPLE = dict(seed=12345, roots=256)
# R-MAT scale 24, edge factor 32, seed 3, with 256 planted cliques of 40-200
RMAT24 = dict(scale=24, edge_factor=32, seed=3, planted=256, planted_lo=40, planted_hi=200, planted_seed=3)


def csr_digest(off, adj, labels):
    """sha256 over the ordered CSR as the engine exports it (uint32, little-endian)."""
    h = hashlib.sha256()
    for a in (off, adj, labels):
        h.update(np.ascontiguousarray(a, dtype="<u4").tobytes())
    return h.hexdigest()


def sample_roots(m, k, seed):
    """The bench's seeded root sample: k distinct root ids of [0, m), ascending."""
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(m, size=min(k, m), replace=False)).astype(np.uint64)


def rmat24_pairs(mce):
    c = RMAT24
    u, v = mce.gen_rmat(c["scale"], c["edge_factor"], c["seed"])
    pu, pv = mce.gen_planted(1 << c["scale"], c["planted"], c["planted_lo"], c["planted_hi"], c["planted_seed"])
    return np.concatenate([u, pu]), np.concatenate([v, pv])


def ordered_oracle_graph(oracle, u, v):
    g = oracle.Graph.from_pairs(u, v)
    g.sort_gpu_rounds()
    return g


def graph_record(g):
    off, adj, lab = g.export()
    return {"n": int(g.n), "m": int(g.m), "degeneracy": int(g.degeneracy), "max_degree": int(g.max_degree),
            "csr_sha256": csr_digest(off.astype(np.uint32), adj, lab)}


def solve_record(g, roots, threads):
    t = time.time()
    cnt, chk, res = g.mce_root_set(roots, threads=threads)
    return {"roots": [int(r) for r in roots], "counts": [int(c) for c in cnt], "checksums": [f"{int(c):016x}" for c in chk],
            "count": int(res.count), "checksum": f"{res.checksum:016x}", "max_size": int(res.max_size),
            "hist": {str(k): int(c) for k, c in sorted(res.hist.items())},
            # the search tree of the reference's method (canonical pivot, EXPAND_R) over these roots: the
            # algorithmic work the enumeration roofline is stated against
            "canonical_tree": {"nodes": int(res.nodes), "pivot_words": int(res.pivot_words),
                               "filter_rows": int(res.filter_rows), "build_bytes": int(res.build_bytes)},
            "oracle_seconds": round(time.time() - t, 1)}


def make_rmat20(threads):
    import oracle
    import rdmce_b200 as mce

    c = RMAT20
    u, v = mce.gen_rmat(c["scale"], c["edge_factor"], c["seed"])
    g = ordered_oracle_graph(oracle, u, v)
    rec = {"graph": dict(c, generator="rdmce_b200.gen_rmat a/b/c/d=0.57/0.19/0.19/0.05"), **graph_record(g)}
    roots = sample_roots(g.m, RMAT20_SAMPLE["roots"], RMAT20_SAMPLE["seed"])
    rec["sample_seed"] = RMAT20_SAMPLE["seed"]
    rec.update(solve_record(g, roots, threads))
    return rec


def root_ids_of_edges(g, a, b):
    """Root ids of edges (a, b) with a < b in g's CSR: a's first root plus
    b's rank among a's later neighbours."""
    off, adj, _ = g.export()
    n = g.n
    row = np.repeat(np.arange(n, dtype=np.uint32), np.diff(off).astype(np.int64))
    upper = adj > row
    first = np.zeros(n + 1, np.uint64)
    np.cumsum(np.bincount(row[upper], minlength=n).astype(np.uint64), out=first[1:])
    out = np.empty(len(a), np.uint64)
    for k, (x, y) in enumerate(zip(a, b)):
        nb = adj[off[x]:off[x + 1]]
        out[k] = first[x] + np.searchsorted(nb[nb > x], y)
    return out


def make_rmat24(threads, per_stratum, root_budget_s):
    """Roots stratified by candidate-set size p (the ego network's column
    count), plus roots inside planted cliques; each kept only if the oracle
    solves it within root_budget_s on one thread, so the fixture stays cheap to
    regenerate.  Roots of the dense core with astronomically many cliques are
    thereby left to the internal-consistency checks."""
    from concurrent.futures import ThreadPoolExecutor

    import oracle
    import rdmce_b200 as mce

    c = RMAT24
    u, v = mce.gen_rmat(c["scale"], c["edge_factor"], c["seed"])
    pu, pv = mce.gen_planted(1 << c["scale"], c["planted"], c["planted_lo"], c["planted_hi"], c["planted_seed"])
    t = time.time()
    g = ordered_oracle_graph(oracle, np.concatenate([u, pu]), np.concatenate([v, pv]))
    del u, v
    print(f"rmat24: ordered graph n={g.n} m={g.m} k={g.degeneracy} in {time.time() - t:.0f} s", flush=True)
    rec = {"graph": dict(RMAT24, generator="rdmce_b200.gen_rmat + rdmce_b200.gen_planted"), **graph_record(g)}
    rng = np.random.default_rng(777)
    probe = np.sort(rng.choice(g.m, size=min(g.m, 20000), replace=False)).astype(np.uint64)
    sizes = g.root_sizes_list(probe)
    # planted-clique edges, as root ids of the ordered graph
    _, _, lab = g.export()
    order = np.argsort(lab)
    idx = rng.choice(len(pu), size=400, replace=False)
    ia = order[np.searchsorted(lab[order], pu[idx])]
    ib = order[np.searchsorted(lab[order], pv[idx])]
    planted = root_ids_of_edges(g, np.minimum(ia, ib), np.maximum(ia, ib))
    strata = [(0, 1), (1, 8), (8, 32), (32, 64), (64, 128), (128, 256), (256, 512), (512, 1024), (1024, 1 << 20)]
    pools = [(f"p in [{lo},{hi})", probe[(sizes >= lo) & (sizes < hi)], per_stratum) for lo, hi in strata]
    pools.append(("inside a planted clique", np.unique(planted), 2 * per_stratum))

    def solvable(r):
        _, _, el = g.mce_roots_timed(np.array([r], np.uint64), 1, root_budget_s)
        return el < root_budget_s * 0.95

    chosen = []
    with ThreadPoolExecutor(threads) as ex:
        for name, pool, want in pools:
            pool = pool.copy()
            rng.shuffle(pool)
            cand = [int(r) for r in pool[: 4 * want]]
            ok = [r for r, good in zip(cand, ex.map(solvable, cand)) if good][:want]
            chosen += ok
            print(f"rmat24: {name}: {len(ok)} roots kept of {len(cand)} tried ({len(pool)} in the pool)", flush=True)
    roots = np.array(sorted(set(chosen)), np.uint64)
    rec["sample"] = (f"{per_stratum} roots per p stratum of a 20,000-root probe and {2 * per_stratum} inside planted "
                     f"cliques, each solvable by the oracle in {root_budget_s} s on one thread")
    rec["strata"] = strata
    rec["p"] = [int(x) for x in g.root_sizes_list(roots)]
    rec.update(solve_record(g, roots, threads))
    return rec


BATCH_HIST = 64


def _batch_member(i):
    import oracle
    import rdmce_b200 as mce

    u, v, _ = mce.gen_batch_member(i)
    r = oracle.Graph.from_pairs(u, v).sort_degeneracy().mce(threads=1)
    h = np.zeros(BATCH_HIST, np.uint64)
    for s, c in r.hist.items():
        h[min(s, BATCH_HIST - 1)] += c
    return i, r.count, r.checksum, r.max_size, h


def make_batch(count, workers):
    """Oracle results of every many-instance member (count, checksum, largest
    clique, histogram with sizes >= 63 folded into the last bin), one member
    per task in a spawned process pool."""
    import multiprocessing as mp

    cnt = np.zeros(count, np.uint64)
    chk = np.zeros(count, np.uint64)
    mx = np.zeros(count, np.uint32)
    hist = np.zeros((count, BATCH_HIST), np.uint64)
    with mp.get_context("spawn").Pool(workers) as pool:
        for i, c, h, m, hi in pool.imap_unordered(_batch_member, range(count), chunksize=16):
            cnt[i], chk[i], mx[i], hist[i] = c, h, m, hi
    return cnt, chk, mx, hist


def serve_requests(nreq=200, seed=5):
    """The serving loop's requests: R-MAT, scale uniform in [10, 13], edge
    factor uniform in [8, 32], a/b/c/d 0.57/0.19/0.19/0.05, request k seeded
    5000 + k; the (scale, edge factor) draws come from default_rng(seed)."""
    rng = np.random.default_rng(seed)
    return [(int(rng.integers(10, 14)), int(rng.integers(8, 33)), 5000 + k) for k in range(nreq)]


def make_serve(threads):
    import oracle
    import rdmce_b200 as mce

    out = []
    for scale, ef, sd in serve_requests():
        u, v = mce.gen_rmat(scale, ef, sd)
        r = oracle.Graph.from_pairs(u, v).sort_degeneracy().mce(threads=threads)
        out.append({"scale": scale, "edge_factor": ef, "seed": sd, "count": int(r.count),
                    "checksum": f"{r.checksum:016x}", "max_size": int(r.max_size)})
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["rmat20", "rmat24", "batch", "serve"])
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--per-stratum", type=int, default=3)
    ap.add_argument("--root-budget", type=float, default=10.0)
    ap.add_argument("--batch-count", type=int, default=10000)
    a = ap.parse_args()
    os.makedirs(OUT, exist_ok=True)
    t = time.time()
    if a.what == "rmat20":
        rec = make_rmat20(a.threads)
        path = os.path.join(OUT, "rmat20_sample.json")
        with open(path, "w") as f:
            json.dump(rec, f, indent=1)
    elif a.what == "rmat24":
        rec = make_rmat24(a.threads, a.per_stratum, a.root_budget)
        path = os.path.join(OUT, "rmat24_sample.json")
        with open(path, "w") as f:
            json.dump(rec, f, indent=1)
    elif a.what == "batch":
        cnt, chk, mx, hist = make_batch(a.batch_count, a.threads)
        path = os.path.join(OUT, "batch_members.npz")
        np.savez_compressed(path, count=cnt, checksum=chk, max_size=mx, hist=hist)
    else:
        path = os.path.join(OUT, "serve_requests.json")
        with open(path, "w") as f:
            json.dump({"requests": make_serve(a.threads)}, f, indent=1)
    print(f"wrote {path} in {time.time() - t:.0f} s")


if __name__ == "__main__":
    main()
