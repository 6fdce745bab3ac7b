"""Generate the golden maximal-clique fixtures in this directory.

Each fixture is a small edge list plus the expected clique count, clique-size
histogram and checksum.  Expected values come from networkx.find_cliques (an
independent Bron-Kerbosch implementation), restricted to the vertices that
appear in at least one non-loop edge -- the reference loader drops the others
(RDMCE src/graph.cc:64-152).  The checksum is the engine's order-independent
set hash: sum over cliques C (mod 2^64) of
mix64(s1 ^ rotl(s2, 31) ^ (|C| << 56)), s1 = sum mix64(l), s2 = sum
mix64(l ^ 0x9E3779B97F4A7C15) over the labels l of C, mix64 = SplitMix64's
output function.  The zachary fixture reads the one graph the reference ships
(RDMCE/data/zachary.txt) when that tree is present.

Run:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import itertools
import json
import os
import random
from collections import Counter

import networkx as nx

HERE = os.path.dirname(os.path.abspath(__file__))
M64 = (1 << 64) - 1
G = 0x9E3779B97F4A7C15
# the reference's own data/zachary.txt, found through RDMCE_REFERENCE (the
# RDMCE/ directory of the reference tree); skipped when that is not set
REF_ZACHARY = os.path.join(os.environ.get("RDMCE_REFERENCE", ""), "data", "zachary.txt")


def mix64(x: int) -> int:
    z = (x + G) & M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def clique_hash(labels) -> int:
    s1 = s2 = 0
    for l in labels:
        s1 = (s1 + mix64(l)) & M64
        s2 = (s2 + mix64(l ^ G)) & M64
    rot = ((s2 << 31) | (s2 >> 33)) & M64
    return mix64(s1 ^ rot ^ ((len(labels) << 56) & M64))


def expected(edges):
    g = nx.Graph()
    g.add_edges_from((u, v) for u, v in edges if u != v)
    cliques = list(nx.find_cliques(g)) if g.number_of_edges() else []
    hist = Counter(len(c) for c in cliques)
    chk = 0
    for c in cliques:
        chk = (chk + clique_hash(c)) & M64
    return {"count": len(cliques), "checksum": f"{chk:016x}", "hist": {str(k): v for k, v in sorted(hist.items())},
            "n": g.number_of_nodes(), "m": g.number_of_edges(),
            "degeneracy": max(nx.core_number(g).values()) if g.number_of_nodes() else 0}


def fixture(name, edges, note):
    d = {"name": name, "note": note, "edges": [[int(u), int(v)] for u, v in edges]}
    d.update(expected(edges))
    with open(os.path.join(HERE, f"{name}.json"), "w") as f:
        json.dump(d, f, separators=(",", ":"))
    print(name, d["count"], d["checksum"], d["hist"])


def gnp(n, p, seed):
    rnd = random.Random(seed)
    return [(u, v) for u, v in itertools.combinations(range(n), 2) if rnd.random() < p]


def main():
    if os.path.exists(REF_ZACHARY):
        edges = []
        with open(REF_ZACHARY) as f:
            for line in f:
                t = line.split()
                if len(t) >= 2 and t[0].isdigit() and t[1].isdigit():
                    edges.append((int(t[0]), int(t[1])))
        fixture("zachary", edges, "the reference's bundled graph (labels 1..34)")
    fixture("k12", list(itertools.combinations(range(12), 2)), "K_12: one clique")
    fixture("c9", [(i, (i + 1) % 9) for i in range(9)], "C_9: 9 cliques of size 2")
    # Moon-Moser K_{3,3,3,3}: complement of 4 disjoint triangles, 3^4 cliques
    parts = [list(range(3 * i, 3 * i + 3)) for i in range(4)]
    mm = [(u, v) for a, b in itertools.combinations(range(4), 2) for u in parts[a] for v in parts[b]]
    fixture("moon_moser_12", mm, "K_{3,3,3,3}: 81 cliques of size 4")
    fixture("star_with_loops", [(0, i) for i in range(1, 8)] + [(3, 3), (9, 9), (2, 5)],
            "star + a self-loop-only vertex (9) that the loader drops")
    fixture("two_k5_share_vertex",
            list(itertools.combinations(range(5), 2)) + list(itertools.combinations([4, 5, 6, 7, 8], 2)),
            "two K_5 sharing vertex 4")
    fixture("gnp60", gnp(60, 0.3, 11), "G(60, 0.3)")
    fixture("gnp120", gnp(120, 0.15, 12), "G(120, 0.15)")
    fixture("gnp90_dense", gnp(90, 0.55, 13), "G(90, 0.55): wide candidate sets")
    big = [(u + 1000, v + 1000) for u, v in gnp(80, 0.4, 14)]
    fixture("sparse_labels", big + [(5, 4_000_000_000), (5, 77), (77, 4_000_000_000)],
            "labels far from 0 and near 2^32: dense relabel must keep the originals")


if __name__ == "__main__":
    main()
