"""The rule the 32-bit tier uses to decide a node with few candidates in one
step, checked on the CPU against networkx: below a node with clique R,
candidates P and active rows A (the vertices outside R adjacent to all of R),
the maximal cliques are exactly R + K for the cliques K of P that no vertex of
A contains (K is contained in a vertex's row when that vertex is adjacent to
all of K).  Applied at every edge root (v0 < v1 in a vertex order, P = common
neighbours above v1, A = all common neighbours), it must reproduce each
root's share of the maximal cliques."""
from __future__ import annotations

import itertools
import random

import networkx as nx
import pytest


def cliques_by_rule(g: nx.Graph, order):
    pos = {v: i for i, v in enumerate(order)}
    out = set()
    for a, b in g.edges():
        v0, v1 = (a, b) if pos[a] < pos[b] else (b, a)
        common = set(g[v0]) & set(g[v1])
        P = sorted(c for c in common if pos[c] > pos[v1])
        A = common  # every common neighbour is adjacent to R = {v0, v1}
        if not common:
            out.add(frozenset((v0, v1)))
            continue
        for k in range(1, len(P) + 1):
            for K in itertools.combinations(P, k):
                if any(y not in g[x] for x, y in itertools.combinations(K, 2)):
                    continue
                ks = set(K)
                if any(ks <= set(g[w]) for w in A if w not in ks):
                    continue
                out.add(frozenset((v0, v1, *K)))
    return out


@pytest.mark.parametrize("seed", range(6))
def test_rule_reproduces_maximal_cliques(seed):
    rnd = random.Random(seed)
    n, p = 14, 0.45 + 0.05 * (seed % 3)
    g = nx.Graph()
    g.add_edges_from((u, v) for u, v in itertools.combinations(range(n), 2) if rnd.random() < p)
    g.remove_nodes_from([v for v in list(g) if g.degree(v) == 0])
    order = sorted(g, key=lambda v: (nx.core_number(g)[v], v))
    want = {frozenset(c) for c in nx.find_cliques(g)}
    assert cliques_by_rule(g, order) == want
