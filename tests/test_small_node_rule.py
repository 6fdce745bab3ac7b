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


def lanes_with_bit(k):
    """Lanes (subsets 0..31) whose index has bit k set, as a 32-bit mask."""
    return sum(1 << s for s in range(32) if (s >> k) & 1)


def decide_by_masks(n, adj, holds):
    """The 32-bit tier's one-step decision of a node with n (3..7) candidates,
    restated with its warp-uniform masks: subset s = 32 g + lane, the lane
    index carrying candidates 0..4 and the group g the rest.  adj[i] is the
    candidate-adjacency bitmask of candidate i; holds[k] is the set of active
    rows containing candidate k (as a bitmask over rows).  Returns the subsets
    the kernel emits."""
    nl = min(n, 5)
    ng = n - nl
    notclique = 0
    for i, j in itertools.combinations(range(nl), 2):
        if not (adj[i] >> j) & 1:
            notclique |= lanes_with_bit(i) & lanes_with_bit(j)
    full = (1 << 64) - 1
    out = set()
    for g in range(1 << ng):
        group_clique = True
        far_all = 0
        for b in range(ng):
            if not (g >> b) & 1:
                continue
            u = nl + b
            for i in range(nl):
                if not (adj[i] >> u) & 1:
                    far_all |= lanes_with_bit(i)
            for b2 in range(b + 1, ng):
                if (g >> b2) & 1 and not (adj[u] >> (nl + b2)) & 1:
                    group_clique = False
        for lane in range(32):
            if lane >= (1 << nl) or (notclique >> lane) & 1 or (g == 0 and lane == 0):
                continue
            if (far_all >> lane) & 1 or not group_clique:
                continue
            rows = full
            members = [k for k in range(nl) if (lane >> k) & 1] + [nl + b for b in range(ng) if (g >> b) & 1]
            for k in members:
                rows &= holds[k]
            if rows == 0:
                out.add(sum(1 << k for k in members))
    return out


def decide_directly(n, adj, holds):
    out = set()
    for s in range(1, 1 << n):
        members = [k for k in range(n) if (s >> k) & 1]
        if any(not (adj[i] >> j) & 1 for i, j in itertools.combinations(members, 2)):
            continue
        rows = (1 << 64) - 1
        for k in members:
            rows &= holds[k]
        if rows == 0:
            out.add(s)
    return out


@pytest.mark.parametrize("n", [3, 4, 5, 6, 7])
def test_subset_masks_match_direct_decision(n):
    """The kernel's lane and group masks select exactly the cliques of the
    candidates that no active row contains, for 3 to 7 candidates."""
    rnd = random.Random(100 + n)
    for _ in range(300):
        p = rnd.choice([0.3, 0.6, 0.85, 1.0])
        adj = [0] * n
        for i, j in itertools.combinations(range(n), 2):
            if rnd.random() < p:
                adj[i] |= 1 << j
                adj[j] |= 1 << i
        nrows = rnd.randint(0, 12)
        rows = [sum(1 << k for k in range(n) if rnd.random() < 0.5) for _ in range(nrows)]
        holds = [sum(1 << r for r, row in enumerate(rows) if (row >> k) & 1) for k in range(n)]
        assert decide_by_masks(n, adj, holds) == decide_directly(n, adj, holds)


def complement_components(g: nx.Graph, P):
    h = nx.complement(g.subgraph(P))
    return [sorted(c) for c in nx.connected_components(h)]


def maximal_independent_sets(h: nx.Graph, comp):
    out = []
    for k in range(1, len(comp) + 1):
        for s in itertools.combinations(comp, k):
            ss = set(s)
            if any(h.has_edge(x, y) for x, y in itertools.combinations(s, 2)):
                continue
            if any(not any(h.has_edge(w, x) for x in ss) for w in comp if w not in ss):
                continue
            out.append(ss)
    return out


@pytest.mark.parametrize("seed", range(20))
def test_join_rule(seed):
    """The 32-bit tier's join decision: when no vertex outside the candidates
    is adjacent to all of R, the maximal cliques below are R + K for K the
    products of one maximal independent set (in the complement H of G[P]) per
    connected component of H."""
    rnd = random.Random(1000 + seed)
    n = rnd.randint(4, 13)
    g = nx.complete_graph(n)
    for _ in range(rnd.randint(0, n + 3)):
        a, b = rnd.sample(range(n), 2)
        if g.has_edge(a, b):
            g.remove_edge(a, b)
    P = list(range(n))
    h = nx.complement(g.subgraph(P))
    products = {frozenset()}
    for comp in complement_components(g, P):
        sets = maximal_independent_sets(h, comp)
        products = {p | frozenset(s) for p in products for s in sets}
    assert products == {frozenset(c) for c in nx.find_cliques(g)}
