"""The 32-bit tier's join decision (enum.cu t0_join), restated lane by lane on
the CPU and checked against brute force.

The kernel decides a node with candidates P (columns), no active row outside
P and R's columns RM without a search tree: components of the complement H of
G[P] by breadth-first search over closed non-neighbourhoods, each component's
maximal independent sets from its 2^s subsets (one per lane), the size
histogram as a product of polynomials (one coefficient per lane), and the
checksum by walking the products: the first components whose set counts
multiply to at most 32 are carried by the lane index, the rest by a
warp-uniform mixed-radix counter.  This file restates those steps with the
same masks, table layout and counter, on random near-complete candidate
graphs, and compares count, checksum, histogram and largest size with a brute
force enumeration of the maximal cliques of G[P] (plus R).  The clique hash is
the engine's (SplitMix64 finaliser over the two label-hash sums and the size).
"""
from __future__ import annotations

import itertools
import random

import pytest

M64 = (1 << 64) - 1
GOLDEN = 0x9E3779B97F4A7C15
K_COMP = 5  # largest component decided this way (kJoinComp)


def mix64(x):
    z = (x + GOLDEN) & M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def clique_hash(s1, s2, size):
    rot = ((s2 << 31) | (s2 >> 33)) & M64
    return mix64(s1 ^ rot ^ ((size << 56) & M64))


def popc(x):
    return bin(x).count("1")


def lowest(x):
    return x & -x


def join(row, h1, h2, P, RM, s10, s20, rsize0):
    """t0_join for one warp; row/h1/h2 indexed by lane (= column for
    candidate lanes).  Returns None where the kernel declines the node, else
    (count, checksum, histogram, largest size)."""
    lanes = range(32)
    nb = [(P & ~row[l]) & 0xFFFFFFFF if (P >> l) & 1 else 0 for l in lanes]
    if max(popc(x) for x in nb) > K_COMP:
        return None
    single = sum(1 << l for l in lanes if (P >> l) & 1 and nb[l] == 1 << l)
    rem, comps = P & ~single, []
    while rem:
        C = lowest(rem)
        fr = C
        while True:
            nbr = sum(1 << l for l in lanes if nb[l] & fr)
            fr, C = nbr & ~C, C | nbr
            if not (fr and popc(C) <= K_COMP):
                break
        if popc(C) > K_COMP:
            return None
        comps.append(C)
        rem &= ~C
    # the shared-memory table: per entry its hash sums and size
    E1, E2, ES, c_off, c_r, total = [0] * 32, [0] * 32, [0] * 32, [], [], 1
    nent = 0
    for C in comps:
        members = [i for i in lanes if (C >> i) & 1]
        ns = len(members)
        subs = []
        for l in lanes:
            sub = sum(1 << members[k] for k in range(ns) if (l >> k) & 1)
            ok = l != 0 and l < (1 << ns)
            for m in members:
                b = 1 << m
                ok = ok and (((nb[m] & sub) == b) if sub & b else ((nb[m] & sub) != 0))
            if ok:
                subs.append(sub)
        r = len(subs)
        if nent + r > 32:
            return None
        for e, sub in enumerate(subs):
            E1[nent + e] = sum(h1[m] for m in lanes if (sub >> m) & 1) & M64
            E2[nent + e] = sum(h2[m] for m in lanes if (sub >> m) & 1) & M64
            ES[nent + e] = popc(sub)
        c_off.append(nent)
        c_r.append(r)
        nent += r
        total *= r
    base = RM | single
    b1 = (s10 + sum(h1[l] for l in lanes if (base >> l) & 1)) & M64
    b2 = (s20 + sum(h2[l] for l in lanes if (base >> l) & 1)) & M64
    size0 = rsize0 + 2 + popc(base)
    # sizes: product of the components' size polynomials (lane = size - size0)
    poly = [1] + [0] * 31
    for off, r in zip(c_off, c_r):
        acc = [0] * 32
        for d in range(r):
            sz = ES[off + d]
            for l in lanes:
                if l >= sz:
                    acc[l] += poly[l - sz]
        poly = acc
    hist = {size0 + l: poly[l] for l in lanes if poly[l]}
    # lane-carried components 0 .. a - 1
    a, Q = 0, 1
    while a < len(comps) and Q * c_r[a] <= 32:
        Q *= c_r[a]
        a += 1
    p1, p2, psz = [b1] * 32, [b2] * 32, [size0] * 32
    for l in lanes:
        rest = l
        for j in range(a):
            d, rest = rest % c_r[j], rest // c_r[j]
            p1[l] = (p1[l] + E1[c_off[j] + d]) & M64
            p2[l] = (p2[l] + E2[c_off[j] + d]) & M64
            psz[l] += ES[c_off[j] + d]
    # counter-carried components a .. : warp-uniform mixed-radix counter
    dig = [0] * 32
    u1 = sum(E1[c_off[j]] for j in range(a, len(comps))) & M64
    u2 = sum(E2[c_off[j]] for j in range(a, len(comps))) & M64
    usz = sum(ES[c_off[j]] for j in range(a, len(comps)))
    chk = count = 0
    while True:
        for l in range(Q):
            chk = (chk + clique_hash((p1[l] + u1) & M64, (p2[l] + u2) & M64, psz[l] + usz)) & M64
            count += 1
        can = [j for j in range(a, len(comps)) if dig[j] + 1 < c_r[j]]
        if not can:
            break
        jmax = can[0]
        for j in range(a, jmax + 1):
            cur = c_off[j] + dig[j]
            nxt = cur + 1 if j == jmax else c_off[j]
            u1 = (u1 + E1[nxt] - E1[cur]) & M64
            u2 = (u2 + E2[nxt] - E2[cur]) & M64
            usz += ES[nxt] - ES[cur]
        for j in range(a, jmax):
            dig[j] = 0
        dig[jmax] += 1
    assert count == total
    return total, chk, hist, max(hist)


def brute(row, h1, h2, P, RM, s10, s20, rsize0):
    """Every maximal clique K of G[P], reported as R + K."""
    cols = [i for i in range(32) if (P >> i) & 1]
    rcols = [i for i in range(32) if (RM >> i) & 1]

    def adj(i, j):
        return (row[i] >> j) & 1

    chk = count = 0
    hist = {}
    for k in range(1, len(cols) + 1):
        for K in itertools.combinations(cols, k):
            if any(not adj(x, y) for x, y in itertools.combinations(K, 2)):
                continue
            if any(all(adj(w, x) for x in K) for w in cols if w not in K):
                continue
            members = list(K) + rcols
            s1 = (s10 + sum(h1[i] for i in members)) & M64
            s2 = (s20 + sum(h2[i] for i in members)) & M64
            size = rsize0 + 2 + len(members)
            chk = (chk + clique_hash(s1, s2, size)) & M64
            count += 1
            hist[size] = hist.get(size, 0) + 1
    return count, chk, hist, max(hist)


def near_complete_node(rnd, n, n_r):
    """A candidate graph on columns 0..n-1: a clique minus the edges of small
    complement components (and a few random extra non-edges), plus n_r
    columns already in R, adjacent to every candidate."""
    missing = set()
    perm = list(range(n))
    rnd.shuffle(perm)
    i = 0
    while i < n:
        size = rnd.choice([1, 2, 2, 3, 3, 4, 5])
        comp = perm[i:i + size]
        i += size
        if len(comp) < 2:
            continue
        shape = rnd.choice(["path", "cycle", "star", "dense"])
        if shape == "path":
            pairs = list(zip(comp, comp[1:]))
        elif shape == "cycle":
            pairs = list(zip(comp, comp[1:] + comp[:1])) if len(comp) > 2 else [tuple(comp)]
        elif shape == "star":
            pairs = [(comp[0], c) for c in comp[1:]]
        else:
            pairs = [p for p in itertools.combinations(comp, 2) if rnd.random() < 0.7] or [tuple(comp[:2])]
        missing.update((min(a, b), max(a, b)) for a, b in pairs)
    if rnd.random() < 0.2 and n > 3:  # occasionally a node the kernel must decline
        a, b = rnd.sample(range(n), 2)
        missing.add((min(a, b), max(a, b)))
    row = [0] * 32
    ncol = n + n_r
    for a in range(ncol):
        for b in range(ncol):
            if a != b and (min(a, b), max(a, b)) not in missing:
                row[a] |= 1 << b
    return row, (1 << n) - 1, ((1 << ncol) - 1) & ~((1 << n) - 1)


@pytest.mark.parametrize("seed", range(4))
def test_join_steps_match_brute_force(seed):
    rnd = random.Random(4242 + seed)
    decided = declined = 0
    for _ in range(150):
        n = rnd.randint(2, 14)
        row, P, RM = near_complete_node(rnd, n, rnd.randint(0, 3))
        h1 = [rnd.getrandbits(64) for _ in range(32)]
        h2 = [rnd.getrandbits(64) for _ in range(32)]
        s10, s20, rsize0 = rnd.getrandbits(64), rnd.getrandbits(64), rnd.randint(0, 6)
        got = join(row, h1, h2, P, RM, s10, s20, rsize0)
        if got is None:
            declined += 1
            continue
        assert got == brute(row, h1, h2, P, RM, s10, s20, rsize0)
        decided += 1
    assert decided > 100
