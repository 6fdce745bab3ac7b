"""GPU parity: the CUDA path through the C ABI against the CPU oracle and the
golden fixtures.  Integer results are compared bit-exactly: clique count,
clique-size histogram, order-independent checksum, largest clique, degeneracy.

Coverage follows the reference's own checks (RDMCE scripts/analyze.sh compares
the "MC numbers" line across configurations; main.cc `-o` orders): every vertex
order, task sharing on and off, EXPAND_R on and off, root ranges and root lists,
every enumeration tier boundary, and the loader's edge cases.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import edges_uv, golden_fixtures, opts

pytestmark = pytest.mark.gpu

THREADS = max(1, min(32, os.cpu_count() or 1))


def assert_same(r, o, what=""):
    assert r.count == o.count, what
    assert r.checksum == o.checksum, what
    assert r.hist == o.hist, what
    assert r.max_size == o.max_size, what


def oracle_result(oracle_mod, u, v, threads=THREADS):
    g = oracle_mod.Graph.from_pairs(u, v).sort_degeneracy()
    return g, g.mce(threads=threads)


@pytest.mark.parametrize("fx", golden_fixtures(), ids=lambda f: f["name"])
def test_golden(gpu, fx):
    u, v = edges_uv(fx)
    o = opts(gpu)
    with gpu.Graph.from_coo(u, v, o) as g:
        info = g.info()
        assert (info["num_vertices"], info["num_edges"], info["degeneracy"]) == (fx["n"], fx["m"], fx["degeneracy"])
        r = g.solve(o)
    assert r.count == fx["count"]
    assert f"{r.checksum:016x}" == fx["checksum"]
    assert {str(k): c for k, c in r.hist.items()} == fx["hist"]


def _cases(engine):
    yield "chung_lu_1e4", engine.gen_chung_lu(10000, 16, 2.5, 1)
    yield "rmat12", engine.gen_rmat(12, 16, 3)
    yield "rmat13_ef8", engine.gen_rmat(13, 8, 4)
    for s in range(3):
        yield f"gnp400_{s}", engine.gen_gnp(400, 40, 200 + s)
    u, v = engine.gen_planted(2000, 3, 100, 200, 9)
    u2, v2 = engine.gen_gnp(2000, 30, 10)
    yield "planted_wide", (np.concatenate([u, u2]), np.concatenate([v, v2]))
    u, v = engine.gen_planted(600, 8, 50, 70, 11)
    u2, v2 = engine.gen_gnp(600, 20, 12)
    yield "planted_mid", (np.concatenate([u, u2]), np.concatenate([v, v2]))


CASE_NAMES = ["chung_lu_1e4", "rmat12", "rmat13_ef8", "gnp400_0", "gnp400_1", "gnp400_2", "planted_wide",
              "planted_mid"]


@pytest.mark.parametrize("name", CASE_NAMES)
def test_against_oracle(gpu, oracle_mod, name):
    u, v = dict(_cases(gpu))[name]
    og, o = oracle_result(oracle_mod, u, v)
    with gpu.Graph.from_coo(u, v, opts(gpu)) as g:
        r = g.solve(opts(gpu))
        assert (r.num_vertices, r.num_edges, r.degeneracy, r.max_degree) == (og.n, og.m, og.degeneracy,
                                                                             og.max_degree)
    assert_same(r, o, name)


def test_rmat14_all_modes(gpu, oracle_mod):
    u, v = gpu.gen_rmat(14, 16, 1)
    _, o = oracle_result(oracle_mod, u, v)
    assert o.count == 107790386
    with gpu.Graph.from_coo(u, v, opts(gpu)) as g:
        assert_same(g.solve(opts(gpu)), o, "sharing")
        assert_same(g.solve(opts(gpu)), o, "repeat")
        assert_same(g.solve(opts(gpu, flags=gpu.FLAG_NO_SHARING)), o, "no sharing")
        assert_same(g.solve(opts(gpu, expand_r=0)), o, "no EXPAND_R")
        assert_same(g.solve(opts(gpu, share_bound=4)), o, "share bound 4")


@pytest.mark.parametrize("order", [1, 2, 3])
def test_vertex_orders(gpu, oracle_mod, order):
    u, v = gpu.gen_rmat(12, 16, 3)
    _, o = oracle_result(oracle_mod, u, v)
    with gpu.Graph.from_coo(u, v, opts(gpu, order=order)) as g:
        assert_same(g.solve(opts(gpu)), o, f"order {order}")


def test_degeneracy_order_is_valid(gpu, oracle_mod):
    u, v = gpu.gen_rmat(13, 16, 7)
    og = oracle_mod.Graph.from_pairs(u, v)
    core = og.core_numbers()
    og.sort_degeneracy()
    with gpu.Graph.from_coo(u, v, opts(gpu)) as g:
        ro, ci, lab = g.export_csr()
        k = g.info()["degeneracy"]
    assert k == int(core.max()) == og.degeneracy
    n = len(ro) - 1
    ro = ro.astype(np.int64)
    later = np.zeros(n, np.int64)
    for x in range(n):
        row = ci[ro[x]:ro[x + 1]]
        assert np.all(np.diff(row.astype(np.int64)) > 0)
        later[x] = int((row > x).sum())
    assert later.max() <= k
    _, _, olab = og.export()
    assert np.array_equal(np.sort(lab), np.sort(olab))


def test_order_is_deterministic(gpu):
    """Root ids are edges of the ordered CSR: the same input must give the same
    CSR every time, on the dense- and the sparse-label relabel paths."""
    u, v = gpu.gen_rmat(15, 16, 4)
    for uu, vv in [(u, v), (u * np.uint32(4001) + np.uint32(7), v * np.uint32(4001) + np.uint32(7))]:
        outs = []
        for _ in range(3):
            with gpu.Graph.from_coo(uu, vv, opts(gpu)) as g:
                outs.append(g.export_csr())
        for o in outs[1:]:
            assert all(np.array_equal(a, b) for a, b in zip(outs[0], o))


def test_sampled_roots_rmat16(gpu, oracle_mod):
    """Per-root counts and checksums.  Root r is the r-th edge (v0 < v1) of the
    ordered CSR; the GPU peel orders vertices within a k-core level differently
    from the reference's sequential queue, so the oracle is handed the GPU's
    ordered CSR (whose validity test_degeneracy_order_is_valid checks)."""
    u, v = gpu.gen_rmat(16, 16, 1)
    with gpu.Graph.from_coo(u, v, opts(gpu)) as g:
        ro, ci, lab = g.export_csr()
        og = oracle_mod.Graph.from_csr(ro.astype(np.uint64), ci, lab)
        rng = np.random.default_rng(7)
        roots = np.sort(rng.choice(og.m, 400, replace=False)).astype(np.uint64)
        ocnt, ochk = og.mce_roots(roots, threads=THREADS)
        light = roots[ocnt < 2_000_000]
        cnt, chk = g.solve_roots(light, opts(gpu))
        keep = ocnt < 2_000_000
        assert np.array_equal(cnt, ocnt[keep]) and np.array_equal(chk, ochk[keep])
        r = g.solve_root_list(roots, opts(gpu))
    assert r.count == int(ocnt.sum())
    assert r.checksum == int(ochk.sum(dtype=np.uint64))
    assert r.roots == len(roots)


def test_root_ranges_partition(gpu, oracle_mod):
    u, v = gpu.gen_rmat(13, 16, 2)
    _, o = oracle_result(oracle_mod, u, v)
    with gpu.Graph.from_coo(u, v, opts(gpu)) as g:
        m = g.info()["num_edges"]
        cuts = [0, m // 7, m // 2, m - 3, m]
        tot, chk = 0, 0
        hist = {}
        for a, b in zip(cuts[:-1], cuts[1:]):
            r = g.solve(opts(gpu, root_begin=a, root_end=b))
            tot += r.count
            chk = (chk + r.checksum) % (1 << 64)
            for s, c in r.hist.items():
                hist[s] = hist.get(s, 0) + c
    assert (tot, chk, hist) == (o.count, o.checksum, o.hist)


def tier_graph(p_cols, x_rows, seed=5):
    """Under the unchanged order, the root edge (x_rows, x_rows + 1) has exactly
    p_cols candidate columns and up to x_rows X rows."""
    rng = np.random.default_rng(seed)
    X = np.arange(x_rows)
    v0, v1 = x_rows, x_rows + 1
    P = np.arange(x_rows + 2, x_rows + 2 + p_cols)
    e = [(v0, v1)]
    e += [(v0, int(x)) for x in X] + [(v1, int(x)) for x in X]
    e += [(v0, int(p)) for p in P] + [(v1, int(p)) for p in P]
    for i in range(p_cols):
        for j in range(i + 1, p_cols):
            if rng.random() < 0.5:
                e.append((int(P[i]), int(P[j])))
    for x in X:
        for p in P:
            if rng.random() < 0.5:
                e.append((int(x), int(p)))
    a = np.array(e, np.uint32)
    return a[:, 0].copy(), a[:, 1].copy()


@pytest.mark.parametrize("p_cols,x_rows", [(63, 0), (64, 0), (65, 0), (64, 64), (60, 68), (60, 69), (127, 3),
                                           (128, 10), (129, 40)])
@pytest.mark.parametrize("sharing", [True, False])
def test_tier_boundaries(gpu, oracle_mod, p_cols, x_rows, sharing):
    u, v = tier_graph(p_cols, x_rows)
    _, o = oracle_result(oracle_mod, u, v)
    flags = 0 if sharing else gpu.FLAG_NO_SHARING
    with gpu.Graph.from_coo(u, v, opts(gpu, order=gpu.ORDER_UNCHANGED)) as g:
        r = g.solve(opts(gpu, flags=flags, share_bound=4))
    assert_same(r, o, f"{p_cols}x{x_rows}")


def test_edge_cases(gpu):
    o = opts(gpu)
    r = gpu.solve_coo(np.array([7], np.uint32), np.array([9], np.uint32), o)
    assert (r.count, r.hist) == (1, {2: 1})
    r = gpu.solve_coo(np.array([3, 4], np.uint32), np.array([3, 4], np.uint32), o)
    assert (r.count, r.num_vertices) == (0, 0)
    r = gpu.solve_coo(np.zeros(0, np.uint32), np.zeros(0, np.uint32), o)
    assert r.count == 0
    u = np.array([1, 2, 2, 1, 3, 3, 1], np.uint32)
    v = np.array([2, 1, 3, 3, 1, 2, 2], np.uint32)
    r = gpu.solve_coo(u, v, o)
    assert (r.count, r.hist, r.num_edges) == (1, {3: 1}, 3)


def test_bin_roundtrip(gpu, oracle_mod, tmp_path):
    u, v = gpu.gen_rmat(11, 16, 3)
    path = str(tmp_path / "g.bin")
    with gpu.Graph.from_coo(u, v, opts(gpu)) as g:
        r1 = g.solve(opts(gpu))
        g.store_bin(path)
    with gpu.Graph.load_file(path, opts(gpu)) as h:
        r2 = h.solve(opts(gpu))
    assert_same(r2, r1)
    oh = oracle_mod.Graph.load_bin(path)
    assert oh.mce(threads=THREADS).count == r1.count


def hub_pair_graph(p_cols=3000, x_rows=20000, seed=8):
    """Under the unchanged order, root (x_rows, x_rows + 1) is a hub pair with
    p_cols candidates (sparse edges among them) and x_rows X rows, each with
    one or two candidate neighbours, so no X row is dropped: an ego network of
    (p_cols + x_rows) rows x ceil(p_cols / 64) words, far beyond the default
    4 MB per-warp slab."""
    rng = np.random.default_rng(seed)
    X = np.arange(x_rows, dtype=np.int64)
    v0, v1 = x_rows, x_rows + 1
    P = np.arange(x_rows + 2, x_rows + 2 + p_cols, dtype=np.int64)
    parts = [np.array([[v0, v1]])]
    for hub in (v0, v1):
        parts.append(np.stack([np.full(x_rows, hub), X], 1))
        parts.append(np.stack([np.full(p_cols, hub), P], 1))
    a = rng.integers(0, p_cols, size=3 * p_cols)
    b = rng.integers(0, p_cols, size=3 * p_cols)
    parts.append(np.stack([P[a], P[b]], 1))
    for k in range(2):
        keep = X if k == 0 else X[rng.random(x_rows) < 0.5]
        parts.append(np.stack([keep, P[rng.integers(0, p_cols, size=len(keep))]], 1))
    e = np.concatenate(parts).astype(np.uint32)
    return e[:, 0].copy(), e[:, 1].copy()


def test_hub_root_beyond_default_slab(gpu, oracle_mod):
    """A root whose ego network exceeds the default slab is deferred to the
    large-scratch pass and solved there (never skipped), in a full solve and
    in per-root mode."""
    u, v = hub_pair_graph()
    _, o = oracle_result(oracle_mod, u, v)
    with gpu.Graph.from_coo(u, v, opts(gpu, order=gpu.ORDER_UNCHANGED)) as g:
        r = g.solve(opts(gpu))
        assert r.heavy_roots >= 1
        assert_same(r, o, "hub pair")
        ro, ci, lab = g.export_csr()
        og = oracle_mod.Graph.from_csr(ro.astype(np.uint64), ci, lab)
        m = g.info()["num_edges"]
        roots = np.unique(np.concatenate([np.arange(0, m, max(1, m // 300)), [og_root_id(og, 20000, 20001)]]))
        roots = roots.astype(np.uint64)
        ocnt, ochk = og.mce_roots(roots, threads=THREADS)
        cnt, chk = g.solve_roots(roots, opts(gpu))
    assert np.array_equal(cnt, ocnt) and np.array_equal(chk, ochk)


def og_root_id(og, a, b):
    """Root id of edge (a, b), a < b, in the CSR the oracle graph holds."""
    off, adj, _ = og.export()
    rid = 0
    for x in range(a):
        row = adj[off[x]:off[x + 1]]
        rid += int((row > x).sum())
    row = adj[off[a]:off[a + 1]]
    return rid + int(((row > a) & (row < b)).sum())


@pytest.mark.parametrize("heavy_warps", [3, 0])
def test_deferred_roots_with_small_slabs(gpu, oracle_mod, heavy_warps):
    """A 16 KiB slab cap defers every root with a wide ego network; the second
    pass runs with 3 warps (a block smaller than the normal 8-warp block, one
    slab per launched warp) or as many as memory allows.  Totals, histogram
    and per-root values must match the oracle."""
    u, v = gpu.gen_planted(600, 8, 60, 90, 11)
    u2, v2 = gpu.gen_gnp(600, 20, 12)
    u, v = np.concatenate([u, u2]), np.concatenate([v, v2])
    _, o = oracle_result(oracle_mod, u, v)
    small = dict(slab_kib=16, heavy_warps=heavy_warps)
    with gpu.Graph.from_coo(u, v, opts(gpu)) as g:
        r = g.solve(opts(gpu, **small))
        assert r.heavy_roots > 0
        assert_same(r, o, "small slabs")
        assert_same(g.solve(opts(gpu, flags=gpu.FLAG_NO_SHARING, **small)), o, "small slabs, no sharing")
        ro, ci, lab = g.export_csr()
        og = oracle_mod.Graph.from_csr(ro.astype(np.uint64), ci, lab)
        roots = np.arange(g.info()["num_edges"], dtype=np.uint64)
        ocnt, ochk = og.mce_roots(roots, threads=THREADS)
        cnt, chk = g.solve_roots(roots, opts(gpu, **small))
    assert np.array_equal(cnt, ocnt) and np.array_equal(chk, ochk)


def test_build_bytes_counter_matches_oracle(gpu, oracle_mod):
    """The engine's count of algorithmic ego-network build bytes (the
    roofline's traffic baseline, MCE_FLAG_STATS) equals the oracle's, root set
    by root set, including a full solve with deferred roots."""
    u, v = gpu.gen_rmat(15, 16, 2)
    with gpu.Graph.from_coo(u, v, opts(gpu)) as g:
        ro, ci, lab = g.export_csr()
        og = oracle_mod.Graph.from_csr(ro.astype(np.uint64), ci, lab)
        roots = np.sort(np.random.default_rng(3).choice(og.m, 500, replace=False)).astype(np.uint64)
        _, _, o = og.mce_root_set(roots, threads=THREADS)
        r = g.solve_root_list(roots, opts(gpu, flags=gpu.FLAG_STATS))
        assert (r.count, r.checksum) == (o.count, o.checksum)
        assert r.build_bytes == o.build_bytes > 0
        full = g.solve(opts(gpu, flags=gpu.FLAG_STATS, slab_kib=16))
        assert full.heavy_roots > 0
        assert full.build_bytes == og.mce(threads=THREADS).build_bytes


def test_autotuner_tries_each_build_then_keeps_one(gpu, oracle_mod):
    """blocks_per_sm = 0: the first three solves of a workload run the 4-, 5-
    and 3-blocks-per-SM builds (64, 51, 85 registers a thread), later ones the
    fastest of them; every build gives the same cliques.  An explicit setting
    is used as given."""
    u, v = gpu.gen_rmat(13, 16, 6)
    _, o = oracle_result(oracle_mod, u, v)
    with gpu.Graph.from_coo(u, v, opts(gpu)) as g:
        runs = [g.solve(opts(gpu)) for _ in range(5)]
        for r in runs:
            assert_same(r, o, f"blocks per SM {r.blocks_per_sm}")
        assert [(r.blocks_per_sm, r.autotune) for r in runs[:3]] == [(4, 1), (5, 1), (3, 1)]
        assert runs[3].autotune == runs[4].autotune == 2
        assert runs[3].blocks_per_sm == runs[4].blocks_per_sm in (3, 4, 5)
        # a different workload (a root range) is tuned on its own
        part = g.solve(opts(gpu, root_begin=0, root_end=1000))
        assert (part.blocks_per_sm, part.autotune) == (4, 1)
        for b in (1, 2, 3, 4, 5):
            r = g.solve(opts(gpu, blocks_per_sm=b))
            assert (r.blocks_per_sm, r.autotune) == (b, 0)
            assert_same(r, o, f"explicit {b}")


def test_batch_autotuner_recaptures(gpu, oracle_mod):
    graphs = [gpu.gen_batch_member(i)[:2] for i in range(40)]
    b = gpu.Batch(graphs, opts(gpu))
    try:
        outs = [b.solve(opts(gpu))[:2] for _ in range(5)]
    finally:
        b.close()
    for res, hist in outs[1:]:
        assert res == outs[0][0] and np.array_equal(hist, outs[0][1])


def test_batch_options_take_effect(gpu, oracle_mod):
    """A batch re-captures its launch when an option that feeds the plan
    changes: a one-poll wait limit on the second solve must surface as
    MCE_ERR_TIMEOUT (a stale capture would replay the first plan), and the
    third solve, back on the defaults, must be exact again."""
    graphs = [gpu.gen_batch_member(i)[:2] for i in range(200)]
    want = []
    for u, v in graphs[:20]:
        want.append(oracle_mod.Graph.from_pairs(u, v).sort_degeneracy().mce(threads=4))
    b = gpu.Batch(graphs, opts(gpu))
    try:
        first, _, _ = b.solve(opts(gpu, blocks_per_sm=4))
        with pytest.raises(gpu.MceError) as e:
            b.solve(gpu.options(blocks_per_sm=4, spin_limit=1))
        assert e.value.status == gpu.ERR_TIMEOUT
        third, _, _ = b.solve(opts(gpu, blocks_per_sm=4))
    finally:
        b.close()
    assert third == first
    for r, o in zip(third[:20], want):
        assert (r["count"], r["checksum"], r["max_size"]) == (o.count, o.checksum, o.max_size)


def near_complete_blocks(seed, blocks=40, lo=12, hi=30, extra=6):
    """Unions of near-complete blocks: each block is a clique minus the edges
    of small complement components (perfect matchings, paths of three,
    triangles, five-cycles), plus outside vertices adjacent to random parts of
    a block (rows that hold R without being candidates).  Subproblems of such
    blocks are exactly what the 32-bit tier's join decision takes, with and
    without such rows."""
    rng = np.random.default_rng(seed)
    us, vs = [], []
    base = 0
    for _ in range(blocks):
        b = int(rng.integers(lo, hi + 1))
        verts = np.arange(base, base + b)
        missing = set()
        perm = rng.permutation(b)
        i = 0
        while i < b:
            kind = int(rng.integers(0, 5))
            comp = [int(x) for x in perm[i:i + (2, 3, 3, 5, 1)[kind]]]
            i += len(comp)
            if kind == 0 and len(comp) == 2:
                missing.add((min(comp), max(comp)))
            elif kind == 1:
                for a, c in zip(comp, comp[1:]):
                    missing.add((min(a, c), max(a, c)))
            elif kind in (2, 3):
                ring = comp + comp[:1] if len(comp) > 2 else comp
                for a, c in zip(ring, ring[1:]):
                    if a != c:
                        missing.add((min(a, c), max(a, c)))
        for a in range(b):
            for c in range(a + 1, b):
                if (a, c) not in missing:
                    us.append(verts[a])
                    vs.append(verts[c])
        base += b
        for _ in range(extra):
            nbrs = verts[rng.random(b) < rng.uniform(0.3, 0.95)]
            us.extend([base] * len(nbrs))
            vs.extend(nbrs.tolist())
            base += 1
    # sparse links between blocks
    for _ in range(blocks * 3):
        a, c = rng.integers(0, base, 2)
        if a != c:
            us.append(a)
            vs.append(c)
    return np.array(us, np.uint32), np.array(vs, np.uint32)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_near_complete_blocks(gpu, oracle_mod, seed):
    u, v = near_complete_blocks(seed)
    _, o = oracle_result(oracle_mod, u, v)
    with gpu.Graph.from_coo(u, v, opts(gpu)) as g:
        for kw in ({}, {"expand_r": 0}, {"flags": gpu.FLAG_NO_SHARING}):
            r = g.solve(opts(gpu, **kw))
            assert_same(r, o, f"seed {seed} {kw}")


def test_cocktail_party(gpu, oracle_mod):
    """K(2,2,...,2) on 28 vertices: 2^14 maximal cliques of 14 vertices."""
    n = 28
    u, v = zip(*[(a, c) for a in range(n) for c in range(a + 1, n) if c != a + 1 or a % 2])
    u, v = np.array(u, np.uint32), np.array(v, np.uint32)
    _, o = oracle_result(oracle_mod, u, v)
    assert o.count == 2 ** 14 and o.hist == {14: 2 ** 14}
    with gpu.Graph.from_coo(u, v, opts(gpu)) as g:
        assert_same(g.solve(opts(gpu)), o, "cocktail party")
