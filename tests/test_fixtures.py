"""The sampled-root fixtures (tests/golden/samples), pinned on the CPU.

The bench's headline sample (all maximal cliques under 256 seeded edge roots of
R-MAT scale 20) is far too large to re-enumerate here in full, so these tests
check what can be checked in seconds: the oracle still orders the graph into
the CSR the fixture's digest names (its restatement of the engine's
round-synchronous peel), the oracle reproduces the fixture's light roots root
by root, and -- where the reference build exists -- so does the reference's
own solver on the same edge roots of the same ordered graph.  The GPU side is
checked against the same fixture in tests/test_gpu_fixtures.py and by bench.py.
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT

SAMPLES = os.path.join(ROOT, "tests", "golden", "samples")
REF_CPU = os.path.join(ROOT, "oracle", "_ref", "ref_cpu")
LIGHT = 10_000_000


def load(name):
    with open(os.path.join(SAMPLES, name)) as f:
        return json.load(f)


def digest(off, adj, lab):
    h = hashlib.sha256()
    for a in (off, adj, lab):
        h.update(np.ascontiguousarray(a, dtype="<u4").tobytes())
    return h.hexdigest()


@pytest.fixture(scope="module")
def rmat20(oracle_mod, engine):
    fx = load("rmat20_sample.json")
    c = fx["graph"]
    u, v = engine.gen_rmat(c["scale"], c["edge_factor"], c["seed"])
    g = oracle_mod.Graph.from_pairs(u, v).sort_gpu_rounds()
    return fx, g


def test_rmat20_fixture_is_self_consistent():
    fx = load("rmat20_sample.json")
    assert len(fx["roots"]) == len(fx["counts"]) == len(fx["checksums"]) == 256
    assert sum(fx["counts"]) == fx["count"]
    assert sum(int(c, 16) for c in fx["checksums"]) % (1 << 64) == int(fx["checksum"], 16)
    assert sum(fx["hist"].values()) == fx["count"]
    assert max(int(k) for k in fx["hist"]) == fx["max_size"]
    rng = np.random.default_rng(fx["sample_seed"])
    assert list(np.sort(rng.choice(fx["m"], size=256, replace=False))) == fx["roots"]


def test_oracle_orders_rmat20_like_the_fixture(rmat20):
    fx, g = rmat20
    assert (g.n, g.m, g.degeneracy, g.max_degree) == (fx["n"], fx["m"], fx["degeneracy"], fx["max_degree"])
    off, adj, lab = g.export()
    assert digest(off, adj, lab) == fx["csr_sha256"]


def test_oracle_light_roots_match_fixture(rmat20):
    fx, g = rmat20
    light = [(r, c, h) for r, c, h in zip(fx["roots"], fx["counts"], fx["checksums"]) if c < LIGHT]
    roots = np.array([r for r, _, _ in light], np.uint64)
    cnt, chk = g.mce_roots(roots, threads=os.cpu_count() or 1)
    assert [int(x) for x in cnt] == [c for _, c, _ in light]
    assert [f"{int(x):016x}" for x in chk] == [h for _, _, h in light]


@pytest.mark.skipif(not os.path.exists(REF_CPU), reason="reference CPU build absent")
def test_reference_edge_roots_match_fixture(tmp_path):
    """The reference's own solver (BKFixedMemPivotBit2 from R = {v0, v1}) on
    the light sample roots of the engine-ordered graph, loaded from a .bin."""
    fx = load("rmat20_sample.json")
    binp = str(tmp_path / "rmat20.bin")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "oracle", "ordered_bin.py"), "rmat20", binp],
                         capture_output=True, text=True, check=True, timeout=600)
    assert fx["csr_sha256"] in out.stdout
    light = [(r, c) for r, c in zip(fx["roots"], fx["counts"]) if c < LIGHT]
    rf = tmp_path / "roots.txt"
    rf.write_text("\n".join(str(r) for r, _ in light))
    res = subprocess.run([REF_CPU, "edge_roots", binp, str(os.cpu_count() or 1), str(rf)], capture_output=True,
                         text=True, check=True, timeout=600)
    got = {int(p[1]): int(p[2]) for p in (ln.split() for ln in res.stdout.splitlines()) if p[:1] == ["ROOT"]}
    assert all(got[r] == c for r, c in light)


def test_gpu_round_order_is_a_degeneracy_order(oracle_mod, engine):
    for scale, seed in [(10, 7), (13, 7)]:
        u, v = engine.gen_rmat(scale, 16, seed)
        g = oracle_mod.Graph.from_pairs(u, v)
        core = g.core_numbers()
        ref = oracle_mod.Graph.from_pairs(u, v).sort_degeneracy()
        g.sort_gpu_rounds()
        off, adj, _ = g.export()
        later = max(int((adj[off[x]:off[x + 1]] > x).sum()) for x in range(g.n))
        assert g.degeneracy == ref.degeneracy == int(core.max()) == later
        a, b = g.mce(threads=4), ref.mce(threads=4)
        assert (a.count, a.checksum, a.hist) == (b.count, b.checksum, b.hist)


def test_gpu_round_order_by_hand(oracle_mod):
    """Path 0-1-2-3 plus triangle 3-4-5: level 1 claims 0 in its first round,
    then 1 (its degree fell to 1), then 2; the next level (k = 2) claims the
    triangle at once, in id order."""
    u = np.array([0, 1, 2, 3, 4, 5], np.uint32)
    v = np.array([1, 2, 3, 4, 5, 3], np.uint32)
    g = oracle_mod.Graph.from_pairs(u, v).sort_gpu_rounds()
    _, _, lab = g.export()
    assert list(lab) == [0, 1, 2, 3, 4, 5]
    assert g.degeneracy == 2
    u = np.array([5, 5, 5, 1], np.uint32)  # star centred on 5 plus edge 1-2... and 1-5
    v = np.array([1, 2, 3, 2], np.uint32)
    g = oracle_mod.Graph.from_pairs(u, v).sort_gpu_rounds()
    _, _, lab = g.export()
    # degree 1: vertex 3 first; then 5 has degree 2 -> next level k = 2 claims 1, 2, 5 at once
    assert list(lab) == [3, 1, 2, 5]
