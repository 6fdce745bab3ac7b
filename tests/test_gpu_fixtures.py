"""GPU parity against the sampled-root fixtures (tests/golden/samples).

These pin the bench's workloads, which are too large to re-enumerate on the
CPU at test time: the fixtures hold the CPU oracle's answers, generated by
tests/golden/make_samples.py with the oracle ordering each graph by its
restatement of the engine's round-synchronous peel.  A test first checks that
the engine built the same ordered CSR (so root ids agree), then compares
totals, the clique-size histogram and per-root values bit-exactly.
"""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np
import pytest

from conftest import ROOT, opts

pytestmark = pytest.mark.gpu

SAMPLES = os.path.join(ROOT, "tests", "golden", "samples")
THREADS = max(1, min(32, os.cpu_count() or 1))
# roots with at most this many cliques are also compared one by one (per-root
# mode keeps each root on one warp, so the huge ones are compared in total only)
PER_ROOT_MAX = 10_000_000


def load(name):
    path = os.path.join(SAMPLES, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not generated")
    with open(path) as f:
        return json.load(f)


def digest(off, adj, lab):
    h = hashlib.sha256()
    for a in (off, adj, lab):
        h.update(np.ascontiguousarray(a, dtype="<u4").tobytes())
    return h.hexdigest()


def check_sample(gpu, g, fx, **kw):
    info = g.info()
    assert (info["num_vertices"], info["num_edges"], info["degeneracy"], info["max_degree"]) == (
        fx["n"], fx["m"], fx["degeneracy"], fx["max_degree"])
    assert digest(*g.export_csr()) == fx["csr_sha256"]
    roots = np.array(fx["roots"], np.uint64)
    r = g.solve_root_list(roots, opts(gpu, **kw))
    assert r.count == fx["count"]
    assert f"{r.checksum:016x}" == fx["checksum"]
    assert {str(k): c for k, c in r.hist.items()} == fx["hist"]
    assert r.max_size == fx["max_size"]
    keep = np.array([c <= PER_ROOT_MAX for c in fx["counts"]])
    cnt, chk = g.solve_roots(roots[keep], opts(gpu, **kw))
    assert [int(x) for x in cnt] == [c for c, k in zip(fx["counts"], keep) if k]
    assert [f"{int(x):016x}" for x in chk] == [c for c, k in zip(fx["checksums"], keep) if k]
    return r


def test_rmat20_headline_sample(gpu):
    """The bench's headline: all maximal cliques under 256 seeded edge roots of
    R-MAT scale 20 (5,883,333,390 cliques), with and without task sharing."""
    fx = load("rmat20_sample.json")
    c = fx["graph"]
    u, v = gpu.gen_rmat(c["scale"], c["edge_factor"], c["seed"])
    with gpu.Graph.from_coo(u, v, opts(gpu)) as g:
        check_sample(gpu, g, fx)
        r = g.solve_root_list(np.array(fx["roots"], np.uint64), opts(gpu, expand_r=0))
        assert (r.count, f"{r.checksum:016x}") == (fx["count"], fx["checksum"])


def test_rmat24_planted_sample(gpu):
    """R-MAT scale 24, edge factor 32, with 256 planted cliques of 40-200
    vertices: roots stratified by candidate-set size up to the degeneracy."""
    fx = load("rmat24_sample.json")
    c = fx["graph"]
    u, v = gpu.gen_rmat(c["scale"], c["edge_factor"], c["seed"])
    pu, pv = gpu.gen_planted(1 << c["scale"], c["planted"], c["planted_lo"], c["planted_hi"], c["planted_seed"])
    u, v = np.concatenate([u, pu]), np.concatenate([v, pv])
    with gpu.Graph.from_coo(u, v, opts(gpu)) as g:
        del u, v, pu, pv
        check_sample(gpu, g, fx)


def graphs_for_order_check(engine):
    yield "rmat12", engine.gen_rmat(12, 16, 3)
    yield "rmat14", engine.gen_rmat(14, 16, 1)
    yield "rmat16", engine.gen_rmat(16, 16, 1)
    yield "chung_lu", engine.gen_chung_lu(10000, 16, 2.5, 1)
    u, v = engine.gen_planted(3000, 20, 10, 60, 4)
    u2, v2 = engine.gen_gnp(3000, 12, 5)
    yield "planted", (np.concatenate([u, u2]), np.concatenate([v, v2]))
    u, v = engine.gen_rmat(13, 8, 9)
    yield "sparse_labels", (u * np.uint32(9973) + np.uint32(3), v * np.uint32(9973) + np.uint32(3))


@pytest.mark.parametrize("name", ["rmat12", "rmat14", "rmat16", "chung_lu", "planted", "sparse_labels"])
def test_engine_order_equals_oracle_restatement(gpu, oracle_mod, name):
    """The engine's ordered CSR is exactly the oracle's restatement of its
    round-synchronous peel: root ids mean the same edges on both sides."""
    u, v = dict(graphs_for_order_check(gpu))[name]
    og = oracle_mod.Graph.from_pairs(u, v).sort_gpu_rounds()
    with gpu.Graph.from_coo(u, v, opts(gpu)) as g:
        ro, ci, lab = g.export_csr()
        assert g.info()["degeneracy"] == og.degeneracy
    off, adj, olab = og.export()
    assert np.array_equal(ro.astype(np.uint64), off)
    assert np.array_equal(ci, adj)
    assert np.array_equal(lab, olab)


def test_batch_all_members_match_fixture(gpu):
    """All 10,000 many-instance members (G(n,p) + planted cliques, seed
    1000 + index) in one captured launch, each against the oracle: count,
    checksum, largest clique and histogram (sizes >= 63 in the last bin)."""
    path = os.path.join(SAMPLES, "batch_members.npz")
    if not os.path.exists(path):
        pytest.skip("batch_members.npz not generated")
    fx = np.load(path)
    n = len(fx["count"])
    graphs = [gpu.gen_batch_member(i)[:2] for i in range(n)]
    b = gpu.Batch(graphs, opts(gpu))
    try:
        res, hist, _ = b.solve(opts(gpu), hist_len=fx["hist"].shape[1])
    finally:
        b.close()
    assert np.array_equal(np.array([r["count"] for r in res], np.uint64), fx["count"])
    assert np.array_equal(np.array([r["checksum"] for r in res], np.uint64), fx["checksum"])
    assert np.array_equal(np.array([r["max_size"] for r in res], np.uint32), fx["max_size"])
    assert np.array_equal(np.asarray(hist, np.uint64), fx["hist"])


def test_served_requests_match_fixture(gpu):
    """The serving loop's 200 requests (R-MAT, scale 10-13, edge factor 8-32),
    submitted back to back so they share the device, each against the oracle."""
    fx = load("serve_requests.json")["requests"]
    s = gpu.Server(device=0)
    try:
        ids = [s.submit(*gpu.gen_rmat(q["scale"], q["edge_factor"], q["seed"])) for q in fx]
        s.drain()
        got = [s.poll(i)[0] for i in ids]
    finally:
        s.close()
    for q, r in zip(fx, got):
        assert (r.count, f"{r.checksum:016x}", r.max_size) == (q["count"], q["checksum"], q["max_size"]), q
