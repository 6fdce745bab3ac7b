"""The CPU oracle, pinned against the reference's own CPU code and golden fixtures.

oracle/_ref/ref_cpu is the unmodified reference (RDMCE src/graph.cc, src/mce.cc,
src/common.cu) compiled by oracle/Makefile with a driver of ours; these tests
check that the oracle's loader, degeneracy value and clique count agree with it,
and that count, histogram and checksum agree with networkx's find_cliques
fixtures (tests/golden, made by tests/golden/make_golden.py).
"""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

from conftest import ROOT, edges_uv, golden_fixtures

REF_CPU = os.path.join(ROOT, "oracle", "_ref", "ref_cpu")
needs_ref = pytest.mark.skipif(not os.path.exists(REF_CPU), reason="reference CPU build absent")


def write_coo(path, u, v, header=False):
    with open(path, "w") as f:
        if header:
            f.write("% generated\n% n m\n")
        for a, b in zip(u.tolist(), v.tolist()):
            f.write(f"{a} {b}\n")


@pytest.mark.parametrize("fx", golden_fixtures(), ids=lambda f: f["name"])
def test_oracle_matches_golden(oracle_mod, fx):
    u, v = edges_uv(fx)
    g = oracle_mod.Graph.from_pairs(u, v)
    assert (g.n, g.m) == (fx["n"], fx["m"])
    g.sort_degeneracy()
    assert g.degeneracy == fx["degeneracy"]
    for threads, expand in [(1, True), (3, True), (2, False)]:
        r = g.mce(threads=threads, expand_r=expand)
        assert r.count == fx["count"]
        assert f"{r.checksum:016x}" == fx["checksum"]
        assert {str(k): v for k, v in r.hist.items()} == fx["hist"]


def test_clique_hash_is_order_independent(oracle_mod):
    a = oracle_mod.clique_hash([5, 1, 9, 1000])
    assert a == oracle_mod.clique_hash([1000, 9, 5, 1])
    assert a != oracle_mod.clique_hash([5, 1, 9])


@needs_ref
def test_oracle_matches_reference_on_zachary(oracle_mod, tmp_path):
    with open(os.path.join(ROOT, "tests", "golden", "zachary.json")) as f:
        fx = json.load(f)
    u, v = edges_uv(fx)
    path = str(tmp_path / "zachary.txt")
    write_coo(path, u, v, header=True)
    ref = oracle_mod.run_ref_cpu("count", path)
    st = oracle_mod.run_ref_cpu("stats", path)
    g = oracle_mod.Graph.from_text(path).sort_degeneracy()
    assert ref["count"] == g.mce().count == 36
    assert (st["n"], st["m"], st["max_degree"], st["degeneracy"]) == (g.n, g.m, g.max_degree, g.degeneracy)


def _graphs(engine):
    yield "chung_lu_1e4", engine.gen_chung_lu(10000, 16, 2.5, 1)
    yield "rmat10_ef8", engine.gen_rmat(10, 8, 4)
    yield "rmat11_ef16", engine.gen_rmat(11, 16, 5)
    for s in range(3):
        yield f"gnp300_{s}", engine.gen_gnp(300, 25, 100 + s)
    u, v = engine.gen_planted(400, 4, 20, 60, 7)
    u2, v2 = engine.gen_gnp(400, 12, 8)
    yield "planted", (np.concatenate([u, u2]), np.concatenate([v, v2]))


@needs_ref
def test_oracle_matches_reference_counts(oracle_mod, engine, tmp_path):
    """Loader, degeneracy value and clique count vs. the reference's MceSolver."""
    for name, (u, v) in _graphs(engine):
        path = str(tmp_path / f"{name}.txt")
        write_coo(path, u, v)
        st = oracle_mod.run_ref_cpu("stats", path)
        ref = oracle_mod.run_ref_cpu("count", path)
        g = oracle_mod.Graph.from_text(path)
        assert (st["n"], st["m"], st["max_degree"]) == (g.n, g.m, g.max_degree), name
        g.sort_degeneracy()
        assert st["degeneracy"] == g.degeneracy, name
        assert ref["count"] == g.mce(threads=4).count, name


@needs_ref
def test_oracle_order_matches_reference_exactly(oracle_mod, engine, tmp_path):
    """SortByDegeneracy + ApplyOrder restated: identical CSR and labels."""
    u, v = engine.gen_rmat(10, 8, 9)
    path = str(tmp_path / "g.txt")
    write_coo(path, u, v)
    dump = str(tmp_path / "g.csr")
    oracle_mod.subprocess.run([oracle_mod.REF_CPU, "csr", path, dump], check=True, capture_output=True)
    raw = np.fromfile(dump, dtype=np.uint8)
    n, m = np.frombuffer(raw[:16].tobytes(), dtype=np.uint64)
    off = np.frombuffer(raw[16:16 + 4 * (n + 1)].tobytes(), dtype=np.uint32)
    adj = np.frombuffer(raw[16 + 4 * (n + 1):16 + 4 * (n + 1) + 8 * m].tobytes(), dtype=np.uint32)
    lab = np.frombuffer(raw[16 + 4 * (n + 1) + 8 * m:].tobytes(), dtype=np.uint32)
    g = oracle_mod.Graph.from_text(path).sort_degeneracy()
    o_off, o_adj, o_lab = g.export()
    assert np.array_equal(o_off.astype(np.uint32), off)
    assert np.array_equal(o_adj, adj)
    assert np.array_equal(o_lab, lab)


@needs_ref
def test_parse_matches_reference_on_malformed_text(oracle_mod, engine, tmp_path):
    """Bad lines, extra columns, headers, signs, overflow, a split record."""
    text = ("% header line\n# another\n1 2\n2 3 99 extra\n3\n4\n  5\t6\n7 8.5\nabc 9\n"
            "+10 11\n12 -13\n99999999999 1\n14 15")
    path = str(tmp_path / "bad.txt")
    with open(path, "w") as f:
        f.write(text)
    ou, ov = oracle_mod.parse_text(path)
    eu, ev = engine.parse_text(path)
    assert np.array_equal(ou, eu) and np.array_equal(ov, ev)
    st = oracle_mod.run_ref_cpu("stats", path)
    g = oracle_mod.Graph.from_pairs(ou, ov)
    assert (st["n"], st["m"]) == (g.n, g.m)


def test_bin_roundtrip(oracle_mod, engine, tmp_path):
    u, v = engine.gen_rmat(9, 8, 3)
    g = oracle_mod.Graph.from_pairs(u, v).sort_degeneracy()
    path = str(tmp_path / "g.bin")
    g.store_bin(path)
    h = oracle_mod.Graph.load_bin(path)
    a, b = g.export(), h.export()
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    assert h.degeneracy == g.degeneracy
    assert h.mce().count == g.mce().count


def test_per_root_sums_to_total(oracle_mod, engine):
    u, v = engine.gen_rmat(10, 16, 2)
    g = oracle_mod.Graph.from_pairs(u, v).sort_degeneracy()
    total = g.mce(threads=2)
    cnt, chk = g.mce_roots(np.arange(g.m), threads=2)
    assert int(cnt.sum()) == total.count
    assert int(chk.sum(dtype=np.uint64)) == total.checksum
