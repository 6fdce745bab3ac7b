"""Host-side checks of the C ABI that need no GPU: exported symbols, status
strings, the generators that define the synthetic workloads, the text parser,
argument validation and the CLI's usage errors."""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "rdmce.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    names = re.findall(r"^[A-Za-z_][\w \*]*?\b(mce_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_header_function(engine):
    names = header_functions()
    assert len(names) >= 30
    L = C.CDLL(engine.LIB_PATH)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_python_binding_covers_header(engine):
    assert set(header_functions()) <= set(engine._SIGS)


def test_status_strings(engine):
    texts = [engine.status_str(s) for s in range(13)]
    assert all(texts) and len(set(texts)) == 13
    assert "unknown status" not in texts
    assert engine.status_str(99) == "unknown status"


def test_mix64_matches_oracle(engine, oracle_mod):
    for x in [0, 1, 2**63, 0x9E3779B97F4A7C15, 123456789]:
        assert engine.mix64(x) == oracle_mod.mix64(x)


def test_rmat_deterministic_and_thread_invariant(engine):
    a = engine.gen_rmat(12, 8, 5, threads=1)
    b = engine.gen_rmat(12, 8, 5, threads=4)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    c = engine.gen_rmat(12, 8, 6)
    assert not np.array_equal(a[0], c[0])
    assert len(a[0]) == 8 << 12 and a[0].max() < 4096 and a[1].max() < 4096


def test_rmat_quadrant_skew(engine):
    u, v = engine.gen_rmat(14, 8, 1)
    top = (u < (1 << 13)) & (v < (1 << 13))
    assert 0.55 <= top.mean() <= 0.59  # a = 0.57 at the first level


def test_chung_lu_shape(engine):
    u, v = engine.gen_chung_lu(10000, 16, 2.5, 1)
    assert len(u) == 80000
    verts = np.unique(np.concatenate([u, v]))
    assert 9900 <= len(verts) <= 10000
    keep = u != v
    deg = 2.0 * keep.sum() / 10000
    assert 14 <= deg <= 17


def test_batch_member_shapes(engine):
    ns = []
    for i in range(40):
        u, v, n = engine.gen_batch_member(i)
        assert 64 <= n <= 4096
        assert len(u) == len(v) and (len(u) == 0 or max(u.max(), v.max()) < n)
        ns.append(n)
    assert max(ns) > 4 * min(ns)  # log-uniform sizes spread over the range


def test_planted_cliques_present(engine, oracle_mod):
    u, v = engine.gen_planted(300, 2, 30, 30, 3)
    g = oracle_mod.Graph.from_pairs(u, v).sort_degeneracy()
    r = g.mce()
    assert r.hist.get(30, 0) >= 1


def test_parse_text_matches_oracle(engine, oracle_mod, tmp_path):
    path = str(tmp_path / "g.txt")
    with open(path, "w") as f:
        f.write("% c\n1 2\n3 4 5\n\n7\t8\nx 9\n10 11")
    a = engine.parse_text(path)
    b = oracle_mod.parse_text(path)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert a[0].tolist() == [1, 3, 7, 10]


def test_missing_file_is_io_error(engine):
    with pytest.raises(engine.MceError) as e:
        engine.parse_text("/nonexistent/file.txt")
    assert e.value.status == engine.ERR_IO


def test_no_device_status(engine):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(engine.MceError) as e:
        engine.Graph.from_coo(np.array([0], np.uint32), np.array([1], np.uint32))
    assert e.value.status == engine.ERR_NO_DEVICE


def test_invalid_arguments_and_capacity(engine):
    L = engine.lib()
    h = C.c_void_p()
    assert L.mce_graph_from_coo(None, None, 5, None, C.byref(h)) == engine.ERR_INVALID_ARG
    assert L.mce_graph_from_coo(None, None, 0, None, None) == engine.ERR_INVALID_ARG
    cnt = C.c_uint64()
    u = np.empty(4, np.uint32)
    v = np.empty(4, np.uint32)
    s = L.mce_gen_gnp(100, 10.0, 1, engine._ptr(u), engine._ptr(v), 4, C.byref(cnt))
    assert s == engine.ERR_CAPACITY and cnt.value > 4
    assert L.mce_gen_chung_lu(1, 16.0, 2.5, 1, None, None, 0, C.byref(cnt), 0) == engine.ERR_INVALID_ARG
    assert L.mce_gen_planted(10, 1, 5, 4, 1, None, None, 0, C.byref(cnt)) == engine.ERR_INVALID_ARG
    assert L.mce_probe_int_peak(0, None) == engine.ERR_INVALID_ARG


def test_cli_usage_errors(engine):
    if not os.path.exists(engine.CLI_PATH):
        pytest.skip("CLI not built")
    r = subprocess.run([engine.CLI_PATH], capture_output=True, text=True)
    assert r.returncode == 1 and "Usage" in r.stderr
    r = subprocess.run([engine.CLI_PATH, "-i", "x.txt", "-o", "bogus"], capture_output=True, text=True)
    assert r.returncode == 1 and "Usage" in r.stderr


@pytest.mark.parametrize("kind", ["one_per_line", "mixed"])
def test_parallel_parse_matches_sequential_oracle(engine, oracle_mod, tmp_path, kind):
    """Files of several MB are parsed in parallel chunks; records that run
    across a chunk cut (a lone number takes its partner from the next line)
    must come out exactly as a sequential parse gives them."""
    rng = np.random.default_rng(7)
    path = str(tmp_path / "big.txt")
    with open(path, "w") as f:
        if kind == "one_per_line":
            f.write("\n".join(str(x) for x in rng.integers(0, 1 << 20, size=2_500_001)))
        else:
            lines = []
            for _ in range(900_000):
                r = rng.random()
                a, b = rng.integers(0, 1 << 20, size=2)
                if r < 0.7:
                    lines.append(f"{a} {b}")
                elif r < 0.8:
                    lines.append(f"{a}")
                elif r < 0.85:
                    lines.append("% comment")
                elif r < 0.9:
                    lines.append("")
                else:
                    lines.append(f"{a}\t{b} extra tokens 5 6")
            f.write("\n".join(lines))
    assert os.path.getsize(path) > 8 << 20
    a = engine.parse_text(path)
    b = oracle_mod.parse_text(path)
    assert len(a[0]) > 100_000
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_bin_reader_rejects_damaged_files(engine, oracle_mod, tmp_path):
    """The .bin reader (the reference container) checks its input before any
    device work: truncated, inconsistent or oversized headers are FORMAT /
    TOO_LARGE errors, a missing file an IO error."""
    u, v = engine.gen_rmat(8, 8, 3)
    g = oracle_mod.Graph.from_pairs(u, v).sort_degeneracy()
    good = tmp_path / "g.bin"
    g.store_bin(str(good))
    raw = good.read_bytes()
    L = engine.lib()
    h = C.c_void_p()

    def load(data, name):
        path = tmp_path / name
        path.write_bytes(data)
        return L.mce_graph_load_file(str(path).encode(), None, C.byref(h))

    assert load(raw[:20], "short.bin") == engine.ERR_FORMAT           # header cut
    assert load(raw[: len(raw) // 2], "half.bin") == engine.ERR_FORMAT  # adjacency cut
    big = bytearray(raw)
    big[8:16] = (1 << 31).to_bytes(8, "little")  # m with 2m >= 2^32
    assert load(bytes(big), "big.bin") == engine.ERR_TOO_LARGE
    assert L.mce_graph_load_file(str(tmp_path / "missing.bin").encode(), None, C.byref(h)) == engine.ERR_IO
