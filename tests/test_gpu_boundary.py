"""The reference-facing surfaces on the GPU: the `RDMCE -i` command line and
its `-c` conversion, the `.bin` container in both directions with the
reference's own build, the C++ facade with the reference's class names, and
a bounded device wait that runs out.

The reference CLI is main.cc:13-138 (its result lines are parsed by
scripts/analyze.sh); the .bin container is src/graph.cc:154-213; the classes
are include/graph.h:12-52 and include/mce_gpu.cuh:15-24.
"""
from __future__ import annotations

import json
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, edges_uv, opts

pytestmark = pytest.mark.gpu

CLI = os.path.join(ROOT, "rdmce_b200", "bin", "RDMCE")
REF_CPU = os.path.join(ROOT, "oracle", "_ref", "ref_cpu")
needs_ref = pytest.mark.skipif(not os.path.exists(REF_CPU), reason="reference CPU build absent")


def write_coo(path, u, v):
    with open(path, "w") as f:
        f.write("% comment lines and a header are skipped, as the reference's parser does\n")
        for a, b in zip(u.tolist(), v.tolist()):
            f.write(f"{a} {b}\n")


def mc_numbers(out):
    m = re.search(r"MC numbers: (\d+)", out)
    assert m, out
    return int(m.group(1))


def cli(*args):
    r = subprocess.run([CLI, *args], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return r.stdout


def zachary(tmp_path):
    with open(os.path.join(GOLDEN, "zachary.json")) as f:
        fx = json.load(f)
    path = str(tmp_path / "zachary.txt")
    write_coo(path, *edges_uv(fx))
    return path, fx


def test_cli_zachary(gpu, tmp_path):
    path, fx = zachary(tmp_path)
    out = cli("-i", path, "-o", "deg", "-d", "0")
    assert mc_numbers(out) == fx["count"] == 36
    assert re.search(r"MCE GPU Time: [0-9.e+-]+", out)
    assert f"MC checksum: 0x{fx['checksum']}" in out


@pytest.mark.parametrize("order", ["a", "d", "unchange"])
def test_cli_orders(gpu, tmp_path, order):
    path, fx = zachary(tmp_path)
    assert mc_numbers(cli("-i", path, "-o", order)) == fx["count"]


@needs_ref
def test_engine_bin_read_by_reference(gpu, oracle_mod, tmp_path):
    """`RDMCE -i g.txt -c` writes g.bin; the engine and the reference's own
    loader (Graph::LoadFromBin, through oracle/_ref/ref_cpu) read it back and
    count the same cliques."""
    u, v = gpu.gen_rmat(11, 16, 5)
    txt = str(tmp_path / "g.txt")
    write_coo(txt, u, v)
    cli("-i", txt, "-c")
    binp = str(tmp_path / "g.bin")
    assert os.path.exists(binp)
    ours = mc_numbers(cli("-i", binp))
    ref = oracle_mod.run_ref_cpu("count", binp)["count"]
    expect = oracle_mod.Graph.from_pairs(u, v).sort_degeneracy().mce(threads=4).count
    assert ours == ref == expect


@needs_ref
def test_reference_bin_read_by_engine(gpu, oracle_mod, tmp_path):
    """The reference's own Graph::StoreIntoBin output (degeneracy-sorted by
    the reference) loads into the engine in stored order, through the CLI and
    through mce_graph_load_file, with the reference's count and CSR."""
    u, v = gpu.gen_rmat(11, 16, 6)
    txt = str(tmp_path / "r.txt")
    write_coo(txt, u, v)
    subprocess.run([REF_CPU, "storebin", txt, str(tmp_path / "r.txt")], check=True, capture_output=True, timeout=300)
    binp = str(tmp_path / "r.bin")
    assert os.path.exists(binp)
    ref = oracle_mod.run_ref_cpu("count", binp)["count"]
    assert mc_numbers(cli("-i", binp)) == ref
    with gpu.Graph.load_file(binp, opts(gpu)) as g:
        r = g.solve(opts(gpu))
        ro, ci, lab = g.export_csr()
    assert r.count == ref
    oh = oracle_mod.Graph.load_bin(binp)
    off, adj, olab = oh.export()
    assert np.array_equal(ro.astype(np.uint64), off) and np.array_equal(ci, adj) and np.array_equal(lab, olab)


def test_cpp_facade(gpu, tmp_path):
    """A C++ program written against the reference's class names (Graph,
    MceGpuSolver, StoreIntoBin/LoadFromBin, ConvertToCsr) compiles against the
    facade and gets the right answers."""
    path, fx = zachary(tmp_path)
    exe = str(tmp_path / "facade_check")
    csrc = os.path.join(ROOT, "rdmce_b200", "csrc")
    subprocess.run(["g++", "-O1", "-std=c++17", f"-I{csrc}", f"-I{os.path.join(ROOT, 'include')}",
                    os.path.join(ROOT, "tests", "cpp", "facade_check.cc"), os.path.join(csrc, "rdmce_graph.cc"),
                    f"-L{os.path.join(ROOT, 'rdmce_b200')}", "-lrdmce",
                    f"-Wl,-rpath,{os.path.join(ROOT, 'rdmce_b200')}", "-lpthread", "-o", exe],
                   check=True, capture_output=True, timeout=300)
    r = subprocess.run([exe, path, str(tmp_path), str(fx["count"])], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert f"FACADE OK count {fx['count']} checksum {fx['checksum']}" in r.stdout


def test_wait_limit_runs_out_then_device_is_usable(gpu, oracle_mod):
    """Every device-side wait is bounded.  With a limit of one poll, warps that
    run out of roots while others are still busy give up at once: the solve
    returns MCE_ERR_TIMEOUT instead of stalling, and the same device then
    solves correctly."""
    u, v = gpu.gen_rmat(13, 16, 3)
    expect = oracle_mod.Graph.from_pairs(u, v).sort_degeneracy().mce(threads=8)
    with gpu.Graph.from_coo(u, v, opts(gpu)) as g:
        with pytest.raises(gpu.MceError) as e:
            g.solve(gpu.options(spin_limit=1))
        assert e.value.status == gpu.ERR_TIMEOUT
        r = g.solve(opts(gpu))
    assert (r.count, r.checksum) == (expect.count, expect.checksum)
