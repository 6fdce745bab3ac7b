"""COO text parsed on the GPU (ingest.cu) against the oracle's restatement of
the reference's parser (src/graph.cc:82-104: `fin >> u >> v`, the rest of the
line skipped; a failed extraction skips the line).  The oracle parser is
itself pinned to the reference build on malformed text (tests/test_oracle.py).
Output must be identical pair for pair: same records, same order."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import opts

pytestmark = pytest.mark.gpu


def same_parse(gpu, oracle_mod, path):
    ou, ov = oracle_mod.parse_text(path)
    gu, gv = gpu.parse_text(path, device=0)
    assert np.array_equal(ou, gu) and np.array_equal(ov, gv), path
    return ou, ov


CASES = {
    "malformed": "% header line\n# another\n1 2\n2 3 99 extra\n3\n4\n  5\t6\n7 8.5\nabc 9\n+10 11\n12 -13\n"
                 "99999999999 1\n14 15",
    "trailing_newline": "1 2\n3 4\n",
    "crlf": "1 2\r\n3 4\r\n\r\n5 6\r\n",
    "spill_chain": "1\n2\n3\n4\n5\n6 7\n8\n\n\n9 10 11\n",
    "spill_from_hidden_line": "1\n2 3\n4 5\n",
    "failure_after_spill": "7\nx 8\n9 10\n",
    "blank_lines": "\n\n1 2\n\n\n3 4",
    "one_token": "42",
    "only_spaces": "   \n \t \n",
    "signs": "-0 +0\n-1 2\n4294967295 4294967296\n4294967295 1\n",
    "no_final_newline_spill": "5\n",
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_small_cases(gpu, oracle_mod, tmp_path, name):
    path = str(tmp_path / f"{name}.txt")
    with open(path, "w", newline="") as f:
        f.write(CASES[name])
    same_parse(gpu, oracle_mod, path)


def test_empty_file(gpu, oracle_mod, tmp_path):
    path = str(tmp_path / "empty.txt")
    open(path, "w").close()
    u, _ = same_parse(gpu, oracle_mod, path)
    assert len(u) == 0


def random_text(rng, nbytes, long_lines):
    """Random lines: mostly `u v`, with missing / extra / signed / oversized
    tokens, junk, blank lines, CRLF, and (optionally) very long lines that
    cross the GPU's 8 KiB tiles."""
    out = []
    size = 0
    while size < nbytes:
        kind = rng.integers(0, 20)
        if kind < 10:
            line = f"{rng.integers(0, 1 << 20)} {rng.integers(0, 1 << 20)}"
        elif kind == 10:
            line = f"{rng.integers(0, 1 << 20)}"                       # spills onto the next line
        elif kind == 11:
            line = ""                                                  # blank
        elif kind == 12:
            line = f"{rng.integers(0, 99)} {rng.integers(0, 99)} {rng.integers(0, 99)} junk"
        elif kind == 13:
            line = f"-{rng.integers(0, 9)} +{rng.integers(0, 9)}"
        elif kind == 14:
            line = f"{rng.integers(1, 9)}{'9' * int(rng.integers(9, 12))} 3"  # overflow or not
        elif kind == 15:
            line = "% comment " + "x" * int(rng.integers(0, 30))
        elif kind == 16:
            line = f"{rng.integers(0, 1000)}\t\t{rng.integers(0, 1000)}\r"
        elif kind == 17 and long_lines:
            line = f"{rng.integers(0, 1000)} {rng.integers(0, 1000)} " + " 7" * int(rng.integers(2000, 9000))
        elif kind == 18:
            line = "   " + f"{rng.integers(0, 1000)}"                   # leading spaces, spills
        else:
            line = f"{rng.integers(0, 1000)} abc"
        out.append(line)
        size += len(line) + 1
    return "\n".join(out) + ("\n" if rng.integers(0, 2) else "")


@pytest.mark.parametrize("seed", range(8))
def test_random_text(gpu, oracle_mod, tmp_path, seed):
    rng = np.random.default_rng(seed)
    text = random_text(rng, int(rng.integers(1 << 10, 3 << 20)), long_lines=seed % 2 == 1)
    path = str(tmp_path / f"r{seed}.txt")
    with open(path, "w", newline="") as f:
        f.write(text)
    same_parse(gpu, oracle_mod, path)


def test_spill_across_tile_boundary(gpu, oracle_mod, tmp_path):
    """A record whose first number ends a line just before an 8 KiB tile edge
    and whose second number sits past it."""
    pad = "9 9 " + "0" * 8180 + "\n"  # one long record line
    text = pad + "17\n" + "\n" * 3 + "23 x\n1 2\n"
    path = str(tmp_path / "edge.txt")
    with open(path, "w") as f:
        f.write(text)
    same_parse(gpu, oracle_mod, path)


def test_load_file_text_equals_pairs(gpu, tmp_path):
    """mce_graph_load_file on text (GPU parse -> device build) gives the same
    ordered graph and result as the same pairs given in memory."""
    u, v = gpu.gen_rmat(15, 16, 8)
    path = str(tmp_path / "rmat15.txt")
    with open(path, "w") as f:
        f.write("% R-MAT 15\n")
        f.write("\n".join(f"{a} {b}" for a, b in zip(u.tolist(), v.tolist())))
    with gpu.Graph.load_file(path, opts(gpu)) as g1, gpu.Graph.from_coo(u, v, opts(gpu)) as g2:
        a, b = g1.export_csr(), g2.export_csr()
        assert all(np.array_equal(x, y) for x, y in zip(a, b))
        r1, r2 = g1.solve(opts(gpu)), g2.solve(opts(gpu))
    assert (r1.count, r1.checksum) == (r2.count, r2.checksum)


def test_rmat20_text_matches_host_parse(gpu, tmp_path):
    """The bench graph as 16.8M lines of text: the GPU parse equals the
    engine's host parse and the generator's pairs."""
    u, v = gpu.gen_rmat(20, 16, 2)
    path = str(tmp_path / "rmat20.txt")
    with open(path, "w") as f:
        for i in range(0, len(u), 1 << 20):
            f.write("\n".join(f"{a} {b}" for a, b in zip(u[i:i + (1 << 20)].tolist(), v[i:i + (1 << 20)].tolist())))
            f.write("\n")
    gu, gv = gpu.parse_text(path, device=0)
    assert np.array_equal(gu, u) and np.array_equal(gv, v)
    hu, hv = gpu.parse_text(path)
    assert np.array_equal(hu, gu) and np.array_equal(hv, gv)
    os.unlink(path)
