"""The Python mirror of the C structs must match the header byte for byte:
compile a probe against include/rdmce.h with the host C compiler and compare
sizes and field offsets with the ctypes definitions."""
from __future__ import annotations

import ctypes as C
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

PROBE = r"""
#include <stddef.h>
#include <stdio.h>
#include "rdmce.h"
int main(void) {
  printf("mce_options %zu %zu %zu %zu\n", sizeof(mce_options), offsetof(mce_options, stream),
         offsetof(mce_options, flags), offsetof(mce_options, reg_share_bound));
  printf("mce_result %zu %zu %zu %zu %zu\n", sizeof(mce_result), offsetof(mce_result, warp_cycles),
         offsetof(mce_result, max_item_cycles), offsetof(mce_result, phase_ms), offsetof(mce_result, hist));
  printf("mce_graph_info %zu\n", sizeof(mce_graph_info));
  printf("mce_batch_graph_result %zu\n", sizeof(mce_batch_graph_result));
  printf("mce_server_options %zu\n", sizeof(mce_server_options));
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no host C compiler")
def test_ctypes_structs_match_header(engine, tmp_path):
    src = tmp_path / "probe.c"
    src.write_text(PROBE)
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = dict(l.split(" ", 1) for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                       check=True).stdout.splitlines())
    O, R = engine.Options, engine._Result
    assert out["mce_options"].split() == [str(C.sizeof(O)), str(O.stream.offset), str(O.flags.offset),
                                          str(O.reg_share_bound.offset)]
    assert out["mce_result"].split() == [str(C.sizeof(R)), str(R.warp_cycles.offset),
                                         str(R.max_item_cycles.offset), str(R.phase_ms.offset), str(R.hist.offset)]
    assert int(out["mce_graph_info"]) == C.sizeof(engine._Info)
    assert int(out["mce_batch_graph_result"]) == C.sizeof(engine._BatchResult)
    assert int(out["mce_server_options"]) == C.sizeof(engine._ServerOptions)
