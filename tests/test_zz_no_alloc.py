"""mce_csr_offsets_static: the allocation-free CSR row-offset scan, called
through the C ABI and compared with the engine's own graph builder (whose
offsets come from the allocating scan) and with a host prefix sum.

This file is collected last on purpose: it has to pass on its own and after
every other GPU test has run in the same process.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import opts

pytestmark = pytest.mark.gpu

MAX_N = 1 << 26


def _offsets(engine, deg_t, off_t, n, stream):
    return engine.lib().mce_csr_offsets_static(0, C.c_void_p(deg_t.data_ptr()), C.c_void_p(off_t.data_ptr()), n,
                                                C.c_void_p(stream.cuda_stream))


def _builder_offsets(engine, scale, seed):
    u, v = engine.gen_rmat(scale, 16, seed)
    with engine.Graph.from_coo(u, v, opts(engine)) as g:
        ro, _, _ = g.export_csr()
    return ro


def test_matches_graph_builder_two_calls_in_a_row(gpu):
    import torch

    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    ros = [_builder_offsets(gpu, 16, 3), _builder_offsets(gpu, 12, 5)]
    degs = [torch.from_numpy(np.diff(ro.astype(np.int64)).astype(np.int32)).to(dev) for ro in ros]
    outs = [torch.full((len(ro),), -1, dtype=torch.int32, device=dev) for ro in ros]
    # two calls back to back on one stream, no wait in between
    for d, o in zip(degs, outs):
        assert _offsets(gpu, d, o, d.numel(), stream) == gpu.OK
    stream.synchronize()
    for ro, o in zip(ros, outs):
        assert np.array_equal(o.cpu().numpy().view(np.uint32), ro)
    # and again, with the outputs poisoned, to show no state carries over
    for o in outs:
        o.fill_(-1)
    for d, o in zip(reversed(degs), reversed(outs)):
        assert _offsets(gpu, d, o, d.numel(), stream) == gpu.OK
    stream.synchronize()
    for ro, o in zip(ros, outs):
        assert np.array_equal(o.cpu().numpy().view(np.uint32), ro)


@pytest.mark.parametrize("n", [0, 1, 2047, 2048, 2049, 2048 * 2048, 2048 * 2048 + 1, 5_000_000, MAX_N])
def test_every_scan_depth(gpu, n):
    import torch

    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    rng = np.random.default_rng(n)
    deg = rng.integers(0, 64, size=n, dtype=np.uint32)
    deg_t = torch.from_numpy(deg.view(np.int32)).to(dev) if n else torch.zeros(1, dtype=torch.int32, device=dev)
    off_t = torch.full((n + 1,), -1, dtype=torch.int32, device=dev)
    for _ in range(2):
        assert _offsets(gpu, deg_t, off_t, n, stream) == gpu.OK
        stream.synchronize()
        want = np.zeros(n + 1, np.uint64)
        np.cumsum(deg, dtype=np.uint64, out=want[1:])
        assert np.array_equal(off_t.cpu().numpy().view(np.uint32), (want & 0xFFFFFFFF).astype(np.uint32))
        off_t.fill_(-1)


def test_rejects_oversize_before_launch(gpu):
    import torch

    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    small = torch.zeros(4, dtype=torch.int32, device=dev)
    assert _offsets(gpu, small, small, MAX_N + 1, stream) == gpu.ERR_TOO_LARGE
    assert gpu.lib().mce_csr_offsets_static(0, C.c_void_p(small.data_ptr()), None, 4, None) == gpu.ERR_INVALID_ARG
    stream.synchronize()
    assert small.cpu().tolist() == [0, 0, 0, 0]
