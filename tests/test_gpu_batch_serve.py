"""GPU tests of the two modes around the single-graph path: many graphs in one
captured launch (mce_batch_*), and the request loop with footprint admission
(mce_server_*).  Every per-graph result is compared bit-exactly with the
oracle or with the same graph solved alone."""
from __future__ import annotations

import time

import numpy as np
import pytest

from conftest import opts

pytestmark = pytest.mark.gpu


def oracle_of(oracle_mod, u, v, hist_len=64):
    g = oracle_mod.Graph.from_pairs(u, v).sort_degeneracy()
    r = g.mce(threads=4)
    hist = np.zeros(hist_len, np.uint64)
    for size, c in r.hist.items():
        hist[min(size, hist_len - 1)] += c
    return r, hist


def test_batch_members_match_oracle(gpu, oracle_mod):
    graphs = [gpu.gen_batch_member(i)[:2] for i in range(150)]
    b = gpu.Batch(graphs, opts(gpu))
    try:
        res1, hist1, ms1 = b.solve(opts(gpu))
        res2, hist2, _ = b.solve(opts(gpu))  # replay of the captured launch
    finally:
        b.close()
    assert res1 == res2 and np.array_equal(hist1, hist2)
    assert ms1 > 0
    for i, (u, v) in enumerate(graphs):
        o, oh = oracle_of(oracle_mod, u, v)
        assert (res1[i]["count"], res1[i]["checksum"], res1[i]["max_size"]) == (o.count, o.checksum, o.max_size), i
        assert np.array_equal(hist1[i], oh), i


def test_batch_equals_plain_solves_and_handles_empty_members(gpu):
    graphs = [gpu.gen_rmat(9, 8, 11)]
    graphs.append((np.zeros(0, np.uint32), np.zeros(0, np.uint32)))  # empty member
    graphs.append((np.array([5, 5], np.uint32), np.array([5, 5], np.uint32)))  # loops only
    graphs.append(gpu.gen_gnp(300, 30, 3))
    graphs.append((np.array([1], np.uint32), np.array([2], np.uint32)))
    b = gpu.Batch(graphs, opts(gpu))
    try:
        res, _, _ = b.solve(opts(gpu))
    finally:
        b.close()
    for i, (u, v) in enumerate(graphs):
        r = gpu.solve_coo(u, v, opts(gpu))
        assert (res[i]["count"], res[i]["checksum"]) == (r.count, r.checksum), i


def test_server_results_alone_and_in_the_mix(gpu):
    rng = np.random.default_rng(5)
    reqs = []
    for k in range(24):
        scale = int(rng.integers(8, 13))
        ef = int(rng.integers(8, 33))
        reqs.append(gpu.gen_rmat(scale, ef, 100 + k))
    alone = [gpu.solve_coo(u, v, opts(gpu)) for u, v in reqs]
    s = gpu.Server(device=0, max_inflight=6)
    try:
        ids = []
        for u, v in reqs:
            ids.append(s.submit(u, v))
            time.sleep(0.002)  # arrivals overlap the requests already running
        s.drain()
        got = [s.poll(i) for i in ids]
        spans = [s.span(i) for i in ids]
    finally:
        s.close()
    for k, (g, a) in enumerate(zip(got, alone)):
        assert g is not None, k
        r, lat = g
        assert lat > 0
        assert (r.count, r.checksum, r.hist) == (a.count, a.checksum, a.hist), k
        assert (r.num_vertices, r.num_edges, r.degeneracy, r.max_degree) == (a.num_vertices, a.num_edges,
                                                                              a.degeneracy, a.max_degree), k
    # the mix really shared the device: sweep the requests' device-clock spans
    assert max_overlap(spans) >= 2, spans


def max_overlap(spans):
    """Largest number of [start, end) intervals that contain one instant."""
    ev = sorted([(a, 1) for a, _ in spans] + [(b, -1) for _, b in spans], key=lambda t: (t[0], t[1]))
    cur = best = 0
    for _, d in ev:
        cur += d
        best = max(best, cur)
    return best


def test_server_rejects_unknown_request(gpu):
    s = gpu.Server(device=0)
    try:
        with pytest.raises(gpu.MceError) as e:
            s.poll(12345)
        assert e.value.status == gpu.ERR_NOT_FOUND
    finally:
        s.close()
