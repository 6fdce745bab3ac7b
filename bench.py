#!/usr/bin/env python
"""Maximal cliques/s on one B200 (R-MAT scale 20, edge factor 16, seed 2).

Workload.  The R-MAT scale-20 graph (a/b/c/d = 0.57/0.19/0.19/0.05, seed 2,
symmetrised, deduplicated, self-loops dropped) holds about 1.9e14 maximal
cliques, far more than one timed run can enumerate.  A step therefore
enumerates EVERY maximal clique under a fixed, seeded random sample of edge
roots (the edge-rooted decomposition partitions the clique set: each maximal
clique belongs to exactly one root edge), with the graph resident in HBM.
The same sample is solved every step and must give the same count and
checksum every time.  Under torchrun each rank solves its own disjoint-seeded
sample (weak scaling, no collective on the data path).

Lines printed (rank 0): one JSON line per the benchmark contract: device-timed
`value` (inputs resident), `e2e` through the C ABI from pinned host buffers
(graph build + solve + result read-back inside the timed region), the integer
roofline of the enumeration kernel against a live probe of the INT pipe, and
the CPU oracle on the host cores as `cpu_baseline`.

Parity.  tests/golden/samples/rmat20_sample.json holds the CPU oracle's answer
for the headline sample (count, checksum, histogram, per-root values and a
digest of the ordered CSR); the run fails unless the engine reproduces it.

`--impl reference` times the reference's own CPU solver (oracle/_ref/ref_cpu,
compiled from the unmodified reference sources) on the SAME edge roots of the
same ordered graph: MceSolver::BKFixedMemPivotBit2 with R = {v0, v1}, P and X
split at v1, as the reference's edge-root loop does (src/mce.cc:96-131).  The
graph is written as a reference .bin in the engine's vertex order by a
separate process (oracle/ordered_bin.py), so the timed process loads only the
reference build.  Before timing, the sample's light roots are solved to
completion and checked root by root against the fixture; each timed step then
runs all threads over the sample, heaviest roots first, until its deadline.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SCALE, EDGE_FACTOR, GRAPH_SEED = 20, 16, 2
SAMPLE_SEED = 12345
# smaller graphs enumerated in full (profiling and context lines): name -> (scale, edge factor, seed)
FULL_WORKLOADS = {"rmat14": (14, 16, 1), "rmat16": (16, 16, 1), "chunglu": None}
DEFAULT_SAMPLE = int(os.environ.get("RDMCE_BENCH_SAMPLE", "256"))
METRIC = "maximal cliques/s"
UNIT = "cliques/s"
REF_CPU = os.path.join(ROOT, "oracle", "_ref", "ref_cpu")
FIXTURE = os.path.join(ROOT, "tests", "golden", "samples", "rmat20_sample.json")
FIXTURE24 = os.path.join(ROOT, "tests", "golden", "samples", "rmat24_sample.json")
# roots below this many cliques finish in well under a second on one core:
# the reference arm solves them to completion as its parity check
LIGHT_ROOT = 10_000_000


def profiled_traffic(workload):
    """DRAM bytes (read + write) of one k_enumerate launch of this workload,
    as the committed ncu summary records them; None where none was taken."""
    if workload != "rmat20-sample":
        return None
    try:
        with open(os.path.join(ROOT, "profiles", "k_enumerate_dram_traffic.md")) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch_rmat20_sample:"):
                    return int(line.split(":")[1])
    except OSError:
        pass
    return None


def measured_hbm_gbs():
    """The pool's measured copy bandwidth (GB/s), else the earlier fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def preprocess_roofline(m_coo, n, m, ms):
    """Graph build against HBM: algorithmic bytes B_pre = 8 m_coo (read the
    pairs) + 16 m_coo (two sort passes at least) + 4 (n + 1) + 8 m (write the
    CSR) + 8 m (read the adjacency once while peeling) + 16 m (degree
    decrements, read and write) + 16 m (relabel, read and write)."""
    b = 8 * m_coo + 16 * m_coo + 4 * (n + 1) + 8 * m + 8 * m + 16 * m + 16 * m
    peak, kind = measured_hbm_gbs()
    gbs = b / (ms / 1000.0) / 1e9 if ms > 0 else None
    return {"ms": ms, "algorithmic_bytes": int(b), "achieved_gbs": gbs, "peak_gbs": peak,
            "frac": gbs / peak if gbs else None, "peak_kind": kind,
            "note": "device graph build from resident pairs (sort, dedupe, relabel, k-core peel, CSR, roots), "
                    "library phase time per end-to-end step; bound by the peel's synchronous rounds, not by HBM"}


def load_fixture():
    with open(FIXTURE) as f:
        return json.load(f)


def sample_config(fx, sample):
    """The workload-defining config keys, identical for both arms."""
    return {"workload": workload_name(sample), "roots_per_step": len(fx["roots"]), "sample_seed": fx["sample_seed"],
            "vertices": fx["n"], "edges": fx["m"], "degeneracy": fx["degeneracy"], "max_degree": fx["max_degree"],
            "cliques_per_step": fx["count"], "checksum": fx["checksum"],
            "l2": "512 MiB device write before every GPU step (L2 is 126 MB)",
            "parallelism": "1 rank(s), independent root samples"}


def workload_name(sample, workload="rmat20-sample"):
    if workload == "chunglu":
        return "Chung-Lu n=10,000, expected average degree 16, exponent 2.5, seed 1; full enumeration"
    if workload in FULL_WORKLOADS:
        sc, ef, sd = FULL_WORKLOADS[workload]
        return f"R-MAT scale {sc}, edge factor {ef}, a/b/c/d=0.57/0.19/0.19/0.05, seed {sd}; full enumeration"
    if workload == "rmat24-sample":
        return ("R-MAT scale 24, edge factor 32, a/b/c/d=0.57/0.19/0.19/0.05, seed 3, plus 256 planted cliques of "
                f"40-200 vertices; all maximal cliques under {sample} seeded random edge roots per step")
    return (f"R-MAT scale {SCALE}, edge factor {EDGE_FACTOR}, a/b/c/d=0.57/0.19/0.19/0.05, seed {GRAPH_SEED}; "
            f"all maximal cliques under {sample} seeded random edge roots per rank per step")


class Clocks:
    """nvidia-smi sampler (200 ms) over the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) < 9:
                    continue
                try:
                    sm.append(float(p[1]))
                    smax = float(p[2])
                except ValueError:
                    continue
                for name, val in zip(names, p[5:9]):
                    if val.lower() == "active":
                        reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def make_graph_pairs(workload="rmat20-sample"):
    import numpy as np

    import rdmce_b200 as mce

    if workload == "rmat24-sample":
        # R-MAT scale 24, edge factor 32, seed 3, plus 256 planted cliques of
        # 40-200 vertices on uniform random vertex sets (planted seed 3)
        u, v = mce.gen_rmat(24, 32, 3)
        pu, pv = mce.gen_planted(1 << 24, 256, 40, 200, 3)
        return np.concatenate([u, pu]), np.concatenate([v, pv])
    if workload == "chunglu":
        return mce.gen_chung_lu(10000, 16, 2.5, 1)
    if workload in FULL_WORKLOADS:
        sc, ef, sd = FULL_WORKLOADS[workload]
        return mce.gen_rmat(sc, ef, sd)
    return mce.gen_rmat(SCALE, EDGE_FACTOR, GRAPH_SEED)


def root_sample(m, sample, rank):
    import numpy as np

    rng = np.random.default_rng(SAMPLE_SEED + rank)
    return np.sort(rng.choice(m, size=min(sample, m), replace=False)).astype(np.uint64)


def rank_roots(m, rank, world, full, sample):
    """The roots one rank enumerates: a contiguous share of all m roots for a
    full enumeration (the shares partition [0, m)), else the rank's own seeded
    sample.  Ranks never exchange roots or results on the data path."""
    import numpy as np

    if full:
        return np.arange(m * rank // world, m * (rank + 1) // world, dtype=np.uint64)
    return root_sample(m, sample, rank)


def reduce_over_ranks(x, op, world, device):
    """One all-reduce of a scalar (max of times, sum of counts) for the JSON
    line; the identity on one rank."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def emit(line):
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ reference

def run_reference(args):
    rank, world, _ = dist_env()
    base = {"metric": METRIC, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u64", "data": "synthetic"}
    if rank != 0:
        return 0
    if not os.path.exists(REF_CPU):
        base["unavailable"] = "oracle/_ref/ref_cpu (the reference CPU solver) was not built on this machine"
        emit(base)
        return 0
    fx = load_fixture()
    if args.sample != len(fx["roots"]):
        base["unavailable"] = f"the reference arm runs the fixture's {len(fx['roots'])}-root sample only"
        emit(base)
        return 0
    cores = os.cpu_count() or 1
    total = args.warmup + args.steps
    seconds = max(2.0, min(10.0, 150.0 / total))
    roots = fx["roots"]
    counts = dict(zip(roots, fx["counts"]))
    # heaviest first (longest-processing-time order), so every heavy root
    # starts at once and the light ones fill the remaining threads
    order = sorted(roots, key=lambda r: -counts[r])
    light = [r for r in roots if counts[r] < LIGHT_ROOT]
    with tempfile.TemporaryDirectory() as td:
        binp = os.path.join(td, "rmat20.bin")
        # the ordered graph comes from a separate process (generator + oracle)
        gen = subprocess.run([sys.executable, os.path.join(ROOT, "oracle", "ordered_bin.py"), "rmat20", binp],
                             capture_output=True, text=True, timeout=900)
        if gen.returncode != 0 or fx["csr_sha256"] not in gen.stdout:
            base["unavailable"] = f"could not write the ordered graph: {(gen.stdout + gen.stderr).strip()[-200:]}"
            emit(base)
            return 0
        lightf = os.path.join(td, "light.txt")
        with open(lightf, "w") as f:
            f.write("\n".join(map(str, light)))
        chk = subprocess.run([REF_CPU, "edge_roots", binp, str(cores), lightf], capture_output=True, text=True,
                             timeout=600)
        got = {int(p[1]): int(p[2]) for p in (ln.split() for ln in chk.stdout.splitlines()) if p[:1] == ["ROOT"]}
        bad = [r for r in light if got.get(r) != counts[r]]
        if chk.returncode != 0 or bad:
            raise RuntimeError(f"reference edge-root counts differ from the fixture on roots {bad[:5]}")
        orderf = os.path.join(td, "order.txt")
        with open(orderf, "w") as f:
            f.write("\n".join(map(str, order)))
        out = subprocess.run([REF_CPU, "edge_steps", binp, str(cores), orderf, str(seconds), str(args.warmup),
                              str(args.steps)], capture_output=True, text=True,
                             timeout=60 + total * (seconds + 30) + 600)
    steps = []
    for line in out.stdout.splitlines():
        p = line.split()
        if len(p) >= 8 and p[0] == "STEP":
            steps.append((int(p[1]), int(p[3]), float(p[5]), int(p[7])))
    timed = [st for st in steps if st[0] >= args.warmup]
    if out.returncode != 0 or len(timed) != args.steps:
        base["unavailable"] = f"reference CPU run failed (exit {out.returncode}): {out.stderr.strip()[-200:]}"
        emit(base)
        return 0
    cl = sum(st[1] for st in timed)
    sec = sum(st[2] for st in timed)
    value = cl / sec
    heavy = sum(1 for r in roots if counts[r] >= LIGHT_ROOT)
    sample = (f"reference MceSolver::BKFixedMemPivotBit2 on the same {len(roots)} edge roots of the engine-ordered "
              f"graph (.bin), heaviest first, {cores} threads, {seconds:.1f} s per step, cliques counted at the "
              f"deadline; its {len(light)} light roots were first solved to completion and matched the fixture root "
              f"for root.  {heavy} roots hold {sum(counts[r] for r in roots if counts[r] >= LIGHT_ROOT) / fx['count']:.2%} "
              f"of the cliques and the reference parallelises across roots only, so at most {heavy} threads stay "
              f"busy after the light roots")
    base.update({"value": value, "ms_per_step": 1000.0 * sec / len(timed), "config": sample_config(fx, args.sample),
                 "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                                  "sample": sample},
                 "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                 "parity": "reference light roots == oracle fixture"})
    emit(base)
    return 0


# ----------------------------------------------------------------- our engine

def cpu_baseline(g, roots, seconds, fx=None):
    """The oracle (our C restatement of the reference's CPU path) on the host
    cores, time-bounded, on the same graph and root sample: heaviest roots
    first when the fixture gives per-root counts, as the reference arm runs."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    ro, ci, lab = g.export_csr()
    og = oracle.Graph.from_csr(ro.astype(np.uint64), ci, lab)
    cores = os.cpu_count() or 1
    if fx is not None and [int(r) for r in roots] == fx["roots"]:
        cnt = dict(zip(fx["roots"], fx["counts"]))
        order = np.array(sorted(fx["roots"], key=lambda r: -cnt[r]), np.uint64)
        how = "heaviest first"
    else:
        order = np.random.default_rng(SAMPLE_SEED).permutation(roots)
        how = "in random order"
    res, started, el = og.mce_roots_timed(order, cores, seconds)
    return {"value": res.count / el, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"oracle over the same {len(roots)}-root sample {how}, {el:.1f} s on {cores} threads "
                      f"({started} roots started, {res.count} cliques by the deadline); it parallelises across "
                      f"roots only, like the reference's CPU solver"}


def check_fixture(g, r, fx):
    """The engine's ordered graph and the sample's result against the oracle
    fixture: CSR digest, count, checksum, histogram, largest clique."""
    import hashlib

    import numpy as np

    ro, ci, lab = g.export_csr()
    h = hashlib.sha256()
    for a in (ro, ci, lab):
        h.update(np.ascontiguousarray(a, dtype="<u4").tobytes())
    if h.hexdigest() != fx["csr_sha256"]:
        raise RuntimeError("the ordered CSR differs from the oracle fixture's")
    got = (r.count, f"{r.checksum:016x}", {str(k): c for k, c in r.hist.items()}, r.max_size)
    want = (fx["count"], fx["checksum"], fx["hist"], fx["max_size"])
    if got != want:
        raise RuntimeError(f"result differs from the oracle fixture: {got[:2]} vs {want[:2]}")


def run_ours(args):
    import numpy as np
    import torch

    import rdmce_b200 as mce

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()

    def reduce(x, op):
        return reduce_over_ranks(x, op, world, dev)

    full = args.workload in FULL_WORKLOADS
    u, v = make_graph_pairs(args.workload)
    ref_gpu = None
    if args.ref_gpu and full and rank == 0:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle

        expect = oracle.Graph.from_pairs(u, v).sort_degeneracy().mce(threads=os.cpu_count() or 1).count
        ref_gpu = {"oracle_count": expect, "runs": reference_gpu_runs(u, v, expect)}
    stream = torch.cuda.current_stream(dev)
    o = mce.options(device=local, stream=C.c_void_p(stream.cuda_stream))
    g = mce.Graph.from_coo(u, v, o)
    info = g.info()
    roots = rank_roots(info["num_edges"], rank, world, full, args.sample)

    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)  # 4x L2

    # the timed call goes straight to the C ABI with its arguments prepared,
    # and the result struct is unpacked after the closing event: host-side
    # Python work stays out of the timed region
    L = mce.lib()
    roots_c = np.ascontiguousarray(roots, dtype=np.uint64)
    raw = mce._Result()

    def step():
        flush.fill_(1)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        if full and world == 1:
            st = L.mce_solve(g.h, C.byref(o), C.byref(raw))
        else:
            st = L.mce_solve_root_list(g.h, C.c_void_p(roots_c.ctypes.data), len(roots_c), C.byref(o), C.byref(raw))
        e1.record(stream)
        e1.synchronize()
        if st != mce.OK:
            raise mce.MceError(st, "solve")
        return mce.Result._from(raw), e0.elapsed_time(e1)

    ref = None
    trials = []  # the autotuner's trials of the kernel builds (blocks per SM, device ms)
    for _ in range(args.warmup):
        r, _ms = step()
        ref = (r.count, r.checksum)
        if r.autotune == 1:
            trials.append([r.blocks_per_sm, round(r.phase_ms[mce.PHASE_ENUMERATE], 3)])
    # parity: the headline sample must reproduce the CPU oracle's fixture
    fx = None
    parity = "self-consistent across steps (no fixture)"
    if args.workload == "rmat20-sample" and rank == 0 and os.path.exists(FIXTURE):
        fx = load_fixture()
        if len(fx["roots"]) != len(roots) or [int(x) for x in roots] != fx["roots"]:
            fx = None
        else:
            check_fixture(g, r, fx)
            parity = "oracle-fixture"
    if args.workload == "rmat24-sample" and rank == 0 and os.path.exists(FIXTURE24):
        # the timed roots are too heavy for the oracle: the fixture's
        # stratified roots are checked on the same resident graph (untimed),
        # and the timed sample must agree with itself with and without sharing
        with open(FIXTURE24) as f:
            fx24 = json.load(f)
        r24 = g.solve_root_list(np.array(fx24["roots"], np.uint64), o)
        check_fixture(g, r24, fx24)
        ns = g.solve_root_list(roots, mce.options(device=local, stream=C.c_void_p(stream.cuda_stream),
                                                  flags=mce.FLAG_NO_SHARING))
        if (ns.count, ns.checksum) != ref:
            raise RuntimeError("timed sample differs without task sharing")
        parity = (f"oracle-fixture on {len(fx24['roots'])} stratified roots of the same graph; timed sample "
                  f"identical with and without task sharing")
    clocks = Clocks(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    l0 = mce.launch_count()
    times, enum_ms, launches_enum = [], 0.0, 0
    cycles = [0] * 8
    cliques = 0
    used = set()
    longest = []  # per step: the longest root and the longest task, in warp clock cycles
    enum_steps = []  # per step: device time of the enumeration launch alone (CUDA events in the library)
    for _ in range(args.steps):
        r, ms = step()
        used.add((r.blocks_per_sm, r.autotune))
        longest.append([int(x) for x in r.max_item_cycles])
        enum_steps.append(round(r.phase_ms[mce.PHASE_ENUMERATE], 3))
        if ref is not None and (r.count, r.checksum) != ref:
            raise RuntimeError(f"nondeterministic result: {(r.count, r.checksum)} vs {ref}")
        ref = (r.count, r.checksum)
        times.append(ms)
        cliques += r.count
        enum_ms += r.phase_ms[mce.PHASE_ENUMERATE]
        launches_enum += r.launches
        cycles = [a + b for a, b in zip(cycles, r.warp_cycles)]
    torch.cuda.synchronize()
    barrier()
    launches = mce.launch_count() - l0
    clk = clocks.stop()
    t_local = sum(times) / 1000.0
    t_max = reduce(t_local, _max_op())
    total_cliques = reduce(float(cliques), _sum_op())
    value = total_cliques / t_max

    # end to end through the C ABI: pinned host COO in, graph built on the
    # device, the root sample solved, the result struct read back
    L = mce.lib()
    u_pin = torch.from_numpy(u).pin_memory()
    v_pin = torch.from_numpy(v).pin_memory()
    roots_pin = torch.from_numpy(roots.view(np.int64)).pin_memory()
    res = mce._Result()

    # the engine's own stream, as a caller of the C ABI would have; both calls
    # return with the result in host memory, so host time brackets the step
    o_e2e = mce.options(device=local)
    pre_ms = []
    build_ms = []  # the device graph build alone (sort, dedupe, peel, CSR, roots), pairs already resident

    def e2e_step():
        h = C.c_void_p()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s = L.mce_graph_from_coo(C.c_void_p(u_pin.data_ptr()), C.c_void_p(v_pin.data_ptr()), len(u),
                                 C.byref(o_e2e), C.byref(h))
        if s != mce.OK:
            raise mce.MceError(s, "mce_graph_from_coo")
        if full and world == 1:
            s = L.mce_solve(h, C.byref(o_e2e), C.byref(res))
        else:
            s = L.mce_solve_root_list(h, C.c_void_p(roots_pin.data_ptr()), len(roots), C.byref(o_e2e),
                                      C.byref(res))
        t1 = time.perf_counter()
        L.mce_graph_free(h)
        if s != mce.OK:
            raise mce.MceError(s, "mce_solve_root_list")
        if (res.count, res.checksum) != ref:
            raise RuntimeError("end-to-end result differs from the resident-graph result")
        pre_ms.append(res.phase_ms[mce.PHASE_H2D] + res.phase_ms[mce.PHASE_PREPROCESS])
        build_ms.append(res.phase_ms[mce.PHASE_PREPROCESS])
        return 1000.0 * (t1 - t0)

    e2e_step()
    barrier()
    e2e_times = [e2e_step() for _ in range(args.steps)]
    barrier()
    e2e_max = reduce(sum(e2e_times) / 1000.0, _max_op())
    e2e_value = total_cliques / e2e_max

    # The timed kernel counts nothing.  One untimed solve of the same sample
    # with MCE_FLAG_STATS (a separate kernel instance) counts the search-tree
    # nodes and row word-ops the engine executes.  The roofline's algorithmic
    # work is fixed by the workload instead: the row word-ops of the reference
    # method's search tree (canonical pivot, EXPAND_R) over the same roots,
    # 2 per pivot-scanned row word (ANDN + POPC) plus 1 per row filtered into
    # a child, as the oracle counted them for the fixture.  The engine decides
    # many subtrees in closed form, so it executes fewer than that.
    o_stats = mce.options(device=local, stream=C.c_void_p(stream.cuda_stream), flags=mce.FLAG_STATS)
    rs = g.solve(o_stats) if full and world == 1 else g.solve_root_list(roots, o_stats)
    if (rs.count, rs.checksum) != ref:
        raise RuntimeError("counting run differs from the timed runs")
    wops, nodes = rs.word_ops, rs.nodes
    enum_ms_step = enum_ms / args.steps
    peak = mce.probe_int_peak(local)
    canon = fx.get("canonical_tree") if fx is not None else None
    alg_wops = 2 * canon["pivot_words"] + canon["filter_rows"] if canon else wops
    achieved = alg_wops / (enum_ms_step / 1000.0) if enum_ms_step > 0 else 0.0

    line = None
    if rank == 0:
        cpu = cpu_baseline(g, roots, args.cpu_seconds, fx) if world == 1 and args.cpu_seconds > 0 else None
        if fx is not None:
            config = sample_config(fx, args.sample)
        else:
            config = {"workload": workload_name(args.sample, args.workload), "roots_per_step": int(len(roots)),
                      "sample_seed": SAMPLE_SEED, "vertices": info["num_vertices"], "edges": info["num_edges"],
                      "degeneracy": info["degeneracy"], "max_degree": info["max_degree"],
                      "cliques_per_step": int(ref[0]), "checksum": f"{ref[1]:016x}",
                      "l2": "512 MiB device write before every GPU step (L2 is 126 MB)",
                      "parallelism": f"{world} rank(s), independent root samples"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": config,
            "parity": parity,
            "roofline": {"bound": "int", "achieved": achieved / 1e9, "peak": peak / 1e9, "unit": "Gword-ops/s",
                         "frac": achieved / peak if peak else None,
                         "traffic": profiled_traffic(args.workload),
                         "build_bytes": int(rs.build_bytes),
                         "algorithmic_word_ops": int(alg_wops),
                         "note": ("row word-ops of the reference method's search tree over the step's roots "
                                  "(oracle, canonical pivot: 2 per pivot-scanned row word + 1 per filtered row; "
                                  "tests/golden/samples) / the timed k_enumerate time per step"
                                  if canon else
                                  "bitmap row word-ops of one step (ANDN+POPC per active row per node, row "
                                  "filters; counted by an untimed MCE_FLAG_STATS solve of the same sample) / the "
                                  "timed k_enumerate time per step") + "; peak = live INT-pipe probe of the same op mix; "
                                 "traffic = DRAM read+write bytes of one k_enumerate launch of this workload from "
                                 "ncu (profiles/k_enumerate_dram_traffic.md); build_bytes = the algorithmic "
                                 "ego-network build bytes of one step, counted by the same untimed solve"},
            "e2e": {"value": e2e_value, "unit": UNIT,
                    "h2d_bytes_per_step": int(u.nbytes + v.nbytes + (0 if full and world == 1 else roots.nbytes)),
                    "d2h_bytes_per_step": int(C.sizeof(mce._Result)),
                    "graph_build_ms_per_step": sum(pre_ms[1:]) / max(1, len(pre_ms) - 1),
                    "how": "host wall clock around mce_graph_from_coo (pinned host COO in) + mce_solve_root_list "
                           "(result struct out), on the engine's own stream"},
            "preprocess": preprocess_roofline(len(u), info["num_vertices"], info["num_edges"],
                                              sum(build_ms[1:]) / max(1, len(build_ms) - 1)),
            "autotune": {"trials": trials, "timed_steps": sorted(used),
                         "how": "blocks_per_sm = 0: the first solves of the workload try 4, 5 and 3 resident "
                                "8-warp blocks per SM (64, 51, 85 registers a thread), later solves use the "
                                "fastest; [blocks per SM, mode] of the timed steps, mode 2 = the tuner's choice"},
            "gpu_launches": int(launches),
            "clocks": clk,
            "search": {"nodes_per_step": int(nodes), "word_ops_per_step": int(wops),
                       "nodes_per_s": nodes / (enum_ms_step / 1000.0) if enum_ms_step else None,
                       "enumerate_ms_per_step": enum_ms / args.steps,
                       "step_ms": [round(t, 3) for t in times],
                       "enumerate_step_ms": enum_steps,
                       "longest_item_cycles": longest,
                       "enum_launches_per_step": launches_enum / args.steps,
                       "warp_cycle_share": {k: round(c / max(1, sum(cycles)), 4) for k, c in
                                            zip(["build", "tier64", "general", "spawn", "idle", "queue", "tier32", "reserved"],
                                                cycles)}},
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        if ref_gpu is not None:
            line["reference_gpu"] = ref_gpu
        if world == 1 and args.workload == "rmat20-sample" and not args.no_modes:
            # the many-instance and serving modes, measured after the headline
            line["batch"] = batch_measure(args)
            line["serve"] = serve_measure(args)
        emit(line)
    g.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


REF_GPU = {"stock": os.path.join(ROOT, "oracle", "_ref", "rdmce_ref_gpu"),
           "no task sharing": os.path.join(ROOT, "oracle", "_ref", "rdmce_ref_gpu_noshare")}


def reference_gpu_runs(u, v, expect, repeats=2):
    """The reference's own CUDA build (unmodified sources, sm_100a) on the same
    COO text, through its CLI `-i <file> -o deg -d 0` (main.cc): its count and
    its "MCE GPU Time" (CSR upload + device setup + kernel, mce_gpu.cu:14-22).
    Run before this process touches the GPU.  Each build runs `repeats` times
    so a count that changes between runs shows."""
    import numpy as np

    runs = []
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "graph.txt")
        with open(path, "w") as f:
            for i in range(0, len(u), 1 << 20):
                blk = np.stack([u[i:i + (1 << 20)], v[i:i + (1 << 20)]], axis=1)
                f.write("\n".join(f"{a} {b}" for a, b in blk.tolist()))
                f.write("\n")
        for name, exe in REF_GPU.items():
            if not os.path.exists(exe):
                continue
            for rep in range(repeats if name == "stock" else 1):
                try:
                    out = subprocess.run([exe, "-i", path, "-o", "deg", "-d", "0"], capture_output=True, text=True,
                                         timeout=900)
                except subprocess.TimeoutExpired:
                    runs.append({"build": name, "run": rep, "error": "timed out after 900 s"})
                    break
                cnt = sec = None
                for line in out.stdout.splitlines():
                    if line.startswith("MC numbers:"):
                        cnt = int(line.split(":")[1])
                    if line.startswith("MCE GPU Time:"):
                        sec = float(line.split(":")[1].strip().rstrip("s"))
                rec = {"build": name, "run": rep, "count": cnt, "seconds": sec, "exit": out.returncode}
                if cnt is not None and sec:
                    rec["cliques_per_s"] = cnt / sec
                    rec["count_matches_oracle"] = cnt == expect
                runs.append(rec)
    return runs


BATCH_FIXTURE = os.path.join(ROOT, "tests", "golden", "samples", "batch_members.npz")
SERVE_FIXTURE = os.path.join(ROOT, "tests", "golden", "samples", "serve_requests.json")


def batch_measure(args):
    """Many-instance mode (config: 10,000 G(n,p) + planted-clique members, n
    log-uniform in [64, 4096], degree uniform in [8, 64], seed 1000 + index)
    in one captured persistent launch per step, against one plain solve per
    resident graph.  Every member is checked against the oracle fixture."""
    import numpy as np
    import torch

    import rdmce_b200 as mce

    torch.cuda.set_device(0)
    o = mce.options(device=0)
    n = args.batch_graphs
    graphs = [mce.gen_batch_member(i)[:2] for i in range(n)]
    edges = sum(len(u) for u, _ in graphs)
    b = mce.Batch(graphs, o)
    for _ in range(args.warmup):
        res, hist, _ = b.solve(o)
    ref = [(r["count"], r["checksum"]) for r in res]
    times = []
    for _ in range(args.steps):
        res, _, ms = b.solve(o)
        if [(r["count"], r["checksum"]) for r in res] != ref:
            raise RuntimeError("batched results changed between steps")
        times.append(ms)
    b.close()
    parity = "self-consistent across steps (no fixture)"
    if os.path.exists(BATCH_FIXTURE):
        fx = np.load(BATCH_FIXTURE)
        if len(fx["count"]) == n:
            got = np.array([[r["count"], r["checksum"], r["max_size"]] for r in res], np.uint64)
            want = np.stack([fx["count"], fx["checksum"], fx["max_size"].astype(np.uint64)], 1)
            if not (np.array_equal(got, want) and np.array_equal(np.asarray(hist, np.uint64), fx["hist"])):
                raise RuntimeError("batched results differ from the oracle fixture")
            parity = f"oracle-fixture ({n} members: count, checksum, largest clique, histogram)"
    value = n / (sum(times) / len(times) / 1000.0)
    # plain: one solve (one enumeration launch) per resident graph
    p = min(n, args.plain_graphs)
    handles = [mce.Graph.from_coo(u, v, o) for u, v in graphs[:p]]
    for h in handles:
        h.solve(o)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k, h in enumerate(handles):
        r = h.solve(o)
        if (r.count, r.checksum) != ref[k]:
            raise RuntimeError(f"graph {k}: plain solve differs from the batched solve")
    plain_s = time.perf_counter() - t0
    for h in handles:
        h.close()
    plain = p / plain_s
    return {"metric": "graphs/s (many-instance batch, one captured launch)", "value": value, "unit": "graphs/s",
            "ms_per_step": sum(times) / len(times), "steps": args.steps,
            "config": {"workload": f"{n} G(n,p) graphs, n log-uniform in [64, 4096], mean degree uniform in [8, 64], "
                                   f"0-3 planted cliques of size 8-32, seed 1000 + index", "graphs": n,
                       "pairs": int(edges), "cliques_per_step": int(sum(c for c, _ in ref))},
            "parity": parity,
            "plain_per_graph": {"value": plain, "unit": "graphs/s", "graphs_timed": p,
                                "how": "mce_solve on each resident graph in turn, host wall clock"},
            "batched_over_plain": value / plain,
            "how": "CUDA events around the captured launch (graph replay) per step"}


def serve_requests(nreq):
    """Request k: R-MAT with (scale, edge factor) drawn in order from
    default_rng(5) -- scale uniform in [10, 13], edge factor uniform in [8, 32]
    -- and graph seed 5000 + k; the same stream then draws the arrival gaps."""
    import numpy as np

    rng = np.random.default_rng(5)
    return rng, [(int(rng.integers(10, 14)), int(rng.integers(8, 33)), 5000 + k) for k in range(nreq)]


def serve_measure(args):
    """Request loop: Poisson arrivals (seed 5) of R-MAT requests; p50/p99
    latency and cliques/s per arrival rate, against the same requests solved
    one after another.  Every served result is checked against the oracle
    fixture (count, checksum, largest clique)."""
    import numpy as np
    import torch

    import rdmce_b200 as mce

    torch.cuda.set_device(0)
    rng, spec = serve_requests(args.serve_requests)
    reqs = [mce.gen_rmat(sc, ef, sd) for sc, ef, sd in spec]
    want = None
    if os.path.exists(SERVE_FIXTURE):
        with open(SERVE_FIXTURE) as f:
            fxr = json.load(f)["requests"]
        if [(q["scale"], q["edge_factor"], q["seed"]) for q in fxr] == spec:
            want = [(q["count"], q["checksum"], q["max_size"]) for q in fxr]
    o = mce.options(device=0)
    for u, v in reqs[:8]:
        mce.solve_coo(u, v, o)  # warm-up
    t0 = time.perf_counter()
    serial = [mce.solve_coo(u, v, o) for u, v in reqs]
    serial_s = time.perf_counter() - t0
    if want is not None and [(r.count, f"{r.checksum:016x}", r.max_size) for r in serial] != want:
        raise RuntimeError("serial solves differ from the oracle fixture")
    total = sum(r.count for r in serial)
    lines = []
    for rate in args.serve_rates:
        gaps = rng.exponential(1.0 / rate, size=len(reqs))
        s = mce.Server(device=0)
        ids = []
        start = time.perf_counter()
        due = start
        for (u, v), gap in zip(reqs, gaps):
            due += gap
            now = time.perf_counter()
            if due > now:
                time.sleep(due - now)
            ids.append(s.submit(u, v))
        s.drain()
        span = time.perf_counter() - start
        lat, spans = [], []
        for k, rid in enumerate(ids):
            r, ms = s.poll(rid)
            if (r.count, r.checksum) != (serial[k].count, serial[k].checksum):
                raise RuntimeError(f"request {k}: served result differs from the solve alone")
            lat.append(ms)
            spans.append(s.span(rid))
        s.close()
        ev = sorted([(a, 1) for a, _ in spans] + [(b, -1) for _, b in spans])
        cur = peak = 0
        for _, d in ev:
            cur += d
            peak = max(peak, cur)
        lines.append({"rate_per_s": rate, "p50_ms": float(np.percentile(lat, 50)),
                      "p99_ms": float(np.percentile(lat, 99)), "cliques_per_s": total / span, "span_s": span,
                      "peak_requests_on_device": peak})
    return {"metric": "served maximal cliques/s and p50/p99 latency", "value": lines[-1]["cliques_per_s"],
            "unit": "cliques/s",
            "config": {"workload": f"{len(reqs)} R-MAT requests, scale uniform in [10, 13], edge factor uniform in "
                                   f"[8, 32], Poisson arrivals seed 5, request k seeded 5000 + k",
                       "cliques": int(total)},
            "parity": "oracle-fixture (every request: count, checksum, largest clique)" if want is not None else
                      "served == solved alone",
            "rates": lines, "serial_plain": {"cliques_per_s": total / serial_s, "seconds": serial_s},
            "how": "host wall clock from first arrival to the last completion; peak_requests_on_device from the "
                   "requests' device-clock spans (mce_server_request_span)"}


def run_ingest(args):
    """Text ingest: the R-MAT scale-20 graph as 16.8M lines of COO text, loaded
    (a) by the reference's own Graph::LoadFromFile text loop (its printed read
    time, oracle/_ref/ref_cpu), (b) by the engine's parallel host parser, and
    (c) on the GPU: file streamed to device memory, parsed there, pairs handed
    to the device graph build (mce_graph_load_file).  (c) is timed through the
    C ABI with host wall clock, the build included; its parse part is the
    phase_ms[H2D] slot of the result."""
    import numpy as np
    import torch

    import rdmce_b200 as mce

    torch.cuda.set_device(0)
    u, v = mce.gen_rmat(SCALE, EDGE_FACTOR, GRAPH_SEED)
    o = mce.options(device=0)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "rmat20.txt")
        with open(path, "w") as f:
            for i in range(0, len(u), 1 << 20):
                blk = np.stack([u[i:i + (1 << 20)], v[i:i + (1 << 20)]], axis=1)
                f.write("\n".join(f"{a} {b}" for a, b in blk.tolist()))
                f.write("\n")
        size = os.path.getsize(path)
        ref_read = None
        if os.path.exists(REF_CPU):
            out = subprocess.run([REF_CPU, "stats", path], capture_output=True, text=True, timeout=900)
            for line in out.stdout.splitlines():
                if line.startswith("Read ") and " seconds" in line:
                    ref_read = float(line.split(" in ")[1].split()[0])
        for _ in range(args.warmup):
            hu, hv = mce.parse_text(path)
            gu, gv = mce.parse_text(path, device=0)
            if not (np.array_equal(hu, u) and np.array_equal(gu, u) and np.array_equal(gv, v)):
                raise RuntimeError("parsed pairs differ from the generator's")
        host_s, gpu_parse_ms, load_s = [], [], []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            mce.parse_text(path)
            host_s.append(time.perf_counter() - t0)
            t0 = time.perf_counter()
            with mce.Graph.load_file(path, o) as g:
                load_s.append(time.perf_counter() - t0)
                r = g.solve_root_list(np.zeros(1, np.uint64), o)
                gpu_parse_ms.append(r.phase_ms[mce.PHASE_H2D])
    med = statistics.median
    emit({"metric": "COO text ingest (file -> device graph)", "value": size / med(load_s) / 1e9, "unit": "GB/s",
          "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
          "vs_baseline": None, "dtype": "u8", "data": "synthetic",
          "config": {"workload": f"R-MAT scale {SCALE}, edge factor {EDGE_FACTOR}, seed {GRAPH_SEED} as COO text",
                     "bytes": size, "lines": int(len(u))},
          "gpu_file_to_graph_s": med(load_s), "gpu_parse_incl_upload_ms": med(gpu_parse_ms),
          "host_parse_s": med(host_s), "reference_read_s": ref_read,
          "parity": "GPU and host parses equal the generator's pairs",
          "how": "host wall clock; the GPU parse time includes reading the file into pinned memory and the "
                 "uploads; the reference's read time is the one its loader prints"})
    return 0


def run_batch(args):
    line = batch_measure(args)
    emit({**line, "n_gpus": 1, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
          "vs_baseline": None, "dtype": "u64", "data": "synthetic"})
    return 0


def run_serve(args):
    line = serve_measure(args)
    emit({**line, "n_gpus": 1, "steps": len(args.serve_rates), "warmup": 8, "higher_is_better": True,
          "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic"})
    return 0


def _max_op():
    import torch.distributed as dist

    return dist.ReduceOp.MAX


def _sum_op():
    import torch.distributed as dist

    return dist.ReduceOp.SUM


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--sample", type=int, default=None,
                    help=f"edge roots per rank per step (default {DEFAULT_SAMPLE}; 16 for rmat24-sample)")
    ap.add_argument("--workload", choices=["rmat20-sample", "rmat24-sample"] + sorted(FULL_WORKLOADS),
                    default="rmat20-sample",
                    help="the headline root sample of R-MAT scale 20, the R-MAT 24 + planted-clique sample, or a "
                         "smaller graph enumerated in full")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU oracle time bound (0 = skip)")
    ap.add_argument("--mode", choices=["solve", "batch", "serve", "ingest"], default="solve",
                    help="solve: the headline; batch: many-instance graphs/s; serve: the request loop")
    ap.add_argument("--batch-graphs", type=int, default=10000)
    ap.add_argument("--plain-graphs", type=int, default=1000, help="graphs timed with one plain solve each")
    ap.add_argument("--serve-requests", type=int, default=200)
    ap.add_argument("--serve-rates", type=float, nargs="+", default=[10.0, 100.0, 2000.0])
    ap.add_argument("--ref-gpu", action="store_true",
                    help="full workloads: also run the reference's own CUDA builds on the same graph")
    ap.add_argument("--no-modes", action="store_true",
                    help="headline only: skip the batch and serve objects of the default line")
    args = ap.parse_args()
    if args.sample is None:
        args.sample = 16 if args.workload == "rmat24-sample" else DEFAULT_SAMPLE
    if args.warmup < 3:
        ap.error("--warmup must be at least 3")
    if args.impl == "reference":
        return run_reference(args)
    if args.mode == "batch":
        return run_batch(args)
    if args.mode == "serve":
        return run_serve(args)
    if args.mode == "ingest":
        return run_ingest(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
