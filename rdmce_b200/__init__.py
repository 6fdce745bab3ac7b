"""rdmce_b200 -- B200-native maximal clique enumeration.

Python binding over the engine's C ABI (include/rdmce.h, built in-tree as
rdmce_b200/librdmce.so).  The binding is plumbing only: every call goes to the
CUDA library, and importing fails loudly when the library has not been built.

The host API mirrors the RDMCE reference: a graph is loaded from COO pairs, a
COO text file or the reference `.bin` container (Graph::LoadFromFile /
LoadFromBin, src/graph.cc), reordered by degeneracy (Graph::SortByOrder), and
solved (MceGpuSolver::Solve, src/mce_gpu.cu).  Results add a clique-size
histogram and an order-independent checksum to the reference's count.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# RDMCE_LIB points the binding at another build of the same library
LIB_PATH = os.environ.get("RDMCE_LIB", os.path.join(HERE, "librdmce.so"))
CLI_PATH = os.path.join(HERE, "bin", "RDMCE")
HIST_LEN = 8192
PHASES = 6

# mce_status
OK, ERR_INVALID_ARG, ERR_CAPACITY, ERR_IO, ERR_FORMAT, ERR_NO_DEVICE, ERR_CUDA, ERR_OUT_OF_MEMORY, \
    ERR_TIMEOUT, ERR_TOO_LARGE, ERR_BUSY, ERR_NOT_FOUND, ERR_INTERNAL = range(13)
ORDER_DEGENERACY, ORDER_UNCHANGED, ORDER_DEGREE_ASC, ORDER_DEGREE_DESC = range(4)
FLAG_NO_SHARING, FLAG_PER_ROOT, FLAG_QUIET, FLAG_STATS = 1, 2, 4, 8
PHASE_H2D, PHASE_PREPROCESS, PHASE_SETUP, PHASE_ENUMERATE, PHASE_D2H, PHASE_TOTAL = range(6)


class MceError(RuntimeError):
    def __init__(self, status: int, what: str):
        super().__init__(f"{what}: {status_str(status)} (status {status})")
        self.status = status


class Options(C.Structure):
    _fields_ = [
        ("device", C.c_int),
        ("order", C.c_int),
        ("warps_per_block", C.c_uint32),
        ("blocks_per_sm", C.c_uint32),
        ("share_bound", C.c_uint32),
        ("expand_r", C.c_int),
        ("root_begin", C.c_uint64),
        ("root_end", C.c_uint64),
        ("spin_limit", C.c_uint64),
        ("stream", C.c_void_p),
        ("flags", C.c_uint32),
        ("reg_share_bound", C.c_uint32),
        ("slab_kib", C.c_uint32),
        ("heavy_warps", C.c_uint32),
        ("reserved", C.c_uint32 * 4),
    ]


class _Result(C.Structure):
    _fields_ = [
        ("count", C.c_uint64),
        ("checksum", C.c_uint64),
        ("max_size", C.c_uint32),
        ("degeneracy", C.c_uint32),
        ("max_degree", C.c_uint32),
        ("status_detail", C.c_uint32),
        ("blocks_per_sm", C.c_uint32),
        ("autotune", C.c_uint32),
        ("num_vertices", C.c_uint64),
        ("num_edges", C.c_uint64),
        ("roots", C.c_uint64),
        ("shared_tasks", C.c_uint64),
        ("heavy_roots", C.c_uint64),
        ("nodes", C.c_uint64),
        ("word_ops", C.c_uint64),
        ("build_bytes", C.c_uint64),
        ("launches", C.c_uint64),
        ("warp_cycles", C.c_uint64 * 8),
        ("max_item_cycles", C.c_uint64 * 2),
        ("phase_ms", C.c_double * PHASES),
        ("hist", C.c_uint64 * HIST_LEN),
    ]


class _Info(C.Structure):
    _fields_ = [
        ("num_vertices", C.c_uint64),
        ("num_edges", C.c_uint64),
        ("max_degree", C.c_uint32),
        ("degeneracy", C.c_uint32),
        ("device_bytes", C.c_uint64),
    ]


class _BatchResult(C.Structure):
    _fields_ = [
        ("count", C.c_uint64),
        ("checksum", C.c_uint64),
        ("max_size", C.c_uint32),
        ("num_vertices", C.c_uint32),
        ("num_edges", C.c_uint64),
    ]


class _ServerOptions(C.Structure):
    _fields_ = [
        ("device", C.c_int),
        ("memory_budget", C.c_uint64),
        ("max_inflight", C.c_uint32),
        ("reserved", C.c_uint32 * 5),
    ]


@dataclass
class Result:
    count: int
    checksum: int
    hist: dict = field(default_factory=dict)
    max_size: int = 0
    degeneracy: int = 0
    max_degree: int = 0
    num_vertices: int = 0
    num_edges: int = 0
    roots: int = 0
    shared_tasks: int = 0
    heavy_roots: int = 0
    phase_ms: list = field(default_factory=list)
    nodes: int = 0
    word_ops: int = 0
    launches: int = 0
    # warp clock cycles: root build, register tiers, general tier, exposing tasks, idle, queue
    warp_cycles: list = field(default_factory=list)
    max_item_cycles: list = field(default_factory=list)
    build_bytes: int = 0
    blocks_per_sm: int = 0
    autotune: int = 0

    @classmethod
    def _from(cls, r: _Result) -> "Result":
        hist = {s: int(r.hist[s]) for s in range(HIST_LEN) if r.hist[s]}
        return cls(r.count, r.checksum, hist, r.max_size, r.degeneracy, r.max_degree, r.num_vertices,
                   r.num_edges, r.roots, r.shared_tasks, r.heavy_roots, list(r.phase_ms), r.nodes, r.word_ops,
                   r.launches, list(r.warp_cycles), list(r.max_item_cycles), r.build_bytes, r.blocks_per_sm,
                   r.autotune)


_lib = None

# name -> (restype, argtypes); every function of include/rdmce.h
_P, _U32, _U64, _I, _D = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int, C.c_double
_SIGS = {
    "mce_default_options": (None, [C.POINTER(Options)]),
    "mce_status_str": (C.c_char_p, [_I]),
    "mce_version": (C.c_char_p, []),
    "mce_graph_from_coo": (_I, [_P, _P, _U64, C.POINTER(Options), C.POINTER(_P)]),
    "mce_graph_from_coo_device": (_I, [_P, _P, _U64, C.POINTER(Options), C.POINTER(_P)]),
    "mce_graph_from_csr": (_I, [_U64, _P, _P, _P, _I, C.POINTER(Options), C.POINTER(_P)]),
    "mce_graph_load_file": (_I, [C.c_char_p, C.POINTER(Options), C.POINTER(_P)]),
    "mce_graph_store_bin": (_I, [_P, C.c_char_p]),
    "mce_graph_info_get": (_I, [_P, C.POINTER(_Info)]),
    "mce_graph_export_csr": (_I, [_P, _P, _P, _P]),
    "mce_graph_free": (None, [_P]),
    "mce_solve": (_I, [_P, C.POINTER(Options), C.POINTER(_Result)]),
    "mce_solve_roots": (_I, [_P, _P, _U64, C.POINTER(Options), _P, _P]),
    "mce_solve_root_list": (_I, [_P, _P, _U64, C.POINTER(Options), C.POINTER(_Result)]),
    "mce_launch_count": (_U64, []),
    "mce_csr_offsets_static": (_I, [_I, _P, _P, _U64, _P]),
    "mce_probe_int_peak": (_I, [_I, C.POINTER(_D)]),
    "mce_solve_coo": (_I, [_P, _P, _U64, C.POINTER(Options), C.POINTER(_Result)]),
    "mce_batch_create": (_I, [_P, _P, _P, _U32, C.POINTER(Options), C.POINTER(_P)]),
    "mce_batch_solve": (_I, [_P, C.POINTER(Options), _P, _P, _U32, C.POINTER(_D)]),
    "mce_batch_free": (None, [_P]),
    "mce_server_create": (_I, [C.POINTER(_ServerOptions), C.POINTER(_P)]),
    "mce_server_submit": (_I, [_P, _P, _P, _U64, C.POINTER(_U64)]),
    "mce_server_poll": (_I, [_P, _U64, C.POINTER(_I), C.POINTER(_Result), C.POINTER(_D)]),
    "mce_server_drain": (_I, [_P]),
    "mce_server_request_span": (_I, [_P, C.c_uint64, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "mce_server_free": (None, [_P]),
    "mce_mix64": (_U64, [_U64]),
    "mce_gen_rmat": (_I, [_U32, _U32, _D, _D, _D, _U64, _P, _P, _U64, C.POINTER(_U64), _I]),
    "mce_gen_chung_lu": (_I, [_U32, _D, _D, _U64, _P, _P, _U64, C.POINTER(_U64), _I]),
    "mce_gen_gnp": (_I, [_U32, _D, _U64, _P, _P, _U64, C.POINTER(_U64)]),
    "mce_gen_planted": (_I, [_U32, _U32, _U32, _U32, _U64, _P, _P, _U64, C.POINTER(_U64)]),
    "mce_gen_batch_member": (_I, [_U32, _U64, _P, _P, _U64, C.POINTER(_U64), C.POINTER(_U32)]),
    "mce_parse_text": (_I, [C.c_char_p, C.POINTER(_P), C.POINTER(_P), C.POINTER(_U64)]),
    "mce_parse_text_gpu": (_I, [C.c_char_p, _I, C.POINTER(_P), C.POINTER(_P), C.POINTER(_U64)]),
    "mce_free_host": (None, [_P]),
}


def build(quiet: bool = True) -> None:
    """Compile the CUDA library and the CLI in-tree (nvcc, sm_100a)."""
    cmd = ["make", "-j8", "-C", os.path.join(HERE, "csrc")]
    if quiet:
        cmd.insert(1, "-s")
    subprocess.run(cmd, check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with rdmce_b200.build() or __graft_entry__.build()")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def status_str(s: int) -> str:
    return lib().mce_status_str(s).decode()


def _check(s: int, what: str):
    if s != OK:
        raise MceError(s, what)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def options(**kw) -> Options:
    o = Options()
    lib().mce_default_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def mix64(x: int) -> int:
    return lib().mce_mix64(x)


# ---------------------------------------------------------------- generators

def gen_rmat(scale, edge_factor, seed, a=0.57, b=0.19, c=0.19, threads=0):
    n = edge_factor << scale
    u = np.empty(n, np.uint32)
    v = np.empty(n, np.uint32)
    cnt = C.c_uint64()
    _check(lib().mce_gen_rmat(scale, edge_factor, a, b, c, seed, _ptr(u), _ptr(v), n, C.byref(cnt), threads),
           "mce_gen_rmat")
    return u, v


def _two_pass(fn, *args):
    cnt = C.c_uint64()
    _check(fn(*args, None, None, 0, C.byref(cnt)), fn.__name__)
    n = cnt.value
    u = np.empty(max(n, 1), np.uint32)
    v = np.empty(max(n, 1), np.uint32)
    _check(fn(*args, _ptr(u), _ptr(v), n, C.byref(cnt)), fn.__name__)
    return u[:n], v[:n]


def gen_chung_lu(n, avg_degree, gamma, seed, threads=0):
    cnt = C.c_uint64()
    L = lib()
    _check(L.mce_gen_chung_lu(n, avg_degree, gamma, seed, None, None, 0, C.byref(cnt), threads), "chung_lu")
    k = cnt.value
    u = np.empty(k, np.uint32)
    v = np.empty(k, np.uint32)
    _check(L.mce_gen_chung_lu(n, avg_degree, gamma, seed, _ptr(u), _ptr(v), k, C.byref(cnt), threads), "chung_lu")
    return u, v


def gen_gnp(n, avg_degree, seed):
    return _two_pass(lib().mce_gen_gnp, n, avg_degree, seed)


def gen_planted(n, num_cliques, size_lo, size_hi, seed):
    return _two_pass(lib().mce_gen_planted, n, num_cliques, size_lo, size_hi, seed)


def gen_batch_member(index, base_seed=1000):
    L = lib()
    cnt, nv = C.c_uint64(), C.c_uint32()
    _check(L.mce_gen_batch_member(index, base_seed, None, None, 0, C.byref(cnt), C.byref(nv)), "batch_member")
    k = cnt.value
    u = np.empty(max(k, 1), np.uint32)
    v = np.empty(max(k, 1), np.uint32)
    _check(L.mce_gen_batch_member(index, base_seed, _ptr(u), _ptr(v), k, C.byref(cnt), C.byref(nv)),
           "batch_member")
    return u[:k], v[:k], nv.value


def parse_text(path: str, device: int | None = None):
    """COO text with the reference parser's semantics: on the host, or on the
    GPU `device` (the path mce_graph_load_file takes for text)."""
    L = lib()
    pu, pv, n = C.c_void_p(), C.c_void_p(), C.c_uint64()
    if device is None:
        _check(L.mce_parse_text(path.encode(), C.byref(pu), C.byref(pv), C.byref(n)), "mce_parse_text")
    else:
        _check(L.mce_parse_text_gpu(path.encode(), device, C.byref(pu), C.byref(pv), C.byref(n)),
               "mce_parse_text_gpu")
    k = n.value
    if k:
        u = np.ctypeslib.as_array(C.cast(pu, C.POINTER(C.c_uint32)), shape=(k,)).copy()
        v = np.ctypeslib.as_array(C.cast(pv, C.POINTER(C.c_uint32)), shape=(k,)).copy()
    else:
        u = np.empty(0, np.uint32)
        v = np.empty(0, np.uint32)
    L.mce_free_host(pu)
    L.mce_free_host(pv)
    return u, v


# ----------------------------------------------------------------- graphs

class Graph:
    """A device-resident, degeneracy-ordered graph (mce_graph handle)."""

    def __init__(self, handle):
        self.h = handle

    @classmethod
    def from_coo(cls, u, v, opts: Options | None = None):
        u = np.ascontiguousarray(u, dtype=np.uint32)
        v = np.ascontiguousarray(v, dtype=np.uint32)
        if u.shape != v.shape:
            raise ValueError("u and v differ in length")
        h = C.c_void_p()
        _check(lib().mce_graph_from_coo(_ptr(u), _ptr(v), len(u), C.byref(opts) if opts else None, C.byref(h)),
               "mce_graph_from_coo")
        return cls(h)

    @classmethod
    def from_coo_device(cls, u_ptr: int, v_ptr: int, n: int, opts: Options | None = None):
        h = C.c_void_p()
        _check(lib().mce_graph_from_coo_device(C.c_void_p(u_ptr), C.c_void_p(v_ptr), n,
                                               C.byref(opts) if opts else None, C.byref(h)),
               "mce_graph_from_coo_device")
        return cls(h)

    @classmethod
    def from_csr(cls, rowoffset, colidx, labels=None, already_ordered=False, opts: Options | None = None):
        ro = np.ascontiguousarray(rowoffset, dtype=np.uint32)
        ci = np.ascontiguousarray(colidx, dtype=np.uint32)
        lab = None if labels is None else np.ascontiguousarray(labels, dtype=np.uint32)
        h = C.c_void_p()
        _check(lib().mce_graph_from_csr(len(ro) - 1, _ptr(ro), _ptr(ci), None if lab is None else _ptr(lab),
                                        1 if already_ordered else 0, C.byref(opts) if opts else None, C.byref(h)),
               "mce_graph_from_csr")
        return cls(h)

    @classmethod
    def load_file(cls, path: str, opts: Options | None = None):
        h = C.c_void_p()
        _check(lib().mce_graph_load_file(path.encode(), C.byref(opts) if opts else None, C.byref(h)),
               "mce_graph_load_file")
        return cls(h)

    def close(self):
        if getattr(self, "h", None):
            lib().mce_graph_free(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def info(self) -> dict:
        i = _Info()
        _check(lib().mce_graph_info_get(self.h, C.byref(i)), "mce_graph_info_get")
        return {"num_vertices": i.num_vertices, "num_edges": i.num_edges, "max_degree": i.max_degree,
                "degeneracy": i.degeneracy, "device_bytes": i.device_bytes}

    def export_csr(self):
        i = self.info()
        ro = np.zeros(i["num_vertices"] + 1, np.uint32)
        ci = np.zeros(max(2 * i["num_edges"], 1), np.uint32)
        lab = np.zeros(max(i["num_vertices"], 1), np.uint32)
        _check(lib().mce_graph_export_csr(self.h, _ptr(ro), _ptr(ci), _ptr(lab)), "mce_graph_export_csr")
        return ro, ci[:2 * i["num_edges"]], lab[:i["num_vertices"]]

    def store_bin(self, path: str):
        _check(lib().mce_graph_store_bin(self.h, path.encode()), "mce_graph_store_bin")

    def solve(self, opts: Options | None = None) -> Result:
        r = _Result()
        _check(lib().mce_solve(self.h, C.byref(opts) if opts else None, C.byref(r)), "mce_solve")
        return Result._from(r)

    def solve_roots(self, roots, opts: Options | None = None):
        roots = np.ascontiguousarray(roots, dtype=np.uint64)
        cnt = np.zeros(len(roots), np.uint64)
        chk = np.zeros(len(roots), np.uint64)
        _check(lib().mce_solve_roots(self.h, _ptr(roots), len(roots), C.byref(opts) if opts else None, _ptr(cnt),
                                     _ptr(chk)), "mce_solve_roots")
        return cnt, chk

    def solve_root_list(self, roots, opts: Options | None = None) -> Result:
        """Enumerate only the listed roots (indices into the degeneracy-ordered edge list)."""
        roots = np.ascontiguousarray(roots, dtype=np.uint64)
        r = _Result()
        _check(lib().mce_solve_root_list(self.h, _ptr(roots), len(roots), C.byref(opts) if opts else None,
                                         C.byref(r)), "mce_solve_root_list")
        return Result._from(r)


def launch_count() -> int:
    """Kernels this process has launched through the engine so far."""
    return int(lib().mce_launch_count())


def probe_int_peak(device: int = 0) -> float:
    """Measured 64-bit ANDN+POPC word-op throughput of the device (ops/s)."""
    d = C.c_double()
    _check(lib().mce_probe_int_peak(device, C.byref(d)), "mce_probe_int_peak")
    return d.value


def solve_coo(u, v, opts: Options | None = None) -> Result:
    u = np.ascontiguousarray(u, dtype=np.uint32)
    v = np.ascontiguousarray(v, dtype=np.uint32)
    r = _Result()
    _check(lib().mce_solve_coo(_ptr(u), _ptr(v), len(u), C.byref(opts) if opts else None, C.byref(r)),
           "mce_solve_coo")
    return Result._from(r)


class Batch:
    """Many graphs enumerated in one captured persistent launch."""

    def __init__(self, graphs, opts: Options | None = None):
        offs = [0]
        for u, _v in graphs:
            offs.append(offs[-1] + len(u))
        self.n_graphs = len(graphs)
        u = np.ascontiguousarray(np.concatenate([np.asarray(g[0], np.uint32) for g in graphs]) if offs[-1]
                                 else np.zeros(1, np.uint32))
        v = np.ascontiguousarray(np.concatenate([np.asarray(g[1], np.uint32) for g in graphs]) if offs[-1]
                                 else np.zeros(1, np.uint32))
        po = np.asarray(offs, np.uint64)
        h = C.c_void_p()
        _check(lib().mce_batch_create(_ptr(u), _ptr(v), _ptr(po), self.n_graphs, C.byref(opts) if opts else None,
                                      C.byref(h)), "mce_batch_create")
        self.h = h

    def solve(self, opts: Options | None = None, hist_len: int = 64):
        res = (_BatchResult * self.n_graphs)()
        hist = np.zeros(self.n_graphs * hist_len, np.uint64)
        ms = C.c_double()
        _check(lib().mce_batch_solve(self.h, C.byref(opts) if opts else None, C.cast(res, C.c_void_p), _ptr(hist),
                                     hist_len, C.byref(ms)), "mce_batch_solve")
        out = [{"count": r.count, "checksum": r.checksum, "max_size": r.max_size, "num_vertices": r.num_vertices,
                "num_edges": r.num_edges} for r in res]
        return out, hist.reshape(self.n_graphs, hist_len), ms.value

    def close(self):
        if getattr(self, "h", None):
            lib().mce_batch_free(self.h)
            self.h = None

    def __del__(self):
        self.close()


class Server:
    """Continuous-batching request loop (mce_server)."""

    def __init__(self, device=0, memory_budget=0, max_inflight=0):
        o = _ServerOptions()
        o.device, o.memory_budget, o.max_inflight = device, memory_budget, max_inflight
        h = C.c_void_p()
        _check(lib().mce_server_create(C.byref(o), C.byref(h)), "mce_server_create")
        self.h = h

    def submit(self, u, v) -> int:
        u = np.ascontiguousarray(u, dtype=np.uint32)
        v = np.ascontiguousarray(v, dtype=np.uint32)
        rid = C.c_uint64()
        _check(lib().mce_server_submit(self.h, _ptr(u), _ptr(v), len(u), C.byref(rid)), "mce_server_submit")
        return rid.value

    def poll(self, rid: int):
        done = C.c_int()
        r = _Result()
        lat = C.c_double()
        s = lib().mce_server_poll(self.h, rid, C.byref(done), C.byref(r), C.byref(lat))
        if not done.value:
            _check(s, "mce_server_poll")
            return None
        _check(s, "request")
        return Result._from(r), lat.value

    def span(self, rid: int):
        """(start, end) of a finished request's device work, ms on the device
        clock since the server was created."""
        a, b = C.c_double(), C.c_double()
        _check(lib().mce_server_request_span(self.h, rid, C.byref(a), C.byref(b)), "mce_server_request_span")
        return a.value, b.value

    def drain(self):
        _check(lib().mce_server_drain(self.h), "mce_server_drain")

    def close(self):
        if getattr(self, "h", None):
            lib().mce_server_free(self.h)
            self.h = None

    def __del__(self):
        self.close()


def solve_file_cli(path: str, *args: str) -> str:
    """Run the RDMCE-compatible command line and return its stdout."""
    return subprocess.run([CLI_PATH, "-i", path, *args], capture_output=True, text=True, check=True).stdout
