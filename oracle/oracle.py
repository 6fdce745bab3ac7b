"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: tests/, ``__graft_entry__.smoke()`` and bench.py's
CPU-baseline leg import this module as the checker; the product package never
does.  The C code it wraps restates the RDMCE reference's host loader
(src/graph.cc), degeneracy order (src/graph.cc:281-306) and edge-rooted bitmap
Bron-Kerbosch with pivot (src/kernels/BkPivotBitBalance.cuh) on the CPU.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_CPU = os.path.join(HERE, "_ref", "ref_cpu")
REF_GPU = os.path.join(HERE, "_ref", "rdmce_ref_gpu")
HIST_LEN = 8192


class _Result(C.Structure):
    _fields_ = [
        ("count", C.c_uint64),
        ("checksum", C.c_uint64),
        ("nodes", C.c_uint64),
        ("pivot_words", C.c_uint64),
        ("filter_rows", C.c_uint64),
        ("build_bytes", C.c_uint64),
        ("max_size", C.c_uint32),
        ("pad", C.c_uint32),
        ("hist", C.c_uint64 * HIST_LEN),
    ]


@dataclass
class OracleResult:
    count: int
    checksum: int
    hist: dict = field(default_factory=dict)
    max_size: int = 0
    nodes: int = 0
    pivot_words: int = 0
    filter_rows: int = 0
    build_bytes: int = 0


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P, U32, U64, I = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int
        sig = {
            "og_mix64": (U64, [U64]),
            "og_parse_text": (I, [C.c_char_p, C.POINTER(P), C.POINTER(P), C.POINTER(U64)]),
            "og_free_buf": (None, [P]),
            "og_from_pairs": (P, [P, P, U64]),
            "og_from_csr": (P, [U32, P, P, P]),
            "og_free": (None, [P]),
            "og_num_vertices": (U32, [P]),
            "og_num_edges": (U64, [P]),
            "og_max_degree": (U32, [P]),
            "og_degeneracy": (U32, [P]),
            "og_export": (None, [P, P, P, P]),
            "og_sort_degeneracy": (None, [P]),
            "og_sort_gpu_rounds": (None, [P]),
            "og_apply_order": (I, [P, P]),
            "og_core_numbers": (None, [P, P]),
            "og_root": (None, [P, U64, C.POINTER(U32), C.POINTER(U32)]),
            "og_mce": (I, [P, U64, U64, I, I, C.POINTER(_Result)]),
            "og_mce_roots": (I, [P, P, U64, I, P, P]),
            "og_mce_root_set": (I, [P, P, U64, I, P, P, C.POINTER(_Result)]),
            "og_mce_roots_timed": (I, [P, P, U64, I, C.c_double, C.POINTER(_Result), C.POINTER(U64),
                                       C.POINTER(C.c_double)]),
            "og_list_cliques": (I, [P, C.c_char_p]),
            "og_store_bin": (I, [P, C.c_char_p]),
            "og_root_sizes": (None, [P, U64, U64, P, P, P]),
            "og_root_sizes_list": (None, [P, P, U64, P, P, P]),
            "og_load_bin": (P, [C.c_char_p]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def parse_text(path: str):
    L = lib()
    pu, pv, n = C.c_void_p(), C.c_void_p(), C.c_uint64()
    rc = L.og_parse_text(path.encode(), C.byref(pu), C.byref(pv), C.byref(n))
    if rc != 0:
        raise OSError(f"og_parse_text({path}) failed: {rc}")
    cnt = n.value
    u = np.ctypeslib.as_array(C.cast(pu, C.POINTER(C.c_uint32)), shape=(max(cnt, 1),))[:cnt].copy()
    v = np.ctypeslib.as_array(C.cast(pv, C.POINTER(C.c_uint32)), shape=(max(cnt, 1),))[:cnt].copy()
    L.og_free_buf(pu)
    L.og_free_buf(pv)
    return u, v


class Graph:
    """A host graph built with the reference loader conventions."""

    def __init__(self, handle):
        if not handle:
            raise ValueError("oracle graph construction failed")
        self.h = handle

    @classmethod
    def from_pairs(cls, u, v):
        u = np.ascontiguousarray(u, dtype=np.uint32)
        v = np.ascontiguousarray(v, dtype=np.uint32)
        return cls(lib().og_from_pairs(_ptr(u), _ptr(v), len(u)))

    @classmethod
    def from_csr(cls, off, adj, labels=None):
        off = np.ascontiguousarray(off, dtype=np.uint64)
        adj = np.ascontiguousarray(adj, dtype=np.uint32)
        lab = None if labels is None else np.ascontiguousarray(labels, dtype=np.uint32)
        return cls(lib().og_from_csr(len(off) - 1, _ptr(off), _ptr(adj), None if lab is None else _ptr(lab)))

    @classmethod
    def from_text(cls, path):
        u, v = parse_text(path)
        return cls.from_pairs(u, v)

    @classmethod
    def load_bin(cls, path):
        return cls(lib().og_load_bin(path.encode()))

    def __del__(self):
        if getattr(self, "h", None):
            lib().og_free(self.h)
            self.h = None

    @property
    def n(self):
        return lib().og_num_vertices(self.h)

    @property
    def m(self):
        return lib().og_num_edges(self.h)

    @property
    def max_degree(self):
        return lib().og_max_degree(self.h)

    @property
    def degeneracy(self):
        return lib().og_degeneracy(self.h)

    def sort_degeneracy(self):
        lib().og_sort_degeneracy(self.h)
        return self

    def sort_gpu_rounds(self):
        """The engine's round-synchronous peel order: after this, root ids (and
        the whole CSR) agree with the engine's for the same input."""
        lib().og_sort_gpu_rounds(self.h)
        return self

    def apply_order(self, order):
        order = np.ascontiguousarray(order, dtype=np.uint32)
        if lib().og_apply_order(self.h, _ptr(order)) != 0:
            raise ValueError("not a permutation")
        return self

    def core_numbers(self):
        out = np.zeros(self.n, dtype=np.uint32)
        lib().og_core_numbers(self.h, _ptr(out))
        return out

    def export(self):
        off = np.zeros(self.n + 1, dtype=np.uint64)
        adj = np.zeros(2 * self.m, dtype=np.uint32)
        lab = np.zeros(self.n, dtype=np.uint32)
        lib().og_export(self.h, _ptr(off), _ptr(adj), _ptr(lab))
        return off, adj, lab

    def root(self, r):
        a, b = C.c_uint32(), C.c_uint32()
        lib().og_root(self.h, r, C.byref(a), C.byref(b))
        return a.value, b.value

    def mce(self, begin=0, end=None, threads=1, expand_r=True) -> OracleResult:
        res = _Result()
        end = self.m if end is None else end
        lib().og_mce(self.h, begin, end, threads, 1 if expand_r else 0, C.byref(res))
        hist = {s: int(res.hist[s]) for s in range(HIST_LEN) if res.hist[s]}
        return OracleResult(res.count, res.checksum, hist, res.max_size, res.nodes, res.pivot_words,
                            res.filter_rows, res.build_bytes)

    def mce_roots(self, roots, threads=1):
        roots = np.ascontiguousarray(roots, dtype=np.uint64)
        cnt = np.zeros(len(roots), dtype=np.uint64)
        chk = np.zeros(len(roots), dtype=np.uint64)
        if lib().og_mce_roots(self.h, _ptr(roots), len(roots), threads, _ptr(cnt), _ptr(chk)) != 0:
            raise ValueError("root id out of range")
        return cnt, chk

    def mce_root_set(self, roots, threads=1):
        """Per-root counts and checksums plus the merged result (histogram
        included) over an explicit root list."""
        roots = np.ascontiguousarray(roots, dtype=np.uint64)
        cnt = np.zeros(len(roots), dtype=np.uint64)
        chk = np.zeros(len(roots), dtype=np.uint64)
        res = _Result()
        if lib().og_mce_root_set(self.h, _ptr(roots), len(roots), threads, _ptr(cnt), _ptr(chk),
                                 C.byref(res)) != 0:
            raise ValueError("root id out of range")
        hist = {s: int(res.hist[s]) for s in range(HIST_LEN) if res.hist[s]}
        return cnt, chk, OracleResult(res.count, res.checksum, hist, res.max_size, res.nodes, res.pivot_words,
                                      res.filter_rows, res.build_bytes)

    def mce_roots_timed(self, roots, threads, seconds):
        """Cliques found under the listed roots within `seconds` (all threads);
        returns (OracleResult so far, roots started, elapsed seconds)."""
        roots = np.ascontiguousarray(roots, dtype=np.uint64)
        res = _Result()
        started, el = C.c_uint64(), C.c_double()
        if lib().og_mce_roots_timed(self.h, _ptr(roots), len(roots), threads, seconds, C.byref(res),
                                    C.byref(started), C.byref(el)) != 0:
            raise ValueError("root id out of range")
        hist = {s: int(res.hist[s]) for s in range(HIST_LEN) if res.hist[s]}
        return (OracleResult(res.count, res.checksum, hist, res.max_size, res.nodes, res.pivot_words,
                             res.filter_rows, res.build_bytes), started.value, el.value)

    def root_sizes_list(self, roots):
        """Candidate-column count p of each listed root's ego network."""
        roots = np.ascontiguousarray(roots, dtype=np.uint64)
        p = np.zeros(len(roots), np.uint32)
        x = np.zeros(len(roots), np.uint32)
        xc = np.zeros(len(roots), np.uint32)
        lib().og_root_sizes_list(self.h, _ptr(roots), len(roots), _ptr(p), _ptr(x), _ptr(xc))
        return p

    def list_cliques(self, path):
        if lib().og_list_cliques(self.h, path.encode()) != 0:
            raise OSError(path)

    def store_bin(self, path):
        if lib().og_store_bin(self.h, path.encode()) != 0:
            raise OSError(path)


def mix64(x: int) -> int:
    return lib().og_mix64(x)


def clique_hash(labels) -> int:
    """Set hash of one clique given its original labels (any order)."""
    G = 0x9E3779B97F4A7C15
    M = (1 << 64) - 1
    s1 = s2 = 0
    for l in labels:
        s1 = (s1 + mix64(int(l))) & M
        s2 = (s2 + mix64(int(l) ^ G)) & M
    rot = ((s2 << 31) | (s2 >> 33)) & M
    return mix64(s1 ^ rot ^ ((len(labels) << 56) & M))


def run_ref_cpu(mode: str, path: str, *extra) -> dict:
    """Run the reference's own CPU code (oracle/_ref/ref_cpu) and parse its RESULT line."""
    out = subprocess.run([REF_CPU, mode, path, *map(str, extra)], capture_output=True, text=True, check=True)
    res = {}
    for line in out.stdout.splitlines():
        if line.startswith("RESULT") or line.startswith("n "):
            toks = line.split()
            start = 1 if toks[0] == "RESULT" else 0
            for k, v in zip(toks[start::2], toks[start + 1::2]):
                res[k] = float(v) if "." in v else int(v)
    return res
