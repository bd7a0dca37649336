"""ctypes binding of the CPU oracle (oracle.cpp).  Test infrastructure only:
imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg."""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB = None

I64P = ctypes.POINTER(ctypes.c_int64)
I32P = ctypes.POINTER(ctypes.c_int32)
U64P = ctypes.POINTER(ctypes.c_uint64)
F64P = ctypes.POINTER(ctypes.c_double)


class RefineStats(ctypes.Structure):
    _fields_ = [("rounds", ctypes.c_int), ("proposals", ctypes.c_uint64), ("accepted", ctypes.c_uint64),
                ("initial_cut", ctypes.c_uint64), ("final_cut", ctypes.c_uint64),
                ("final_max_part_weight", ctypes.c_uint64), ("admission_iterations", ctypes.c_int),
                ("admission_fallbacks", ctypes.c_int)]


class OracleError(Exception):
    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


def lib():
    global _LIB
    if _LIB is None:
        path = _HERE / "liboracle.so"
        if not path.exists():
            raise RuntimeError(f"{path} missing: run `make -C oracle`")
        L = ctypes.CDLL(str(path))
        L.or_last_error.restype = ctypes.c_char_p
        L.or_partition_capacity.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_double, U64P]
        L.or_recount.argtypes = [ctypes.c_int64, I64P, I32P, U64P, U64P, I32P, ctypes.c_int, ctypes.c_int,
                                 U64P, U64P]
        L.or_aggregate.argtypes = [ctypes.c_int64, I64P, I32P, U64P, U64P, ctypes.c_int, ctypes.c_uint32,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_int, I32P, I64P, U64P]
        L.or_contract.argtypes = [ctypes.c_int64, I64P, I32P, U64P, U64P, I32P, ctypes.c_int64, I64P, I32P,
                                  U64P, U64P, I64P]
        L.or_coarsen.argtypes = [ctypes.c_int64, I64P, I32P, U64P, U64P, ctypes.c_int, ctypes.c_uint32,
                                 ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                 ctypes.POINTER(ctypes.c_void_p)]
        L.or_hier_levels.argtypes = [ctypes.c_void_p]
        L.or_hier_level_size.argtypes = [ctypes.c_void_p, ctypes.c_int, I64P, I64P]
        L.or_hier_level_copy.argtypes = [ctypes.c_void_p, ctypes.c_int, I64P, I32P, U64P, U64P, I32P]
        L.or_hier_write.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        L.or_hier_free.argtypes = [ctypes.c_void_p]
        L.or_diffusion.argtypes = [ctypes.c_int64, I64P, I32P, U64P, I32P, ctypes.c_int, ctypes.c_uint32,
                                   ctypes.c_int, F64P]
        L.or_initial_partition.argtypes = [ctypes.c_int64, I64P, I32P, U64P, U64P, ctypes.c_int,
                                           ctypes.c_double, ctypes.c_uint32, I32P]
        L.or_refine.argtypes = [ctypes.c_int64, I64P, I32P, U64P, U64P, I32P, ctypes.c_int, ctypes.c_double,
                                ctypes.c_int, ctypes.POINTER(RefineStats)]
        L.or_partition.argtypes = [ctypes.c_int64, I64P, I32P, U64P, U64P, ctypes.c_int, ctypes.c_double,
                                   ctypes.c_uint32, I32P, U64P]
        L.or_partition_from.argtypes = [ctypes.c_int64, I64P, I32P, U64P, U64P, ctypes.c_int, ctypes.c_double,
                                        ctypes.c_uint32, I32P, ctypes.c_int64, I32P, U64P]
        L.or_initial_partition_replay.argtypes = [ctypes.c_int64, I64P, I32P, U64P, U64P, ctypes.c_int,
                                                  ctypes.c_double, ctypes.c_uint32,
                                                  ctypes.POINTER(ctypes.c_float), ctypes.c_int, I32P, F64P]
        _LIB = L
    return _LIB


def _p(a, t):
    return None if a is None else a.ctypes.data_as(t)


def _check(rc: int):
    if rc != 0:
        raise OracleError(rc, lib().or_last_error().decode())


class Graph:
    """Host CSR in the oracle's widths (int64 offsets, int32 ids, uint64 weights)."""

    def __init__(self, offsets, neighbors, edge_weights=None, vertex_weights=None):
        self.off = np.ascontiguousarray(offsets, dtype=np.int64)
        self.nbr = np.ascontiguousarray(neighbors, dtype=np.int32)
        self.ew = None if edge_weights is None else np.ascontiguousarray(edge_weights, dtype=np.uint64)
        self.vw = None if vertex_weights is None else np.ascontiguousarray(vertex_weights, dtype=np.uint64)
        self.n = len(self.off) - 1

    def args(self):
        return (self.n, _p(self.off, I64P), _p(self.nbr, I32P), _p(self.ew, U64P), _p(self.vw, U64P))


def partition_capacity(total: int, parts: int, ratio: float) -> int:
    out = ctypes.c_uint64()
    _check(lib().or_partition_capacity(total, parts, ratio, ctypes.byref(out)))
    return out.value


def recount(g: Graph, labels, parts: int, threads: int = 8):
    labels = np.ascontiguousarray(labels, dtype=np.int32)
    cut = ctypes.c_uint64()
    loads = np.zeros(parts, dtype=np.uint64)
    _check(lib().or_recount(*g.args(), _p(labels, I32P), parts, threads, ctypes.byref(cut), _p(loads, U64P)))
    return cut.value, loads


def aggregate(g: Graph, parts: int, seed: int, level: int, beta: int = 256, pack_isolated: bool = False):
    mp = np.zeros(g.n, dtype=np.int32)
    cn, cap = ctypes.c_int64(), ctypes.c_uint64()
    _check(lib().or_aggregate(*g.args(), parts, seed, level, beta, int(pack_isolated), _p(mp, I32P),
                              ctypes.byref(cn), ctypes.byref(cap)))
    return mp, cn.value, cap.value


def contract(g: Graph, mp, coarse_n: int) -> Graph:
    m = len(g.nbr)
    mp = np.ascontiguousarray(mp, dtype=np.int32)
    off = np.zeros(coarse_n + 1, np.int64)
    nbr = np.zeros(max(m, 1), np.int32)
    ew = np.zeros(max(m, 1), np.uint64)
    vw = np.zeros(coarse_n, np.uint64)
    cm = ctypes.c_int64()
    _check(lib().or_contract(*g.args(), _p(mp, I32P), coarse_n, _p(off, I64P), _p(nbr, I32P), _p(ew, U64P),
                             _p(vw, U64P), ctypes.byref(cm)))
    return Graph(off, nbr[:cm.value].copy(), ew[:cm.value].copy(), vw)


def coarsen(g: Graph, parts: int, seed: int = 0, beta: int = -1, pack_isolated: bool = True,
            max_levels: int = 24, stop_ratio: float = 0.90):
    """Returns (levels, maps): list of Graph and list of int32 maps."""
    h = ctypes.c_void_p()
    _check(lib().or_coarsen(*g.args(), parts, seed, beta, int(pack_isolated), max_levels, stop_ratio,
                            ctypes.byref(h)))
    try:
        L = lib()
        levels, maps = [], []
        count = L.or_hier_levels(h)
        for i in range(count):
            n, m = ctypes.c_int64(), ctypes.c_int64()
            L.or_hier_level_size(h, i, ctypes.byref(n), ctypes.byref(m))
            off = np.zeros(n.value + 1, np.int64)
            nbr = np.zeros(m.value, np.int32)
            ew = np.zeros(m.value, np.uint64)
            vw = np.zeros(n.value, np.uint64)
            mp = np.zeros(n.value, np.int32) if i + 1 < count else None
            L.or_hier_level_copy(h, i, _p(off, I64P), _p(nbr, I32P), _p(ew, U64P), _p(vw, U64P), _p(mp, I32P))
            levels.append(Graph(off, nbr, ew, vw))
            if mp is not None:
                maps.append(mp)
        return levels, maps
    finally:
        lib().or_hier_free(h)


def diffusion(g: Graph, labels, group: int, seed: int, steps: int = 64):
    labels = np.ascontiguousarray(labels, dtype=np.int32)
    x = np.zeros(g.n, np.float64)
    _check(lib().or_diffusion(g.n, _p(g.off, I64P), _p(g.nbr, I32P), _p(g.ew, U64P), _p(labels, I32P), group,
                              seed, steps, _p(x, F64P)))
    return x


def initial_partition(g: Graph, parts: int, ratio: float = 1.03, seed: int = 0):
    labels = np.zeros(g.n, np.int32)
    _check(lib().or_initial_partition(*g.args(), parts, ratio, seed, _p(labels, I32P)))
    return labels


def initial_partition_replay(g: Graph, parts: int, trace, ratio: float = 1.03, seed: int = 0):
    """The initial partition's recursion with each task ordered by the traced
    FP32 vector of its depth (rows of `trace`); returns (labels, largest
    relative L2 distance of a traced vector from the FP64 diffusion)."""
    trace = np.ascontiguousarray(trace, dtype=np.float32)
    labels = np.zeros(g.n, np.int32)
    err = ctypes.c_double()
    _check(lib().or_initial_partition_replay(*g.args(), parts, ratio, seed,
                                             trace.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                             int(trace.shape[0]), _p(labels, I32P), ctypes.byref(err)))
    return labels, err.value


def refine(g: Graph, labels, parts: int, ratio: float = 1.03, max_rounds: int = 32):
    labels = np.array(labels, dtype=np.int32, copy=True)
    st = RefineStats()
    _check(lib().or_refine(*g.args(), _p(labels, I32P), parts, ratio, max_rounds, ctypes.byref(st)))
    return labels, st


def partition(g: Graph, parts: int, ratio: float = 1.03, seed: int = 0):
    labels = np.zeros(g.n, np.int32)
    cut = ctypes.c_uint64()
    _check(lib().or_partition(*g.args(), parts, ratio, seed, _p(labels, I32P), ctypes.byref(cut)))
    return labels, cut.value


def partition_from(g: Graph, parts: int, coarsest_labels, ratio: float = 1.03, seed: int = 0):
    """The oracle's pipeline (coarsen, refine the coarsest level, project and
    refine by the schedule of src/refine.cu:423-646) from given labels of the
    coarsest level."""
    cl = np.ascontiguousarray(coarsest_labels, dtype=np.int32)
    labels = np.zeros(g.n, np.int32)
    cut = ctypes.c_uint64()
    _check(lib().or_partition_from(*g.args(), parts, ratio, seed, _p(cl, I32P), len(cl), _p(labels, I32P),
                                   ctypes.byref(cut)))
    return labels, cut.value


def hierarchy_file_digests(levels, maps):
    """Per-level SHA-256 of the reference's write_hierarchy byte layout."""
    import hashlib
    out = []
    for i, g in enumerate(levels):
        parts = [np.array([g.n, len(g.nbr)], np.int32), g.off.astype(np.int32), g.nbr.astype(np.int32),
                 (g.ew if g.ew is not None else np.ones(len(g.nbr), np.uint64)).astype(np.int32),
                 (g.vw if g.vw is not None else np.ones(g.n, np.uint64)).astype(np.int32)]
        if i > 0:
            parts.append(maps[i - 1].astype(np.int32))
        blob = b"".join(p.tobytes() for p in parts)
        out.append({"n": int(g.n), "m": int(len(g.nbr)), "sha256": hashlib.sha256(blob).hexdigest()})
    return out


def symmetrize(offsets, indices):
    """The reference's CSR symmetriser (graph_untils/csr_symmetrize.cpp:
    277-538) restated with numpy: every entry (v, u), u != v, is the
    undirected edge {min, max} (:298-311); the distinct edges (:346-378) are
    written in both directions sorted by (source, neighbour) (:461-537);
    self loops are counted and dropped.  Returns (int64 offsets, int64
    indices, self loops)."""
    off = np.asarray(offsets, np.int64)
    idx = np.asarray(indices, np.int64)
    n = len(off) - 1
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(off))
    keep = src != idx
    lo, hi = np.minimum(src[keep], idx[keep]), np.maximum(src[keep], idx[keep])
    edges = np.unique(lo * n + hi)
    u, v = edges // n, edges % n
    both = np.sort(np.concatenate([u * n + v, v * n + u]))
    out_off = np.zeros(n + 1, np.int64)
    out_off[1:] = np.cumsum(np.bincount(both // n, minlength=n))
    return out_off, both % n, int((~keep).sum())
