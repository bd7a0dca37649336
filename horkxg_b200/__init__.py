"""B200-native multilevel k-way graph partitioner (horkxg's SCLP coarsening,
spectral initial partition and incremental bucketed refinement).

The product is the C ABI in include/gpart_b200.h, implemented by
libgpart_b200.so, and the drop-in drivers bin/gpart_partition_{standard,big}.
This module is a thin ctypes binding of that ABI for Python callers, tests and
bench.py; it mirrors the reference's library entry points (coarsen,
aggregate, contract, initial_partition_gpu, refine_partition, partition).
Loading fails loudly when the library is missing: there is no fallback.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

# A server runs one CUDA stream per slot; with the driver's default of 8
# hardware work queues, more than 8 streams share queues and their kernels
# serialise behind each other.  The setting is read when the process creates
# its CUDA context, so it only takes effect if this module is imported before
# any CUDA work; an explicit setting is kept.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libgpart_b200.so"
BIN = PKG / "bin"

GP_OK, GP_EINVAL, GP_ERUNTIME, GP_EOVERFLOW, GP_ECUDA, GP_ETIMEOUT, GP_ENOMEM = range(7)
STANDARD, BIG = 0, 1
HOST, DEVICE = 0, 1


class GraphDesc(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("m", ctypes.c_int64), ("width", ctypes.c_int32), ("memory", ctypes.c_int32),
                ("index64", ctypes.c_int32), ("reserved", ctypes.c_int32), ("offsets", ctypes.c_void_p),
                ("neighbors", ctypes.c_void_p), ("edge_weights", ctypes.c_void_p),
                ("vertex_weights", ctypes.c_void_p)]


class Options(ctypes.Structure):
    _fields_ = [("parts", ctypes.c_int32), ("cluster_size_factor", ctypes.c_int32), ("imbalance", ctypes.c_double),
                ("seed", ctypes.c_uint32), ("verify", ctypes.c_int32), ("deterministic", ctypes.c_int32),
                ("pack_isolated", ctypes.c_int32), ("max_levels", ctypes.c_int32), ("max_rounds", ctypes.c_int32),
                ("stop_ratio", ctypes.c_double), ("growth_ratio", ctypes.c_double), ("log", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


class Report(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("m", ctypes.c_int64), ("cut", ctypes.c_uint64), ("capacity", ctypes.c_uint64),
                ("total_edge_weight", ctypes.c_uint64), ("part_weights", ctypes.c_uint64 * 32),
                ("levels", ctypes.c_int32), ("reserved", ctypes.c_int32), ("coarsest_n", ctypes.c_int64),
                ("initial_cut", ctypes.c_uint64), ("coarsen_seconds", ctypes.c_double),
                ("initial_seconds", ctypes.c_double), ("uncoarsen_seconds", ctypes.c_double),
                ("free_seconds", ctypes.c_double), ("algorithm_seconds", ctypes.c_double),
                ("prepare_seconds", ctypes.c_double)]


class RequestInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("slot", ctypes.c_int32), ("queued_seconds", ctypes.c_double),
                ("service_seconds", ctypes.c_double), ("latency_seconds", ctypes.c_double),
                ("footprint_bytes", ctypes.c_uint64), ("message", ctypes.c_char * 192)]


class PartStats(ctypes.Structure):
    _fields_ = [("vertices", ctypes.c_uint64), ("internal_edges", ctypes.c_uint64),
                ("outgoing_cut_edges", ctypes.c_uint64), ("incoming_cut_edges", ctypes.c_uint64),
                ("weighted_internal", ctypes.c_uint64), ("weighted_outgoing", ctypes.c_uint64),
                ("weighted_incoming", ctypes.c_uint64)]


class Analysis(ctypes.Structure):
    _fields_ = [("parts", ctypes.c_int32), ("reserved", ctypes.c_int32), ("directed_edge_cut", ctypes.c_uint64),
                ("weighted_directed_edge_cut", ctypes.c_uint64), ("max_local_cut", ctypes.c_uint64),
                ("weighted_max_local_cut", ctypes.c_uint64), ("avg_local_cut", ctypes.c_double),
                ("weighted_avg_local_cut", ctypes.c_double), ("vertex_avg", ctypes.c_double),
                ("min_vertices", ctypes.c_uint64), ("max_vertices", ctypes.c_uint64),
                ("vertex_imbalance", ctypes.c_double), ("vertex_max_deviation", ctypes.c_double),
                ("edge_set_avg", ctypes.c_double), ("min_edge_set", ctypes.c_uint64),
                ("max_edge_set", ctypes.c_uint64), ("edge_set_imbalance", ctypes.c_double),
                ("edge_set_max_deviation", ctypes.c_double)]


class SymmetrizeInfo(ctypes.Structure):
    _fields_ = [("self_loops_removed", ctypes.c_int64), ("unique_undirected_edges", ctypes.c_int64),
                ("output_directed_edges", ctypes.c_int64)]


class RefineStats(ctypes.Structure):
    _fields_ = [("rounds", ctypes.c_int32), ("proposals", ctypes.c_uint64), ("accepted", ctypes.c_uint64),
                ("initial_cut", ctypes.c_uint64), ("final_cut", ctypes.c_uint64),
                ("final_max_part_weight", ctypes.c_uint64), ("admission_iterations", ctypes.c_int32),
                ("admission_fallbacks", ctypes.c_int32)]


EXPORTS = ["gp_options_default", "gp_ctx_create", "gp_ctx_destroy", "gp_ctx_error", "gp_partition_capacity",
           "gp_partition", "gp_aggregate", "gp_contract", "gp_coarsen", "gp_hierarchy_levels", "gp_hierarchy_level",
           "gp_hierarchy_write", "gp_hierarchy_free", "gp_initial_partition", "gp_diffusion", "gp_refine", "gp_cut",
           "gp_launch_count", "gp_sync_count", "gp_ctx_set_sync_mode", "gp_ctx_set_device_share", "gp_ctx_set_small_diffusion", "gp_ctx_set_hub_tables", "gp_ctx_set_graph_loops", "gp_ctx_stream", "gp_profile_enable", "gp_profile_dump",
           "gp_initial_partition_static", "gp_initial_partition_trace", "gp_analyze", "gp_symmetrize", "gp_generate_rmat", "gp_partition_range", "gp_ctx_memory", "gp_ctx_trim", "gp_ctx_allocator_stats",
           "gp_footprint_bytes", "gp_server_create", "gp_server_destroy", "gp_server_error", "gp_server_submit",
           "gp_server_submit_range", "gp_server_poll", "gp_server_wait", "gp_partition_batch"]

_LIB = None


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: the CUDA library must be built (__graft_entry__.build())")
        L = ctypes.CDLL(str(LIB_PATH))
        vp, i64, i32, u32, dbl = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_uint32, ctypes.c_double
        P = ctypes.POINTER
        L.gp_options_default.argtypes = [P(Options)]
        L.gp_ctx_create.argtypes = [i32, P(vp)]
        L.gp_ctx_destroy.argtypes = [vp]
        L.gp_ctx_error.argtypes = [vp]
        L.gp_ctx_error.restype = ctypes.c_char_p
        L.gp_partition_capacity.argtypes = [ctypes.c_uint64, i32, dbl, P(ctypes.c_uint64)]
        L.gp_partition.argtypes = [vp, P(GraphDesc), P(Options), vp, P(Report)]
        L.gp_aggregate.argtypes = [vp, P(GraphDesc), i32, u32, i32, i32, i32, vp, P(i64), P(ctypes.c_uint64)]
        L.gp_contract.argtypes = [vp, P(GraphDesc), vp, i64, vp, vp, vp, vp, P(i64)]
        L.gp_coarsen.argtypes = [vp, P(GraphDesc), P(Options), P(vp)]
        L.gp_hierarchy_levels.argtypes = [vp]
        L.gp_hierarchy_level.argtypes = [vp, i32, P(i64), P(i64), vp, vp, vp, vp, vp]
        L.gp_hierarchy_write.argtypes = [vp, ctypes.c_char_p]
        L.gp_hierarchy_free.argtypes = [vp]
        L.gp_initial_partition.argtypes = [vp, P(GraphDesc), i32, dbl, u32, vp]
        L.gp_initial_partition_trace.argtypes = [vp, P(GraphDesc), i32, dbl, u32, vp, vp, i32, P(ctypes.c_int32)]
        L.gp_diffusion.argtypes = [vp, P(GraphDesc), vp, i32, u32, i32, vp]
        L.gp_refine.argtypes = [vp, P(GraphDesc), vp, i32, dbl, i32, i32, P(RefineStats)]
        L.gp_cut.argtypes = [vp, P(GraphDesc), vp, i32, P(ctypes.c_uint64), vp]
        L.gp_analyze.argtypes = [vp, P(GraphDesc), vp, i32, P(PartStats), P(Analysis)]
        L.gp_symmetrize.argtypes = [vp, P(GraphDesc), vp, vp, i32, i64, P(SymmetrizeInfo)]
        L.gp_generate_rmat.argtypes = [vp, i32, i32, dbl, dbl, dbl, ctypes.c_uint64, i32, vp, vp, i32, i64,
                                       P(SymmetrizeInfo)]
        L.gp_launch_count.argtypes = [vp]
        L.gp_launch_count.restype = ctypes.c_uint64
        L.gp_sync_count.argtypes = [vp]
        L.gp_sync_count.restype = ctypes.c_uint64
        L.gp_ctx_set_sync_mode.argtypes = [vp, i32]
        L.gp_ctx_set_device_share.argtypes = [vp, i32]
        L.gp_ctx_set_small_diffusion.argtypes = [vp, i32]
        L.gp_ctx_set_hub_tables.argtypes = [vp, i32]
        L.gp_ctx_set_graph_loops.argtypes = [vp, i32]
        L.gp_ctx_stream.argtypes = [vp]
        L.gp_ctx_stream.restype = vp
        L.gp_profile_enable.argtypes = [vp, i32]
        L.gp_profile_dump.argtypes = [vp, ctypes.c_char_p, ctypes.c_uint64]
        L.gp_initial_partition_static.argtypes = [P(GraphDesc), i32, dbl, u32, vp, vp, ctypes.c_char_p,
                                                  ctypes.c_uint64]
        u64 = ctypes.c_uint64
        L.gp_partition_range.argtypes = [vp, P(GraphDesc), i64, i64, P(Options), vp, P(Report)]
        L.gp_ctx_memory.argtypes = [vp, P(u64), P(u64), P(u64), i32]
        L.gp_ctx_trim.argtypes = [vp]
        L.gp_ctx_allocator_stats.argtypes = [vp, P(u64), P(u64), P(u64), P(dbl)]
        L.gp_footprint_bytes.argtypes = [i64, i64, i32, i32, i32]
        L.gp_footprint_bytes.restype = u64
        L.gp_server_create.argtypes = [i32, i32, u64, P(vp)]
        L.gp_server_destroy.argtypes = [vp]
        L.gp_server_error.argtypes = [vp]
        L.gp_server_error.restype = ctypes.c_char_p
        L.gp_server_submit.argtypes = [vp, P(GraphDesc), P(Options), vp, P(u64)]
        L.gp_server_submit_range.argtypes = [vp, P(GraphDesc), i64, i64, P(Options), vp, P(u64)]
        L.gp_server_poll.argtypes = [vp, u64, P(i32)]
        L.gp_server_wait.argtypes = [vp, u64, P(Report), P(RequestInfo)]
        L.gp_partition_batch.argtypes = [vp, P(GraphDesc), i32, vp, vp, vp, vp, vp]
        _LIB = L
    return _LIB


class PartitionError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


def default_options(**kw) -> Options:
    o = Options()
    lib().gp_options_default(ctypes.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def capacity(total: int, parts: int, ratio: float) -> int:
    out = ctypes.c_uint64()
    rc = lib().gp_partition_capacity(total, parts, ratio, ctypes.byref(out))
    if rc:
        raise PartitionError(rc, "invalid partition capacity")
    return out.value


def plan_depths(parts: int) -> list[list[tuple[int, int]]]:
    """The bisection task tree for `parts`, level by level: each task is
    (first_part, parts); a task of one part is a leaf and not listed."""
    levels, cur = [], [(0, parts)]
    while cur:
        levels.append(cur)
        nxt = []
        for first, p in cur:
            lp, rp = p // 2, p - p // 2
            nxt += [t for t in ((first, lp), (first + lp, rp)) if t[1] >= 2]
        cur = nxt
    return levels


class HostGraph:
    """A host CSR in one of the two widths (keeps the numpy arrays alive)."""

    def __init__(self, offsets, neighbors, edge_weights=None, vertex_weights=None, width: int = STANDARD,
                 index64: bool = False):
        self.width = width
        self.index64 = index64
        wdt = np.uint32 if width == STANDARD else np.uint64
        if index64:
            self.off = np.ascontiguousarray(offsets, dtype=np.int64)
            self.nbr = np.ascontiguousarray(neighbors, dtype=np.int64)
        else:
            self.off = np.ascontiguousarray(offsets, dtype=np.int32 if width == STANDARD else np.int64)
            self.nbr = np.ascontiguousarray(neighbors, dtype=np.int32)
        self.ew = None if edge_weights is None else np.ascontiguousarray(edge_weights, dtype=wdt)
        self.vw = None if vertex_weights is None else np.ascontiguousarray(vertex_weights, dtype=wdt)
        self.n = len(self.off) - 1
        self.m = len(self.nbr)

    def desc(self) -> GraphDesc:
        d = GraphDesc()
        d.n, d.m, d.width, d.memory, d.index64 = self.n, self.m, self.width, HOST, int(self.index64)
        d.offsets = self.off.ctypes.data
        d.neighbors = self.nbr.ctypes.data
        d.edge_weights = None if self.ew is None else self.ew.ctypes.data
        d.vertex_weights = None if self.vw is None else self.vw.ctypes.data
        return d


class PackedGraph:
    """Several graphs in one concatenated CSR: global int64 offsets into the
    concatenated neighbour array, neighbour ids local to their instance, and
    per-instance vertex offsets (the layout gp_partition_range and
    gp_partition_batch take)."""

    def __init__(self, offsets, neighbors, vertex_offsets, width: int = STANDARD):
        self.width = width
        self.off = np.ascontiguousarray(offsets, dtype=np.int64)
        self.nbr = np.ascontiguousarray(neighbors, dtype=np.int32)
        self.vertex_offsets = np.ascontiguousarray(vertex_offsets, dtype=np.int64)
        self.n = len(self.off) - 1
        self.m = len(self.nbr)
        self.count = len(self.vertex_offsets) - 1

    @classmethod
    def pack(cls, graphs, width: int = STANDARD) -> "PackedGraph":
        """graphs: iterable of (offsets, neighbours) pairs with local ids."""
        graphs = list(graphs)
        vo = np.zeros(len(graphs) + 1, np.int64)
        for i, (off, _) in enumerate(graphs):
            vo[i + 1] = vo[i] + len(off) - 1
        off_all = np.zeros(int(vo[-1]) + 1, np.int64)
        nbr_all = np.concatenate([np.asarray(nb, np.int32) for _, nb in graphs]) if graphs else np.zeros(0, np.int32)
        base = 0
        for i, (off, nb) in enumerate(graphs):
            off = np.asarray(off, np.int64)
            off_all[vo[i]:vo[i + 1] + 1] = off + base
            base += len(nb)
        return cls(off_all, nbr_all, vo, width)

    def instance(self, i: int):
        a, b = int(self.vertex_offsets[i]), int(self.vertex_offsets[i + 1])
        e0, e1 = int(self.off[a]), int(self.off[b])
        return self.off[a:b + 1] - e0, self.nbr[e0:e1]

    def desc(self) -> GraphDesc:
        # int64 offsets with int32 neighbours (index64 = 2)
        d = GraphDesc()
        d.n, d.m, d.width, d.memory, d.index64 = self.n, self.m, self.width, HOST, 2
        d.offsets = self.off.ctypes.data
        d.neighbors = self.nbr.ctypes.data
        return d


def footprint_bytes(n: int, m: int, parts: int, width: int = STANDARD, index64_host: bool = False) -> int:
    return int(lib().gp_footprint_bytes(n, m, parts, width, int(index64_host)))


class Server:
    """Continuous-batching partition server on one GPU (gp_server_*): `slots`
    contexts with their own streams, FIFO admission under a device memory
    budget."""

    def __init__(self, device: int = 0, slots: int = 8, memory_budget: int = 120 << 30):
        self._h = ctypes.c_void_p()
        rc = lib().gp_server_create(device, slots, memory_budget, ctypes.byref(self._h))
        if rc:
            raise PartitionError(rc, "cannot create server")
        self._live = {}

    def close(self):
        if self._h:
            lib().gp_server_destroy(self._h)
            self._h = ctypes.c_void_p()
            self._live.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, g: HostGraph, options: Options | None = None, **kw) -> int:
        o = options or default_options(**kw)
        labels = np.zeros(g.n, np.int32)
        d = g.desc()
        t = ctypes.c_uint64()
        rc = lib().gp_server_submit(self._h, ctypes.byref(d), ctypes.byref(o), labels.ctypes.data, ctypes.byref(t))
        if rc:
            raise PartitionError(rc, lib().gp_server_error(self._h).decode())
        self._live[t.value] = (g, d, o, labels)
        return t.value

    def poll(self, ticket: int) -> bool:
        done = ctypes.c_int32()
        rc = lib().gp_server_poll(self._h, ticket, ctypes.byref(done))
        if rc:
            raise PartitionError(rc, "unknown ticket")
        return bool(done.value)

    def wait(self, ticket: int):
        """Returns (labels, report, info); raises on a failed request."""
        rep, info = Report(), RequestInfo()
        rc = lib().gp_server_wait(self._h, ticket, ctypes.byref(rep), ctypes.byref(info))
        g, d, o, labels = self._live.pop(ticket, (None, None, None, None))
        if rc:
            raise PartitionError(rc, info.message.decode() or "unknown ticket")
        return labels, rep, info

    def partition_batch(self, packed: PackedGraph, options=None):
        """Partition every instance of a packed CSR; options: one Options or a
        list of them.  Returns (labels of all instances, list of reports)."""
        count = packed.count
        if options is None:
            options = default_options()
        if isinstance(options, Options):
            options = [options] * count
        opts = (Options * max(count, 1))(*options)
        reps = (Report * max(count, 1))()
        st = np.zeros(max(count, 1), np.int32)
        labels = np.zeros(packed.n, np.int32)
        d = packed.desc()
        rc = lib().gp_partition_batch(self._h, ctypes.byref(d), count, packed.vertex_offsets.ctypes.data, opts,
                                      labels.ctypes.data, reps, st.ctypes.data)
        if rc:
            raise PartitionError(rc, lib().gp_server_error(self._h).decode())
        return labels, [reps[i] for i in range(count)]


class Context:
    """One GPU context (stream + memory pool).  Not thread-safe."""

    def __init__(self, device: int = 0):
        self._h = ctypes.c_void_p()
        rc = lib().gp_ctx_create(device, ctypes.byref(self._h))
        if rc:
            raise PartitionError(rc, "cannot create context")

    def close(self):
        if self._h:
            lib().gp_ctx_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int):
        if rc:
            raise PartitionError(rc, lib().gp_ctx_error(self._h).decode())

    @property
    def launches(self) -> int:
        return int(lib().gp_launch_count(self._h))

    @property
    def syncs(self) -> int:
        return int(lib().gp_sync_count(self._h))

    def set_small_diffusion(self, enable: bool):
        """One-block diffusion for small coarsest graphs (same values)."""
        self._check(lib().gp_ctx_set_small_diffusion(self._h, int(enable)))

    def set_hub_tables(self, on_chip: bool):
        """On-chip hub hash tables where they fit (same hierarchy)."""
        self._check(lib().gp_ctx_set_hub_tables(self._h, int(on_chip)))

    def set_graph_loops(self, mode: int):
        """Rebalance loop of the default mode as a CUDA graph: 0 never (host
        loop, the default), 1 once a level's host loop ran 8 iterations, 2 always."""
        self._check(lib().gp_ctx_set_graph_loops(self._h, int(mode)))

    def set_device_share(self, share: int):
        """Contexts expected to run at once on the device (grid sizing only)."""
        self._check(lib().gp_ctx_set_device_share(self._h, int(share)))

    def set_sync_mode(self, blocking: bool):
        """Host waits sleep (True) or poll (False, the default)."""
        self._check(lib().gp_ctx_set_sync_mode(self._h, int(blocking)))

    @property
    def stream(self) -> int:
        return int(lib().gp_ctx_stream(self._h) or 0)

    def profile(self, on: bool):
        self._check(lib().gp_profile_enable(self._h, int(on)))

    def profile_dump(self) -> dict:
        buf = ctypes.create_string_buffer(1 << 16)
        self._check(lib().gp_profile_dump(self._h, buf, len(buf)))
        out = {}
        for line in buf.value.decode().splitlines():
            name, launches, ms, nbytes = line.split()
            out[name] = {"launches": int(launches), "ms": float(ms), "bytes": float(nbytes)}
        return out

    def partition_desc(self, desc: GraphDesc, labels_ptr: int, options: Options):
        """Partition a graph described by a raw GraphDesc (host or device
        pointers); labels_ptr is in the graph's memory space."""
        rep = Report()
        self._check(lib().gp_partition(self._h, ctypes.byref(desc), ctypes.byref(options), labels_ptr,
                                       ctypes.byref(rep)))
        return rep

    def partition(self, g: HostGraph, options: Options | None = None, **kw):
        o = options or default_options(**kw)
        labels = np.zeros(g.n, np.int32)
        rep = Report()
        d = g.desc()
        self._check(lib().gp_partition(self._h, ctypes.byref(d), ctypes.byref(o), labels.ctypes.data,
                                       ctypes.byref(rep)))
        return labels, rep

    def partition_range(self, packed: PackedGraph, i: int, options: Options | None = None, **kw):
        """Partition instance i of a packed CSR, as gp_partition would alone."""
        o = options or default_options(**kw)
        a, b = int(packed.vertex_offsets[i]), int(packed.vertex_offsets[i + 1])
        labels = np.zeros(b - a, np.int32)
        rep = Report()
        d = packed.desc()
        self._check(lib().gp_partition_range(self._h, ctypes.byref(d), a, b, ctypes.byref(o), labels.ctypes.data,
                                             ctypes.byref(rep)))
        return labels, rep

    def memory(self, reset_peak: bool = False) -> dict:
        live, cached, peak = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        self._check(lib().gp_ctx_memory(self._h, ctypes.byref(live), ctypes.byref(cached), ctypes.byref(peak),
                                        int(reset_peak)))
        return {"live": live.value, "cached": cached.value, "peak": peak.value}

    def allocator_stats(self) -> dict:
        """Caching-allocator counters: requests, driver allocations, cached
        blocks freed to make room, host milliseconds in the allocator."""
        r, a, f, ms = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_double()
        self._check(lib().gp_ctx_allocator_stats(self._h, ctypes.byref(r), ctypes.byref(a), ctypes.byref(f),
                                                 ctypes.byref(ms)))
        return {"requests": r.value, "driver_allocs": a.value, "cache_frees": f.value, "host_ms": ms.value}

    def trim(self):
        self._check(lib().gp_ctx_trim(self._h))

    def aggregate(self, g: HostGraph, parts: int, seed: int, level: int, cluster_size_factor: int = 256,
                  pack_isolated: bool = False):
        mp = np.zeros(g.n, np.int32)
        cn, cap = ctypes.c_int64(), ctypes.c_uint64()
        d = g.desc()
        self._check(lib().gp_aggregate(self._h, ctypes.byref(d), parts, seed, level, cluster_size_factor,
                                       int(pack_isolated), mp.ctypes.data, ctypes.byref(cn), ctypes.byref(cap)))
        return mp, cn.value, cap.value

    def contract(self, g: HostGraph, mp, coarse_n: int):
        mp = np.ascontiguousarray(mp, np.int32)
        off = np.zeros(coarse_n + 1, np.int64)
        nbr = np.zeros(max(g.m, 1), np.int32)
        ew = np.zeros(max(g.m, 1), np.uint64)
        vw = np.zeros(coarse_n, np.uint64)
        cm = ctypes.c_int64()
        d = g.desc()
        self._check(lib().gp_contract(self._h, ctypes.byref(d), mp.ctypes.data, coarse_n, off.ctypes.data,
                                      nbr.ctypes.data, ew.ctypes.data, vw.ctypes.data, ctypes.byref(cm)))
        return off, nbr[:cm.value].copy(), ew[:cm.value].copy(), vw

    def coarsen(self, g: HostGraph, options: Options | None = None, **kw):
        """Returns a list of levels (offsets, neighbors, edge_weights,
        vertex_weights, map_to_next or None)."""
        o = options or default_options(**kw)
        h = ctypes.c_void_p()
        d = g.desc()
        self._check(lib().gp_coarsen(self._h, ctypes.byref(d), ctypes.byref(o), ctypes.byref(h)))
        try:
            L = lib()
            count = L.gp_hierarchy_levels(h)
            out = []
            for i in range(count):
                n, m = ctypes.c_int64(), ctypes.c_int64()
                L.gp_hierarchy_level(h, i, ctypes.byref(n), ctypes.byref(m), None, None, None, None, None)
                off = np.zeros(n.value + 1, np.int64)
                nbr = np.zeros(max(m.value, 1), np.int32)
                ew = np.zeros(max(m.value, 1), np.uint64)
                vw = np.zeros(n.value, np.uint64)
                mp = np.zeros(n.value, np.int32) if i + 1 < count else None
                L.gp_hierarchy_level(h, i, None, None, off.ctypes.data, nbr.ctypes.data, ew.ctypes.data,
                                     vw.ctypes.data, None if mp is None else mp.ctypes.data)
                out.append((off, nbr[:m.value], ew[:m.value], vw, mp))
            return out
        finally:
            lib().gp_hierarchy_free(h)

    def coarsen_to_file(self, g: HostGraph, path, options: Options | None = None, **kw) -> int:
        """Coarsens and writes the hierarchy in the reference's file layout
        (include/hierarchy.hpp:42-126); returns the number of levels."""
        o = options or default_options(**kw)
        h = ctypes.c_void_p()
        d = g.desc()
        self._check(lib().gp_coarsen(self._h, ctypes.byref(d), ctypes.byref(o), ctypes.byref(h)))
        try:
            if lib().gp_hierarchy_write(h, str(path).encode()) != GP_OK:
                raise PartitionError(GP_ERUNTIME, f"cannot write {path}")
            return lib().gp_hierarchy_levels(h)
        finally:
            lib().gp_hierarchy_free(h)

    def initial_partition(self, g: HostGraph, parts: int, ratio: float = 1.03, seed: int = 0):
        labels = np.zeros(g.n, np.int32)
        d = g.desc()
        self._check(lib().gp_initial_partition(self._h, ctypes.byref(d), parts, ratio, seed, labels.ctypes.data))
        return labels

    def initial_partition_trace(self, g: HostGraph, parts: int, ratio: float = 1.03, seed: int = 0):
        """Labels plus the FP32 diffusion value of every vertex at every
        recursion depth (rows of a depths x n array, NaN outside open tasks)."""
        labels = np.zeros(g.n, np.int32)
        depths = ctypes.c_int32()
        d = g.desc()
        rows = len(plan_depths(min(max(parts, 2), 32)))
        trace = np.zeros((rows, g.n), np.float32)
        self._check(lib().gp_initial_partition_trace(self._h, ctypes.byref(d), parts, ratio, seed,
                                                     labels.ctypes.data, trace.ctypes.data, rows,
                                                     ctypes.byref(depths)))
        return labels, trace[:depths.value]

    def diffusion(self, g: HostGraph, labels, group: int, seed: int, steps: int = 64):
        labels = np.ascontiguousarray(labels, np.int32)
        x = np.zeros(g.n, np.float32)
        d = g.desc()
        self._check(lib().gp_diffusion(self._h, ctypes.byref(d), labels.ctypes.data, group, seed, steps,
                                       x.ctypes.data))
        return x

    def refine(self, g: HostGraph, labels, parts: int, ratio: float = 1.03, max_rounds: int = 32,
               deterministic: bool = True):
        labels = np.array(labels, dtype=np.int32, copy=True)
        st = RefineStats()
        d = g.desc()
        self._check(lib().gp_refine(self._h, ctypes.byref(d), labels.ctypes.data, parts, ratio, max_rounds,
                                    int(deterministic), ctypes.byref(st)))
        return labels, st

    def cut(self, g: HostGraph, labels, parts: int):
        labels = np.ascontiguousarray(labels, np.int32)
        c = ctypes.c_uint64()
        loads = np.zeros(parts, np.uint64)
        d = g.desc()
        self._check(lib().gp_cut(self._h, ctypes.byref(d), labels.ctypes.data, parts, ctypes.byref(c),
                                 loads.ctypes.data))
        return c.value, loads

    def analyze(self, g: HostGraph, labels, parts: int):
        """The reference analyzer's report on the GPU: (per-part stats as a
        dict of uint64 arrays, summary dict)."""
        labels = np.ascontiguousarray(labels, np.int32)
        st = (PartStats * parts)()
        a = Analysis()
        d = g.desc()
        self._check(lib().gp_analyze(self._h, ctypes.byref(d), labels.ctypes.data, parts, st, ctypes.byref(a)))
        per = {f: np.array([getattr(x, f) for x in st], np.uint64) for f, _ in PartStats._fields_}
        return per, {f: getattr(a, f) for f, _ in Analysis._fields_ if f != "reserved"}

    def symmetrize(self, g: HostGraph, neighbor_bytes: int = 8):
        """The reference symmetriser's output on the GPU: (int64 offsets,
        neighbours (int64 or int32), SymmetrizeInfo)."""
        off = np.zeros(g.n + 1, np.int64)
        nbr = np.zeros(max(2 * g.m, 1), np.int64 if neighbor_bytes == 8 else np.int32)
        info = SymmetrizeInfo()
        d = g.desc()
        self._check(lib().gp_symmetrize(self._h, ctypes.byref(d), off.ctypes.data, nbr.ctypes.data, neighbor_bytes,
                                        2 * g.m, ctypes.byref(info)))
        return off, nbr[:info.output_directed_edges].copy(), info

    def generate_rmat(self, scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
                      seed: int = 1, neighbor_bytes: int = 8):
        """R-MAT generated and symmetrised on the GPU, copied to the host."""
        n = 1 << scale
        off = np.zeros(n + 1, np.int64)
        nbr = np.zeros(2 * n * edge_factor, np.int64 if neighbor_bytes == 8 else np.int32)
        info = SymmetrizeInfo()
        self._check(lib().gp_generate_rmat(self._h, scale, edge_factor, a, b, c, seed, HOST, off.ctypes.data,
                                           nbr.ctypes.data, neighbor_bytes, len(nbr), ctypes.byref(info)))
        return off, nbr[:info.output_directed_edges].copy(), info
