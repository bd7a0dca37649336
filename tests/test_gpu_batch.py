"""Batching and serving on the GPU: every instance of a packed batch and every
served request gives the same result as the same graph partitioned alone
(bit-identical labels in deterministic mode), each passes the exact recount
and capacity, and the projected footprint used for admission bounds the
measured peak of the library's allocations."""
import time

import numpy as np
import pytest

import horkxg_b200 as hb
from horkxg_b200 import graphs
import pyoracle as O

pytestmark = pytest.mark.gpu


def mixed_graphs():
    """Uneven instances: grids, RGGs, RMATs, a graph with isolated vertices."""
    out = []
    out.append(graphs.grid2d_csr(40, 25))
    out.append(graphs.rgg_csr(3000, 10.0, 5))
    out.append(graphs.rmat_csr(12, 16, 3))
    out.append(graphs.grid2d_csr(7, 9))
    out.append(graphs.rgg_csr(20000, 10.0, 9))
    off, nbr = graphs.rgg_csr(1500, 2.0, 4)          # sparse: many isolated vertices
    out.append((off, nbr))
    out.append(graphs.rmat_csr(14, 16, 8))
    out.append(graphs.grid2d_csr(64, 64))
    return out


KS = [2, 4, 32, 3, 8, 5, 16, 4]


def alone(ctx, off, nbr, k, det=1):
    g = hb.HostGraph(off, nbr)
    return ctx.partition(g, parts=k, deterministic=det)


def check(off, nbr, labels, k, rep):
    cut, loads = O.recount(O.Graph(off, nbr), labels, k)
    assert cut // 2 == rep.cut
    assert loads.max() <= O.partition_capacity(len(off) - 1, k, 1.03)


def test_partition_range_equals_partition(ctx):
    gs = mixed_graphs()
    packed = hb.PackedGraph.pack(gs)
    for i in (0, 2, 5, 7):
        off, nbr = gs[i]
        la, ra = alone(ctx, off, nbr, KS[i])
        lb, rb = ctx.partition_range(packed, i, parts=KS[i], deterministic=1)
        assert np.array_equal(la, lb) and ra.cut == rb.cut


def test_batch_equals_one_by_one(ctx):
    gs = mixed_graphs()
    packed = hb.PackedGraph.pack(gs)
    opts = [hb.default_options(parts=k, deterministic=1) for k in KS]
    with hb.Server(0, slots=4, memory_budget=16 << 30) as srv:
        labels, reps = srv.partition_batch(packed, opts)
    for i, (off, nbr) in enumerate(gs):
        a, b = int(packed.vertex_offsets[i]), int(packed.vertex_offsets[i + 1])
        la, ra = alone(ctx, off, nbr, KS[i])
        assert np.array_equal(labels[a:b], la), i
        assert reps[i].cut == ra.cut
        check(off, nbr, labels[a:b], KS[i], reps[i])


def test_server_mix_equals_alone(ctx):
    gs = mixed_graphs()
    expect = [alone(ctx, off, nbr, k) for (off, nbr), k in zip(gs, KS)]
    with hb.Server(0, slots=3, memory_budget=16 << 30) as srv:
        tickets = []
        for rep in range(2):                      # each graph twice, interleaved
            for (off, nbr), k in zip(gs, KS):
                tickets.append(srv.submit(hb.HostGraph(off, nbr), parts=k, deterministic=1))
        results = [srv.wait(t) for t in tickets]
    for j, (labels, rep, info) in enumerate(results):
        i = j % len(gs)
        assert np.array_equal(labels, expect[i][0]), j
        assert rep.cut == expect[i][1].cut
        assert info.status == 0 and info.latency_seconds >= info.service_seconds > 0
        assert 0 <= info.slot < 3


def test_server_nondeterministic_results_valid():
    gs = mixed_graphs()
    with hb.Server(0, slots=4, memory_budget=16 << 30) as srv:
        tickets = [srv.submit(hb.HostGraph(off, nbr), parts=k) for (off, nbr), k in zip(gs, KS)]
        for t, (off, nbr), k in zip(tickets, gs, KS):
            labels, rep, info = srv.wait(t)
            check(off, nbr, labels, k, rep)


def test_server_admission_budget():
    off, nbr = graphs.rmat_csr(14, 16, 8)
    need = hb.footprint_bytes(len(off) - 1, len(nbr), 8)
    with hb.Server(0, slots=2, memory_budget=need - 1) as srv:
        with pytest.raises(hb.PartitionError) as e:
            srv.submit(hb.HostGraph(off, nbr), parts=8)
        assert e.value.status == hb.GP_ENOMEM
    # a budget for one request at a time serialises the requests
    with hb.Server(0, slots=4, memory_budget=need + need // 2) as srv:
        ts = [srv.submit(hb.HostGraph(off, nbr), parts=8, deterministic=1) for _ in range(3)]
        infos = [srv.wait(t)[2] for t in ts]
    spans = sorted((i.latency_seconds - i.service_seconds, i.latency_seconds) for i in infos)
    for (s0, e0), (s1, e1) in zip(spans, spans[1:]):
        assert s1 >= e0 - 1e-3


def test_blocking_sync_mode_same_labels(ctx):
    off, nbr = graphs.rmat_csr(13, 16, 5)
    la, ra = alone(ctx, off, nbr, 8)
    with hb.Context(0) as c:
        c.set_sync_mode(True)
        s0 = c.syncs
        lb, rb = alone(c, off, nbr, 8)
        assert c.syncs > s0
    assert np.array_equal(la, lb) and ra.cut == rb.cut


def test_device_share_same_labels(ctx):
    """Smaller grids for contexts that share the device change no result."""
    off, nbr = graphs.rmat_csr(14, 16, 8)
    la, ra = alone(ctx, off, nbr, 16)
    with hb.Context(0) as c:
        c.set_device_share(8)
        lb, rb = alone(c, off, nbr, 16)
    assert np.array_equal(la, lb) and ra.cut == rb.cut


@pytest.mark.parametrize("make,k", [(lambda: graphs.rmat_csr(16, 16, 1), 32), (lambda: graphs.grid2d_csr(300, 300), 4),
                                    (lambda: graphs.rgg_csr(100000, 10.0, 3), 16)])
def test_footprint_bounds_measured_peak(make, k):
    off, nbr = make()
    with hb.Context(0) as c:
        c.memory(reset_peak=True)
        c.partition(hb.HostGraph(off, nbr), parts=k)
        peak = c.memory()["peak"]
    assert peak <= hb.footprint_bytes(len(off) - 1, len(nbr), k)
