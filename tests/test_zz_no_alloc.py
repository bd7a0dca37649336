"""The allocation-free initial partition (gp_initial_partition_static).

Callers that cannot allocate device memory -- a process whose memory belongs
to another allocator's budget, or a latency-bound caller that cannot afford
cudaMalloc -- get the spectral initial partition from a fixed scratch array
compiled into the library.  These tests call it through the C ABI on device
arrays, twice in a row (the array keeps the previous call's contents), and
check each result against the allocating entry point gp_initial_partition:
the labels are integers, so they must be identical.  They also check that
repeated calls leave the device's free memory unchanged, the size limit, and
that a malformed CSR is rejected by the bounds checks before any kernel reads
through it.  The file runs last so that a failure here leaves every other
test already run.
"""
import ctypes

import numpy as np
import pytest

import horkxg_b200 as hb
from horkxg_b200 import graphs

pytestmark = pytest.mark.gpu


def device_graph(torch, off, nbr, ew=None, vw=None, width=None):
    width = hb.STANDARD if width is None else width
    odt, wdt, wview = (np.int32, np.uint32, np.int32) if width == hb.STANDARD else (np.int64, np.uint64, np.int64)
    t = {"off": torch.from_numpy(np.ascontiguousarray(off, odt)).cuda(),
         "nbr": torch.from_numpy(np.ascontiguousarray(nbr, np.int32)).cuda()}
    if ew is not None:
        t["ew"] = torch.from_numpy(np.ascontiguousarray(ew, wdt).view(wview)).cuda()
    if vw is not None:
        t["vw"] = torch.from_numpy(np.ascontiguousarray(vw, wdt).view(wview)).cuda()
    d = hb.GraphDesc()
    d.n, d.m, d.width, d.memory, d.index64 = len(off) - 1, len(nbr), width, hb.DEVICE, 0
    d.offsets, d.neighbors = t["off"].data_ptr(), t["nbr"].data_ptr()
    d.edge_weights = t["ew"].data_ptr() if "ew" in t else None
    d.vertex_weights = t["vw"].data_ptr() if "vw" in t else None
    return d, t


def static_partition(torch, desc, parts, seed, labels=None):
    if labels is None:
        labels = torch.full((desc.n,), -7, dtype=torch.int32, device="cuda")
    else:
        labels.fill_(-7)
    msg = ctypes.create_string_buffer(256)
    torch.cuda.synchronize()
    rc = hb.lib().gp_initial_partition_static(ctypes.byref(desc), parts, 1.03, seed, labels.data_ptr(), None, msg,
                                              len(msg))
    torch.cuda.synchronize()
    return rc, labels.cpu().numpy(), msg.value.decode()


def coarsest_rmat14(ctx):
    off, idx = graphs.load(*graphs.by_name("rmat14"))
    levels = ctx.coarsen(hb.HostGraph(off, idx, index64=True), parts=32)
    coff, cnbr, cew, cvw, _ = levels[-1]
    return coff, cnbr, cew, cvw


@pytest.mark.parametrize("width", ["standard", "big"])
def test_static_initial_partition_matches_allocating_entry_point(width):
    torch = pytest.importorskip("torch")
    w = hb.STANDARD if width == "standard" else hb.BIG
    with hb.Context(0) as ctx:
        # the coarsest level of an RMAT hierarchy (weighted, dense rows) and a grid
        coff, cnbr, cew, cvw = coarsest_rmat14(ctx)
        goff, gidx = graphs.load(*graphs.by_name("grid2d_64"))
        cases = [(coff, cnbr, cew, cvw, 32, 3), (goff, np.asarray(gidx), None, None, 8, 0)]
        for off_, nbr_, ew_, vw_, parts, seed in cases:
            expected = ctx.initial_partition(hb.HostGraph(off_, nbr_, ew_, vw_, index64=True, width=w), parts, 1.03,
                                             seed)
            desc, keep = device_graph(torch, off_, nbr_, ew_, vw_, width=w)
            for _ in range(2):
                rc, labels, msg = static_partition(torch, desc, parts, seed)
                assert rc == hb.GP_OK, msg
                assert np.array_equal(labels, expected)


def test_static_initial_partition_allocates_nothing():
    torch = pytest.importorskip("torch")
    with hb.Context(0) as ctx:
        coff, cnbr, cew, cvw = coarsest_rmat14(ctx)
    desc, keep = device_graph(torch, coff, cnbr, cew, cvw)
    labels = torch.empty(desc.n, dtype=torch.int32, device="cuda")
    rc, first, msg = static_partition(torch, desc, 32, 1, labels)     # warm: symbol lookup, module load
    assert rc == hb.GP_OK, msg
    free_before = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        rc, again, msg = static_partition(torch, desc, 32, 1, labels)
        assert rc == hb.GP_OK, msg
        assert np.array_equal(again, first)
    assert torch.cuda.mem_get_info()[0] == free_before


def test_static_initial_partition_rejects_large_graphs():
    torch = pytest.importorskip("torch")
    n = 65537
    off = np.zeros(n + 1, np.int64)
    desc, keep = device_graph(torch, off, np.zeros(1, np.int32)[:0])
    rc, _, msg = static_partition(torch, desc, 4, 0)
    assert rc == hb.GP_EINVAL and "at most 65536" in msg


def test_static_initial_partition_rejects_malformed_csr():
    torch = pytest.importorskip("torch")
    off, idx = graphs.load(*graphs.by_name("grid2d_64"))
    n = len(off) - 1
    bad_nbr = np.asarray(idx).copy()
    bad_nbr[len(bad_nbr) // 2] = n                       # one neighbour id equal to n
    desc, keep = device_graph(torch, off, bad_nbr)
    rc, _, msg = static_partition(torch, desc, 4, 0)
    assert rc == hb.GP_EINVAL and "neighbor out of range" in msg
    bad_off = off.copy()
    bad_off[n // 2] = bad_off[n // 2 + 1] + 1            # offsets not monotone
    desc, keep = device_graph(torch, bad_off, np.asarray(idx))
    rc, _, msg = static_partition(torch, desc, 4, 0)
    assert rc == hb.GP_EINVAL
    # the entry point still works after the rejections
    desc, keep = device_graph(torch, off, np.asarray(idx))
    rc, _, msg = static_partition(torch, desc, 4, 0)
    assert rc == hb.GP_OK, msg
