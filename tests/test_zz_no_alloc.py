"""The allocation-free initial partition (gp_initial_partition_static).

Callers that cannot allocate device memory -- a process whose memory belongs
to another allocator's budget, or a latency-bound caller that cannot afford
cudaMalloc -- get the spectral initial partition from a fixed scratch array
compiled into the library.  This test calls it through the C ABI on device
arrays, twice in a row (the array keeps the previous call's contents), and
checks each result against the allocating entry point gp_initial_partition:
the labels are integers, so they must be identical.  It also checks the size
limit.  Runs last so that a failure here leaves every other test already run.
"""
import ctypes

import numpy as np
import pytest

import horkxg_b200 as hb
from horkxg_b200 import graphs

pytestmark = pytest.mark.gpu


def device_graph(torch, off, nbr, ew=None, vw=None):
    t = {"off": torch.from_numpy(np.ascontiguousarray(off, np.int32)).cuda(),
         "nbr": torch.from_numpy(np.ascontiguousarray(nbr, np.int32)).cuda()}
    if ew is not None:
        t["ew"] = torch.from_numpy(np.ascontiguousarray(ew, np.uint32).view(np.int32)).cuda()
    if vw is not None:
        t["vw"] = torch.from_numpy(np.ascontiguousarray(vw, np.uint32).view(np.int32)).cuda()
    d = hb.GraphDesc()
    d.n, d.m, d.width, d.memory, d.index64 = len(off) - 1, len(nbr), hb.STANDARD, hb.DEVICE, 0
    d.offsets, d.neighbors = t["off"].data_ptr(), t["nbr"].data_ptr()
    d.edge_weights = t["ew"].data_ptr() if "ew" in t else None
    d.vertex_weights = t["vw"].data_ptr() if "vw" in t else None
    return d, t


def static_partition(torch, desc, parts, seed):
    labels = torch.full((desc.n,), -7, dtype=torch.int32, device="cuda")
    msg = ctypes.create_string_buffer(256)
    torch.cuda.synchronize()
    rc = hb.lib().gp_initial_partition_static(ctypes.byref(desc), parts, 1.03, seed, labels.data_ptr(), None, msg,
                                              len(msg))
    torch.cuda.synchronize()
    return rc, labels.cpu().numpy(), msg.value.decode()


def test_static_initial_partition_matches_allocating_entry_point():
    torch = pytest.importorskip("torch")
    # the coarsest level of an RMAT hierarchy (weighted, dense rows) and a grid
    off, idx = graphs.load(*graphs.by_name("rmat14"))
    with hb.Context(0) as ctx:
        levels = ctx.coarsen(hb.HostGraph(off, idx, index64=True), parts=32)
        coff, cnbr, cew, cvw, _ = levels[-1]
        goff, gidx = graphs.load(*graphs.by_name("grid2d_64"))
        cases = [(coff, cnbr, cew, cvw, 32, 3), (goff, np.asarray(gidx), None, None, 8, 0)]
        for off_, nbr_, ew_, vw_, parts, seed in cases:
            expected = ctx.initial_partition(hb.HostGraph(off_, nbr_, ew_, vw_, index64=True), parts, 1.03, seed)
            desc, keep = device_graph(torch, off_, nbr_, ew_, vw_)
            for _ in range(2):
                rc, labels, msg = static_partition(torch, desc, parts, seed)
                assert rc == hb.GP_OK, msg
                assert np.array_equal(labels, expected)


def test_static_initial_partition_rejects_large_graphs():
    torch = pytest.importorskip("torch")
    n = 65537
    off = np.zeros(n + 1, np.int64)
    desc, keep = device_graph(torch, off, np.zeros(1, np.int32)[:0])
    rc, _, msg = static_partition(torch, desc, 4, 0)
    assert rc == hb.GP_EINVAL and "at most 65536" in msg
