"""Host-side logic that needs no GPU: the packed multi-graph layout, the
batched workload's generator, the projected footprint used for serving
admission, and the bench's roofline arithmetic."""
import sys
from pathlib import Path

import numpy as np

import horkxg_b200 as hb
from horkxg_b200 import graphs

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))


def test_packed_graph_layout_round_trips():
    gs = [graphs.grid2d_csr(5, 4), graphs.rgg_csr(300, 6.0, 2), graphs.grid2d_csr(3, 3)]
    p = hb.PackedGraph.pack(gs)
    assert p.count == 3 and p.n == sum(len(o) - 1 for o, _ in gs) and p.m == sum(len(x) for _, x in gs)
    assert list(np.diff(p.vertex_offsets)) == [len(o) - 1 for o, _ in gs]
    for i, (off, nbr) in enumerate(gs):
        o, x = p.instance(i)
        assert np.array_equal(np.asarray(o) - o[0], off) and np.array_equal(x, nbr)


def test_rgg_batch_is_seeded_and_in_range(tmp_path, monkeypatch):
    monkeypatch.setenv("GP_GRAPH_CACHE", str(tmp_path))
    a = graphs.rgg_batch(count=6, seed=7, n_lo=1e3, n_hi=5e3)
    b = graphs.rgg_batch(count=6, seed=7, n_lo=1e3, n_hi=5e3)   # from the cache
    off, nbr, vo, ks = a
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    ns = np.diff(vo)
    assert len(ns) == 6 and ns.min() >= 1000 and ns.max() <= 5000
    assert set(ks.tolist()) <= {2, 4, 8, 16, 32}
    assert off[0] == 0 and off[-1] == len(nbr) and np.all(np.diff(off) >= 0)
    for i in range(6):                       # neighbour ids local to the instance
        seg = nbr[off[vo[i]]:off[vo[i + 1]]]
        assert seg.size == 0 or (seg.min() >= 0 and seg.max() < ns[i])


def test_footprint_grows_with_the_graph():
    f = hb.footprint_bytes
    base = f(100_000, 1_000_000, 8)
    assert f(200_000, 1_000_000, 8) > base
    assert f(100_000, 2_000_000, 8) > base
    assert f(100_000, 1_000_000, 32) > base
    assert f(100_000, 1_000_000, 8, hb.BIG) > base


def test_roofline_picks_the_top_modelled_kernel():
    import bench
    prof = {"a_kernel": {"launches": 10, "ms": 5.0, "bytes": 0.0},        # no model: skipped
            "hub_insert_kernel": {"launches": 4, "ms": 2.0, "bytes": 4e9},
            "cut_kernel": {"launches": 2, "ms": 1.0, "bytes": 5e9}}
    r = bench.roofline(prof, 8000.0, "measured")
    assert r["kernel"] == "hub_insert_kernel"
    assert abs(r["achieved"] - 2000.0) < 1e-6 and abs(r["frac"] - 0.25) < 1e-9
    assert r["algorithmic_bytes_per_launch"] == 1e9
    assert r["traffic"] == round(bench.DRAM_PER_ALGORITHMIC_BYTE["hub_insert_kernel"] * 1e9)
    assert abs(r["share_of_gpu_time"] - 2.0 / 8.0) < 1e-9
