"""CPU tests of the product boundary: the C-ABI library loads and exports
every symbol include/gpart_b200.h declares; host-only entry points; the
drop-in drivers' argument and input errors (they fail before any CUDA call);
generator determinism."""
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

import horkxg_b200 as hb
from horkxg_b200 import graphs

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "gpart_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(gp_[a-z_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    names = declared_symbols()
    assert len(names) >= 20
    out = subprocess.run(["nm", "-D", "--defined-only", str(hb.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (gp_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    lib = hb.lib()
    for n in names:
        getattr(lib, n)
    assert set(hb.EXPORTS) <= set(names)


def test_library_is_built_for_sm100a_only():
    # the build recipe compiles every CUDA source for sm_100a and nothing else
    from horkxg_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert all(flag in build.NVFLAGS for flag in build.ARCH)
    assert not any("compute_" in f and "100a" not in f for f in build.NVFLAGS)


@pytest.mark.parametrize("total,parts,ratio,expected", [(6, 2, 1.10, 3), (100, 4, 1.03, 25), (1000, 4, 1.03, 257),
                                                        (6, 2, 1.34, 4)])
def test_host_capacity(total, parts, ratio, expected):
    assert hb.capacity(total, parts, ratio) == expected


@pytest.mark.parametrize("total,parts,ratio,status", [(4, 3, 1.03, hb.GP_EINVAL), (100, 0, 1.03, hb.GP_EINVAL),
                                                      (100, 33, 1.03, hb.GP_EINVAL), (100, 4, 0.99, hb.GP_EINVAL),
                                                      (100, 4, float("nan"), hb.GP_EINVAL),
                                                      (2**64 - 1, 2, 4.0, hb.GP_EOVERFLOW)])
def test_host_capacity_rejections(total, parts, ratio, status):
    with pytest.raises(hb.PartitionError) as e:
        hb.capacity(total, parts, ratio)
    assert e.value.status == status


def driver(width="standard"):
    return str(hb.BIN / f"gpart_partition_{width}")


@pytest.mark.parametrize("width", ["standard", "big"])
def test_driver_usage_exit_code(width):
    r = subprocess.run([driver(width), "a", "b"], capture_output=True, text=True)
    assert r.returncode == 2 and "Usage:" in r.stderr


def test_driver_missing_file(tmp_path):
    r = subprocess.run([driver(), str(tmp_path / "no"), str(tmp_path / "no2"), "4", str(tmp_path / "o")],
                       capture_output=True, text=True)
    assert r.returncode == 1 and r.stderr.startswith("gpart_partition: cannot open")


def test_driver_bad_sizes(tmp_path):
    (tmp_path / "p").write_bytes(b"\0" * 12)
    (tmp_path / "i").write_bytes(b"")
    r = subprocess.run([driver(), str(tmp_path / "p"), str(tmp_path / "i"), "2", str(tmp_path / "o")],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "invalid binary size" in r.stderr
    np.array([0, 1, 1], np.int64).tofile(tmp_path / "p")
    np.array([0, 0], np.int64).tofile(tmp_path / "i")
    r = subprocess.run([driver(), str(tmp_path / "p"), str(tmp_path / "i"), "2", str(tmp_path / "o")],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "CSR offsets do not match indices" in r.stderr


def test_driver_infeasible_capacity(tmp_path):
    np.array([0, 0, 0, 0, 0], np.int64).tofile(tmp_path / "p")
    np.array([], np.int64).tofile(tmp_path / "i")
    r = subprocess.run([driver(), str(tmp_path / "p"), str(tmp_path / "i"), "3", str(tmp_path / "o")],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "capacity" in r.stderr


def test_generators_deterministic(tmp_path, monkeypatch):
    monkeypatch.setenv("GP_GRAPH_CACHE", str(tmp_path / "a"))
    a = [p.read_bytes() for p in graphs.rmat(10)]
    monkeypatch.setenv("GP_GRAPH_CACHE", str(tmp_path / "b"))
    b = [p.read_bytes() for p in graphs.rmat(10)]
    assert a == b
    off, idx = np.frombuffer(a[0], np.int64), np.frombuffer(a[1], np.int64)
    src = np.repeat(np.arange(len(off) - 1), np.diff(off))
    assert (src != idx).all()
    key = np.sort(src * (len(off) - 1) + idx)
    assert np.array_equal(key, np.sort(idx * (len(off) - 1) + src))
    assert (np.diff(key) > 0).all()


def test_grid_sizes():
    off, idx = graphs.load(*graphs.grid2d(256, 256))
    assert len(off) - 1 == 65536 and len(idx) == 261120


def symmetric_simple(off, idx):
    src = np.repeat(np.arange(len(off) - 1), np.diff(off))
    key = np.sort(src * (len(off) - 1) + idx)
    return (src != idx).all() and np.array_equal(key, np.sort(idx.astype(np.int64) * (len(off) - 1) + src)) \
        and (np.diff(key) > 0).all()


def test_in_memory_generators_match_files(tmp_path, monkeypatch):
    monkeypatch.setenv("GP_GRAPH_CACHE", str(tmp_path))
    off, idx = graphs.load(*graphs.rmat(10))
    off2, idx2 = graphs.rmat_csr(10, 16, 1)
    assert np.array_equal(off, off2) and np.array_equal(np.asarray(idx), idx2)
    a = graphs.rgg_csr(5000, 10.0, 3)
    b = graphs.rgg_csr(5000, 10.0, 3)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    assert symmetric_simple(*a) and symmetric_simple(*graphs.grid2d_csr(9, 7))


def test_packed_graph_layout():
    gs = [graphs.grid2d_csr(3, 4), graphs.rgg_csr(200, 6.0, 1), (np.zeros(4, np.int64), np.zeros(0, np.int32))]
    p = hb.PackedGraph.pack(gs)
    assert p.count == 3 and p.n == sum(len(o) - 1 for o, _ in gs) and p.m == sum(len(x) for _, x in gs)
    assert (np.diff(p.off) >= 0).all() and p.off[0] == 0 and p.off[-1] == p.m
    for i, (off, nbr) in enumerate(gs):
        o2, n2 = p.instance(i)
        assert np.array_equal(o2, off) and np.array_equal(n2, nbr)
    d = p.desc()
    assert d.index64 == 2 and d.n == p.n and d.m == p.m


def test_rgg_batch_shape(tmp_path, monkeypatch):
    monkeypatch.setenv("GP_GRAPH_CACHE", str(tmp_path))
    off, nbr, vo, ks = graphs.rgg_batch(count=6, seed=3, n_lo=100, n_hi=2000)
    assert len(vo) == 7 and vo[-1] == len(off) - 1 and off[-1] == len(nbr)
    sizes = np.diff(vo)
    assert (sizes >= 100).all() and (sizes <= 2000).all()
    assert set(ks.tolist()) <= {2, 4, 8, 16, 32}
    p = hb.PackedGraph(off, nbr, vo)
    for i in range(6):
        assert symmetric_simple(*p.instance(i))
    again = graphs.rgg_batch(count=6, seed=3, n_lo=100, n_hi=2000)
    assert all(np.array_equal(x, y) for x, y in zip((off, nbr, vo, ks), again))


def test_serving_mix_kinds():
    mix = graphs.serving_mix(6, seed=11, n_lo=1e3, n_hi=4e3)
    assert len(mix) == 6 and {k for k, *_ in mix} <= {"grid", "rgg", "rmat"}
    for kind, off, nbr, k in mix:
        assert 2 <= k <= 32 and symmetric_simple(off, nbr)


def test_footprint_projection_is_monotone():
    base = hb.footprint_bytes(1 << 20, 16 << 20, 8)
    assert hb.footprint_bytes(1 << 21, 16 << 20, 8) > base
    assert hb.footprint_bytes(1 << 20, 32 << 20, 8) > base
    assert hb.footprint_bytes(1 << 20, 16 << 20, 32) > base
    assert hb.footprint_bytes(1 << 20, 16 << 20, 8, hb.BIG) > base
