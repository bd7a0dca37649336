"""The GPU symmetriser (gp_symmetrize) against the reference's own tool
(graph_untils/csr_symmetrize.cpp, built from its source into
oracle/_ref/csr_symmetrize): byte-identical int64 offsets and indices on
directed inputs with duplicates and self loops; and the device R-MAT
generator (gp_generate_rmat) against the host generator's files, byte for
byte.  The oracle's numpy restatement is pinned to the same tool on the CPU
(tests/test_oracle.py)."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import horkxg_b200 as hb
import pyoracle as O
from horkxg_b200 import graphs

pytestmark = pytest.mark.gpu
TOOL = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "csr_symmetrize"


def directed_input(n, max_deg, seed):
    rng = np.random.default_rng(seed)
    deg = rng.integers(0, max_deg, n)
    off = np.zeros(n + 1, np.int64)
    off[1:] = np.cumsum(deg)
    idx = rng.integers(0, n, int(off[-1])).astype(np.int64)
    src = np.repeat(np.arange(n), deg)
    idx[::13] = src[::13]                 # self loops
    idx[5::29] = idx[4::29][:len(idx[5::29])]   # repeated entries
    return off, idx


def reference_tool(off, idx, tmp_path):
    off.tofile(tmp_path / "in_indptr.bin")
    idx.tofile(tmp_path / "in_indices.bin")
    r = subprocess.run([str(TOOL), "--indptr", str(tmp_path / "in_indptr.bin"), "--indices",
                        str(tmp_path / "in_indices.bin"), "--output-dir", str(tmp_path / "out"), "--output-name", "g"],
                       capture_output=True, text=True, check=True)
    loops = int(next(line for line in r.stdout.splitlines() if line.startswith("self_loops_removed:")).split()[1])
    return (np.fromfile(tmp_path / "out" / "g_indptr.bin", np.int64),
            np.fromfile(tmp_path / "out" / "g_indices.bin", np.int64), loops)


@pytest.mark.parametrize("n,max_deg,seed", [(1000, 12, 3), (5000, 40, 4), (300, 400, 5), (1, 1, 6)])
def test_symmetrize_matches_reference_tool(ctx, n, max_deg, seed, tmp_path):
    off, idx = directed_input(n, max_deg, seed)
    ro, ri, loops = reference_tool(off, idx, tmp_path)
    g = hb.HostGraph(off, idx, index64=True)
    go, gi, info = ctx.symmetrize(g)
    assert np.array_equal(go, ro) and np.array_equal(gi, ri)
    assert (info.self_loops_removed, info.output_directed_edges) == (loops, len(ri))
    assert info.unique_undirected_edges * 2 == len(ri)
    go32, gi32, _ = ctx.symmetrize(g, neighbor_bytes=4)
    assert np.array_equal(go32, ro) and np.array_equal(gi32.astype(np.int64), ri)


def test_symmetrize_device_memory_and_capacity(ctx):
    torch = pytest.importorskip("torch")
    off, idx = directed_input(2000, 20, 7)
    eo, ei, loops = O.symmetrize(off, idx)
    d_off = torch.from_numpy(off.astype(np.int32)).cuda()
    d_idx = torch.from_numpy(idx.astype(np.int32)).cuda()
    desc = hb.GraphDesc()
    desc.n, desc.m, desc.width, desc.memory, desc.index64 = len(off) - 1, len(idx), hb.STANDARD, hb.DEVICE, 0
    desc.offsets, desc.neighbors = d_off.data_ptr(), d_idx.data_ptr()
    out_off = torch.zeros(len(off), dtype=torch.int64, device="cuda")
    out_nbr = torch.zeros(len(ei), dtype=torch.int32, device="cuda")
    info = hb.SymmetrizeInfo()
    import ctypes
    rc = hb.lib().gp_symmetrize(ctx._h, ctypes.byref(desc), out_off.data_ptr(), out_nbr.data_ptr(), 4, len(ei),
                                ctypes.byref(info))
    assert rc == hb.GP_OK
    assert np.array_equal(out_off.cpu().numpy(), eo) and np.array_equal(out_nbr.cpu().numpy(), ei)
    # one entry short: refused, sizes still reported
    rc = hb.lib().gp_symmetrize(ctx._h, ctypes.byref(desc), out_off.data_ptr(), out_nbr.data_ptr(), 4, len(ei) - 1,
                                ctypes.byref(info))
    assert rc == hb.GP_EINVAL and info.output_directed_edges == len(ei) and info.self_loops_removed == loops


@pytest.mark.parametrize("name,scale", [("rmat12", 12), ("rmat16", 16), ("rmat20", 20)])
def test_device_rmat_equals_host_generator(ctx, name, scale):
    off, idx = graphs.load(*graphs.by_name(name))
    go, gi, info = ctx.generate_rmat(scale)
    assert np.array_equal(go, off) and np.array_equal(gi, np.asarray(idx))
    assert info.output_directed_edges == len(idx)
