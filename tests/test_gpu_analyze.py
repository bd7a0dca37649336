"""The GPU analyzer (gp_analyze) against the reference's own CPU analyzer
(graph_untils/analyze_partition.cpp, built from its source into
oracle/_ref/analyze_partition) run on the same CSR files and labels: the
per-part counts (|V(pi)|, |E(pi)|, internal, outgoing and incoming cut
entries, local cut) must be equal, and the summary figures equal to the six
decimals the analyzer prints.  Also a numpy restatement on weighted inputs and
the rejection of labels outside [0, parts)."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import horkxg_b200 as hb
from horkxg_b200 import graphs

pytestmark = pytest.mark.gpu
ANALYZER = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "analyze_partition"


def reference_report(indptr, indices, labels, parts, tmp_path):
    txt = tmp_path / "labels.txt"
    txt.write_text("\n".join(map(str, labels.tolist())) + "\n")
    out = subprocess.run([str(ANALYZER), "--partition", str(txt), "--indptr", str(indptr), "--indices",
                          str(indices), "--parts", str(parts), "--detail"], capture_output=True, text=True,
                         check=True).stdout
    def section(title):   # the lines between a section's title line and the next blank line
        lines = out.split(f"=========== {title} ===========\n", 1)[1].splitlines()
        return lines[:lines.index("")] if "" in lines else lines
    rows = [list(map(int, line.split())) for line in section("Per-Part Metrics: Counts")[1:]]
    quality = section("Partition Quality")[1].split()
    return np.array(rows, np.int64), {"edge_cut": int(quality[2]), "vertex_imb": float(quality[4]),
                                      "edge_imb": float(quality[5]), "avg_local_cut": float(quality[6]),
                                      "max_local_cut": int(quality[7])}


@pytest.mark.parametrize("name,k", [("rmat16", 8), ("grid2d_256", 4), ("rmat14", 32)])
def test_analyze_matches_reference_analyzer(ctx, name, k, tmp_path):
    indptr, indices = graphs.by_name(name)
    off, idx = graphs.load(indptr, indices)
    g = hb.HostGraph(off, idx, index64=True)
    labels, rep = ctx.partition(g, parts=k)
    per, summary = ctx.analyze(g, labels, k)
    rows, quality = reference_report(indptr, indices, labels, k, tmp_path)
    local = per["outgoing_cut_edges"] + per["incoming_cut_edges"]
    edge_set = per["internal_edges"] + local
    mine = np.stack([np.arange(k), per["vertices"], edge_set, per["internal_edges"], per["outgoing_cut_edges"],
                     per["incoming_cut_edges"], local], axis=1).astype(np.int64)
    assert np.array_equal(mine, rows)
    assert summary["directed_edge_cut"] == quality["edge_cut"] == 2 * rep.cut
    assert summary["max_local_cut"] == quality["max_local_cut"]
    for key, ref in (("vertex_imbalance", "vertex_imb"), ("edge_set_imbalance", "edge_imb"),
                     ("avg_local_cut", "avg_local_cut")):
        assert f"{summary[key]:.6f}" == f"{quality[ref]:.6f}"
    # unit weights: the weighted figures equal the counts
    assert np.array_equal(per["weighted_outgoing"], per["outgoing_cut_edges"])


def test_analyze_weighted_matches_numpy(ctx):
    rng = np.random.default_rng(5)
    off, idx = graphs.load(*graphs.by_name("rmat16"))     # 17 rows above the hub threshold
    idx = np.asarray(idx)
    n, m = len(off) - 1, len(idx)
    # symmetric weights: w(u,v) = w(v,u) from a hash of the unordered pair
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(off))
    lo, hi = np.minimum(src, idx), np.maximum(src, idx)
    ew = ((lo * 2654435761 + hi * 40503) % 97 + 1).astype(np.uint64)
    k = 6
    labels = rng.integers(0, k, n).astype(np.int32)
    per, summary = ctx.analyze(hb.HostGraph(off, idx, ew, width=hb.BIG, index64=True), labels, k)
    sp, dp = labels[src], labels[idx]
    inside = sp == dp
    assert np.array_equal(per["vertices"], np.bincount(labels, minlength=k))
    assert np.array_equal(per["internal_edges"], np.bincount(sp[inside], minlength=k))
    assert np.array_equal(per["outgoing_cut_edges"], np.bincount(sp[~inside], minlength=k))
    assert np.array_equal(per["incoming_cut_edges"], np.bincount(dp[~inside], minlength=k))
    w = ew.astype(np.float64)
    assert np.array_equal(per["weighted_internal"], np.bincount(sp[inside], w[inside], k).astype(np.uint64))
    assert np.array_equal(per["weighted_outgoing"], np.bincount(sp[~inside], w[~inside], k).astype(np.uint64))
    assert np.array_equal(per["weighted_incoming"], np.bincount(dp[~inside], w[~inside], k).astype(np.uint64))
    assert summary["directed_edge_cut"] == int((~inside).sum())
    assert summary["weighted_directed_edge_cut"] == int(w[~inside].sum())


def test_analyze_rejects_labels_out_of_range(ctx):
    off, idx = graphs.load(*graphs.by_name("grid2d_64"))
    labels = np.zeros(len(off) - 1, np.int32)
    labels[7] = 4
    with pytest.raises(hb.PartitionError) as e:
        ctx.analyze(hb.HostGraph(off, idx, index64=True), labels, 4)
    assert e.value.status == hb.GP_EINVAL and "partition id" in str(e.value)
    labels[7] = 3
    per, _ = ctx.analyze(hb.HostGraph(off, idx, index64=True), labels, 4)
    assert per["vertices"].sum() == len(off) - 1
