"""CPU tests: the oracle pinned against the reference's golden vectors and
known-answer fixtures (tests/test_partition_capacity.cpp,
tests/test_uncoarsen.cu, tests/test_initial_partition_gpu.cu)."""
from decimal import Decimal, ROUND_FLOOR

import numpy as np
import pytest

import pyoracle as O
from horkxg_b200 import graphs
from helpers import goldens, csr_from_rows, symmetric_rows, weighted_stress

GOLD = goldens()


# --- include/partition_capacity.hpp via tests/test_partition_capacity.cpp:13-29
@pytest.mark.parametrize("total,parts,ratio,expected", [(6, 2, 1.10, 3), (100, 4, 1.03, 25), (1000, 4, 1.03, 257),
                                                        (6, 2, 1.34, 4)])
def test_capacity_known_answers(total, parts, ratio, expected):
    assert O.partition_capacity(total, parts, ratio) == expected


@pytest.mark.parametrize("total,parts,ratio", [(4, 3, 1.03), (100, 0, 1.03), (100, 33, 1.03), (100, 4, 0.99),
                                               (100, 4, float("nan"))])
def test_capacity_rejections(total, parts, ratio):
    with pytest.raises(O.OracleError) as e:
        O.partition_capacity(total, parts, ratio)
    assert e.value.code == 1


def test_capacity_overflow():
    with pytest.raises(O.OracleError) as e:
        O.partition_capacity(2**64 - 1, 2, 4.0)
    assert e.value.code == 3


@pytest.mark.parametrize("n", [65536, 4194304, 100003])
@pytest.mark.parametrize("parts", [2, 4, 8, 32])
def test_capacity_matches_decimal_floor(n, parts):
    # tools/verify_partition.py:55 computes floor(Decimal(ratio) * n / k)
    expected = int((Decimal("1.03") * n / parts).to_integral_value(rounding=ROUND_FLOOR))
    assert O.partition_capacity(n, parts, 1.03) == expected


# --- golden hierarchies of the reference's sm_100a build
@pytest.mark.parametrize("case", GOLD["hierarchies"],
                         ids=lambda h: f"{h['fixture']}-k{h['parts']}-s{h['seed']}-{h['variant']}")
def test_oracle_hierarchy_matches_reference(case):
    off, idx = graphs.load(*graphs.by_name(case["fixture"]))
    levels, maps = O.coarsen(O.Graph(off, np.asarray(idx)), case["parts"], case["seed"], case["beta"],
                             bool(case["pack_isolated"]))
    assert O.hierarchy_file_digests(levels, maps) == case["levels"]


def test_fixture_generators_are_stable():
    import hashlib
    for name, meta in GOLD["fixtures"].items():
        indptr, indices = graphs.by_name(name)
        assert hashlib.sha256(indptr.read_bytes()).hexdigest() == meta["sha256_indptr"], name
        assert hashlib.sha256(indices.read_bytes()).hexdigest() == meta["sha256_indices"], name


# --- contraction, tests/test_uncoarsen.cu:163-231
def contraction_fixture(groups, n=35, weight=3):
    mapping = np.arange(n) % groups
    rows, ws = [], []
    expected = {}
    for v in range(n):
        r, w = [], []
        for u in range(n - 1):
            if v >= n - 1:
                break
            for _ in range(2):
                r.append(u)
                w.append(weight)
                if mapping[v] != mapping[u]:
                    expected[(mapping[v], mapping[u])] = expected.get((mapping[v], mapping[u]), 0) + weight
        rows.append(r)
        ws.append(w)
    off, nbr, ew = csr_from_rows(rows, ws)
    return off, nbr, ew, mapping, expected


@pytest.mark.parametrize("groups", [7, 1])
def test_oracle_contraction_fixture(groups):
    off, nbr, ew, mapping, expected = contraction_fixture(groups)
    c = O.contract(O.Graph(off, nbr, ew), mapping, groups)
    got = {}
    for s in range(groups):
        for e in range(c.off[s], c.off[s + 1]):
            got[(s, int(c.nbr[e]))] = int(c.ew[e])
        assert list(c.nbr[c.off[s]:c.off[s + 1]]) == sorted(c.nbr[c.off[s]:c.off[s + 1]])
    assert got == expected
    assert list(c.vw) == list(np.bincount(mapping, minlength=groups))


def test_oracle_identity_contraction():
    off = np.array([0, 1, 3, 5, 6]); nbr = np.array([1, 0, 2, 1, 3, 2]); ew = np.array([1, 1, 5, 5, 10, 10])
    c = O.contract(O.Graph(off, nbr, ew), np.arange(4), 4)
    assert list(c.off) == list(off) and list(c.nbr) == list(nbr) and list(c.ew) == list(ew)
    e = O.contract(O.Graph(np.zeros(5, np.int64), np.zeros(0, np.int64)), np.arange(4), 4)
    assert list(e.off) == [0] * 5 and len(e.nbr) == 0


# --- isolated packing, tests/test_uncoarsen.cu:53-76
def test_oracle_isolated_packing():
    vw = np.array([7, 7, 1, 4, 4, 1, 1, 8, 1, 3, 6, 2], np.uint64)
    off = np.array([0, 1, 2] + [2] * 10, np.int64)
    g = O.Graph(off, np.array([1, 0]), np.array([3, 3]), vw)
    _, before, _ = O.aggregate(g, 2, 0, 0, 2, False)
    mp, after, cap = O.aggregate(g, 2, 0, 0, 2, True)
    assert after < before
    assert np.bincount(mp, weights=vw.astype(float)).max() <= cap
    assert mp[0] != mp[1]
    assert all(mp[v] not in (mp[0], mp[1]) for v in range(2, 12))


# --- initial partition, tests/test_initial_partition_gpu.cu:34-99
def two_cliques(vw=2, ew=3):
    rows = [[u for u in range(8) if u != v and u // 4 == v // 4] for v in range(8)]
    off, nbr, _ = csr_from_rows(rows)
    return O.Graph(off, nbr, np.full(len(nbr), ew), np.full(8, vw))


def hub_path_259():
    rows = []
    for v in range(259):
        r = []
        if v == 0:
            for u in range(1, 258):
                r += [u, u]
        if 0 < v < 258:
            r += [0, 0]
        if 1 < v < 258:
            r.append(v - 1)
        if 0 < v < 257:
            r.append(v + 1)
        rows.append(sorted(r))
    off, nbr, _ = csr_from_rows(rows)
    return O.Graph(off, nbr, np.full(len(nbr), 7))


def test_oracle_initial_partition_fixtures():
    g = two_cliques()
    lab = O.initial_partition(g, 2)
    assert O.recount(g, lab, 2)[0] == 0
    iso = O.Graph(np.zeros(13, np.int64), np.zeros(0, np.int64))
    lab = O.initial_partition(iso, 3)
    assert np.bincount(lab, minlength=3).max() <= O.partition_capacity(12, 3, 1.03)
    hp = hub_path_259()
    for k in (2, 3, 4, 8):
        lab = O.initial_partition(hp, k)
        assert np.bincount(lab, minlength=k).max() <= O.partition_capacity(259, k, 1.03)
    lab = O.initial_partition(O.Graph(np.zeros(257, np.int64), np.zeros(0, np.int64)), 32)
    assert np.bincount(lab, minlength=32).max() <= O.partition_capacity(256, 32, 1.03)


def test_oracle_initial_partition_rejections():
    heavy = np.ones(256, np.uint64); heavy[0] = 1000
    with pytest.raises(O.OracleError) as e:
        O.initial_partition(O.Graph(np.zeros(257, np.int64), np.zeros(0, np.int64), None, heavy), 3, 1.10)
    assert e.value.code == 1
    with pytest.raises(O.OracleError) as e:
        O.initial_partition(O.Graph(np.zeros(5, np.int64), np.zeros(0, np.int64)), 3, 1.03)
    assert e.value.code == 1
    with pytest.raises(O.OracleError) as e:
        O.initial_partition(O.Graph(np.zeros(4, np.int64), np.zeros(0, np.int64), None, np.full(3, 2)), 2, 1.03)
    assert e.value.code == 2


# --- refinement, tests/test_uncoarsen.cu:456-518
EXCHANGE = dict(off=[0, 2, 5, 7, 10, 11, 12], nbr=[1, 3, 0, 2, 4, 1, 3, 0, 2, 5, 1, 3],
                ew=[1, 4, 1, 4, 100, 4, 1, 4, 1, 100, 100, 100], labels=[0, 0, 1, 1, 0, 1])
REPAIR = dict(off=[0, 2, 4, 5, 5, 7, 8, 8, 8], nbr=[1, 4, 0, 2, 1, 0, 5, 4], ew=[1, 4, 1, 100, 100, 4, 100, 100],
              labels=[0, 0, 0, 0, 1, 1, 1, 1])


def test_oracle_refine_exchange():
    g = O.Graph(EXCHANGE["off"], EXCHANGE["nbr"], EXCHANGE["ew"])
    lab, st = O.refine(g, EXCHANGE["labels"], 2, 1.03, 32)
    assert O.recount(g, lab, 2)[0] // 2 == 2 and (lab == 0).sum() == 3


def test_oracle_refine_repair():
    g = O.Graph(REPAIR["off"], REPAIR["nbr"], REPAIR["ew"])
    lab, st = O.refine(g, REPAIR["labels"], 2, 1.03, 32)
    assert O.recount(g, lab, 2)[0] // 2 == 1 and (lab == 0).sum() == 4 and st.admission_iterations > 0


@pytest.mark.parametrize("k", [2, 4, 8, 32])
def test_oracle_refine_weighted_stress(k):
    off, nbr, ew, vw, labels = weighted_stress(k=k)
    g = O.Graph(off, nbr, ew, vw)
    before = O.recount(g, labels, k)[0]
    lab, st = O.refine(g, labels, k, 1.03, 32)
    cut, loads = O.recount(g, lab, k)
    assert cut <= before
    assert loads.max() <= O.partition_capacity(int(vw.sum()), k, 1.03)


def test_oracle_recount_matches_numpy():
    off, idx = graphs.load(*graphs.by_name("rmat12"))
    idx = np.asarray(idx)
    rng = np.random.default_rng(3)
    lab = rng.integers(0, 8, len(off) - 1).astype(np.int32)
    cut, loads = O.recount(O.Graph(off, idx), lab, 8)
    src = np.repeat(np.arange(len(off) - 1), np.diff(off))
    assert cut == int((lab[src] != lab[idx]).sum())
    assert list(loads) == list(np.bincount(lab, minlength=8))


def test_oracle_partition_quality_near_reference():
    # the CPU port (FP64 diffusion, deterministic ranking) lands near the
    # reference's median cut on the small grid
    off, idx = graphs.load(*graphs.by_name("grid2d_256"))
    g = O.Graph(off, np.asarray(idx))
    lab, cut = O.partition(g, 4, 1.03, 0)
    ref = sorted(p["cut"] for p in GOLD["partitions"] if p["fixture"] == "grid2d_256")
    assert cut <= 1.10 * ref[len(ref) // 2]
    assert np.bincount(lab).max() <= O.partition_capacity(len(off) - 1, 4, 1.03)


def test_oracle_initial_partition_replay_on_its_own_vector():
    # one bisection: a trace holding the FP64 root vector in FP32 gives the
    # FP64 recursion's split (the grid's vector has no near-ties at the split)
    off, idx = graphs.load(*graphs.by_name("grid2d_64"))
    g = O.Graph(off, np.asarray(idx))
    for seed in (0, 3):
        x = O.diffusion(g, np.zeros(g.n, np.int32), 0, seed, 64).astype(np.float32)
        labels, err = O.initial_partition_replay(g, 2, x[None, :], 1.03, seed)
        assert np.array_equal(labels, O.initial_partition(g, 2, 1.03, seed))
        assert err < 1e-6


def test_oracle_partition_from_its_own_initial_partition():
    off, idx = graphs.load(*graphs.by_name("rmat12"))
    g = O.Graph(off, np.asarray(idx))
    levels, _ = O.coarsen(g, 8)
    init = O.initial_partition(levels[-1], 8)
    assert np.array_equal(O.partition_from(g, 8, init)[0], O.partition(g, 8)[0])


def test_oracle_symmetrize_matches_reference_tool(tmp_path):
    # the numpy restatement against the reference's own CPU tool, built from
    # its source by oracle/Makefile (graph_untils/csr_symmetrize.cpp)
    import subprocess
    from pathlib import Path
    tool = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "csr_symmetrize"
    if not tool.exists():
        pytest.skip("the reference tool is built only where its sources are present")
    rng = np.random.default_rng(11)
    n = 700
    deg = rng.integers(0, 15, n)
    off = np.zeros(n + 1, np.int64)
    off[1:] = np.cumsum(deg)
    idx = rng.integers(0, n, int(off[-1])).astype(np.int64)
    idx[::11] = np.repeat(np.arange(n), deg)[::11]
    off.tofile(tmp_path / "p.bin")
    idx.tofile(tmp_path / "i.bin")
    out = subprocess.run([str(tool), "--indptr", str(tmp_path / "p.bin"), "--indices", str(tmp_path / "i.bin"),
                          "--output-dir", str(tmp_path / "o"), "--output-name", "g"], capture_output=True,
                         text=True, check=True).stdout
    eo, ei, loops = O.symmetrize(off, idx)
    assert np.array_equal(np.fromfile(tmp_path / "o" / "g_indptr.bin", np.int64), eo)
    assert np.array_equal(np.fromfile(tmp_path / "o" / "g_indices.bin", np.int64), ei)
    assert f"self_loops_removed: {loops}" in out
