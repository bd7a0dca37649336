import numpy as np
import pytest

import horkxg_b200 as hb
from horkxg_b200 import graphs
import pyoracle as O

pytestmark = pytest.mark.gpu


def load(name, width=hb.STANDARD):
    off, idx = graphs.load(*graphs.by_name(name))
    return off, np.asarray(idx), hb.HostGraph(off, idx, width=width, index64=True)


@pytest.mark.parametrize("name,k", [("grid2d_64", 2), ("rmat12", 8)])
def test_aggregate_matches_oracle(ctx, name, k):
    off, idx, g = load(name)
    mp, cn, cap = ctx.aggregate(g, k, 0, 0, 256, True)
    omp, ocn, ocap = O.aggregate(O.Graph(off, idx), k, 0, 0, 256, True)
    assert (cn, cap) == (ocn, ocap)
    assert np.array_equal(mp, omp)


@pytest.mark.parametrize("name,k", [("grid2d_256", 4), ("rmat14", 32)])
def test_partition_runs(ctx, name, k):
    off, idx, g = load(name)
    labels, rep = ctx.partition(g, parts=k)
    cut, loads = O.recount(O.Graph(off, idx), labels, k)
    assert cut % 2 == 0 and cut // 2 == rep.cut
    assert loads.max() <= O.partition_capacity(len(off) - 1, k, 1.03)
