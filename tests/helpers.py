"""Graph fixtures shared by the tests (CPU-side construction only)."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def goldens() -> dict:
    return json.loads((GOLDEN / "reference_goldens.json").read_text())


def csr_from_rows(rows, weights=None):
    off = [0]
    nbr, ew = [], []
    for i, r in enumerate(rows):
        nbr.extend(r)
        if weights is not None:
            ew.extend(weights[i])
        off.append(len(nbr))
    return (np.array(off, np.int64), np.array(nbr, np.int64),
            None if weights is None else np.array(ew, np.uint64))


def symmetric_rows(n, pairs, self_loops=()):
    rows = [[] for _ in range(n)]
    for a, b in pairs:
        rows[a].append(b)
        rows[b].append(a)
    for v in self_loops:
        rows[v].append(v)
    return [sorted(r) for r in rows]


def weighted_stress(n=384, k=4, scale=1):
    """384-vertex weighted graph with unsorted duplicate entries and self
    loops (the shape of tests/test_uncoarsen.cu:488-518)."""
    rows = [[] for _ in range(n)]

    def add(a, b, w):
        rows[a].append((b, w))
        rows[b].append((a, w))
    vw = []
    for v in range(n):
        add(v, (v + 1) % n, scale * 3)
        add(v, (v + 17) % n, scale * 11)
        add(v, (v + 17) % n, scale * 7)
        add(v, v, scale * 13)
        vw.append(1 + (v // k) % 3)
    off, nbr, ew = [0], [], []
    for r in rows:
        r.reverse()
        for u, w in r:
            nbr.append(u)
            ew.append(w)
        off.append(len(nbr))
    labels = np.arange(n) % k
    return (np.array(off, np.int64), np.array(nbr, np.int64), np.array(ew, np.uint64),
            np.array(vw, np.uint64), labels.astype(np.int32))
