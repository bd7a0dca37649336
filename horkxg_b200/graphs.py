"""Synthetic workloads in the partitioner's on-disk input format.

Each generator writes native-endian int64 ``indptr``/``indices`` files (the
format read by the reference's ``gpart_partition_*`` drivers, ``src/graph.cpp``
lines 47-122) and caches them by parameters, so both the B200 build and the
reference binary read byte-identical inputs.  Generation is done by the
multithreaded C++ code in ``csrc/gen.cpp``.
"""
from __future__ import annotations

import ctypes
import math
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        path = _HERE / "libgpgen.so"
        if not path.exists():
            raise RuntimeError(f"{path} is missing; run __graft_entry__.build()")
        lib = ctypes.CDLL(str(path))
        i64p = ctypes.POINTER(ctypes.c_int64)
        lib.gp_gen_last_error.restype = ctypes.c_char_p
        lib.gp_gen_grid2d.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.c_char_p, ctypes.c_char_p, i64p, i64p]
        lib.gp_gen_grid3d.argtypes = [ctypes.c_int64] * 3 + [ctypes.c_char_p, ctypes.c_char_p, i64p, i64p]
        lib.gp_gen_rmat.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_char_p,
                                    i64p, i64p]
        lib.gp_gen_rgg.argtypes = [ctypes.c_int64, ctypes.c_double, ctypes.c_uint64, ctypes.c_char_p,
                                   ctypes.c_char_p, i64p, i64p]
        vp = ctypes.c_void_p
        lib.gp_gen_grid2d_new.argtypes = [ctypes.c_int64, ctypes.c_int64, i64p, i64p]
        lib.gp_gen_grid2d_new.restype = vp
        lib.gp_gen_rmat_new.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_uint64, i64p, i64p]
        lib.gp_gen_rmat_new.restype = vp
        lib.gp_gen_rgg_new.argtypes = [ctypes.c_int64, ctypes.c_double, ctypes.c_uint64, i64p, i64p]
        lib.gp_gen_rgg_new.restype = vp
        lib.gp_gen_copy.argtypes = [vp, vp, vp, ctypes.c_int]
        lib.gp_gen_free.argtypes = [vp]
        _LIB = lib
    return _LIB


def cache_dir() -> Path:
    root = Path(os.environ.get("GP_GRAPH_CACHE", "/tmp/gp_graphs"))
    root.mkdir(parents=True, exist_ok=True)
    return root


def _run(name: str, fn, *args) -> tuple[Path, Path]:
    root = cache_dir() / name
    root.mkdir(parents=True, exist_ok=True)
    indptr, indices = root / "indptr.bin", root / "indices.bin"
    if indptr.exists() and indices.exists():
        return indptr, indices
    n, m = ctypes.c_int64(), ctypes.c_int64()
    rc = fn(*args, str(indptr).encode(), str(indices).encode(), ctypes.byref(n), ctypes.byref(m))
    if rc != 0:
        raise RuntimeError(_lib().gp_gen_last_error().decode())
    return indptr, indices


def grid2d(nx: int, ny: int) -> tuple[Path, Path]:
    return _run(f"grid2d_{nx}x{ny}", _lib().gp_gen_grid2d, nx, ny)


def grid3d(nx: int, ny: int, nz: int) -> tuple[Path, Path]:
    return _run(f"grid3d_{nx}x{ny}x{nz}", _lib().gp_gen_grid3d, nx, ny, nz)


def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
         seed: int = 1) -> tuple[Path, Path]:
    name = f"rmat_s{scale}_ef{edge_factor}_{a}_{b}_{c}_seed{seed}"
    return _run(name, _lib().gp_gen_rmat, scale, edge_factor, a, b, c, seed)


def rmat_device(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
                seed: int = 1, device: int = 0) -> tuple[Path, Path]:
    """The files of rmat() made by the GPU generator (gp_generate_rmat),
    which draws exactly the host generator's pairs and permutation: the same
    bytes under the same cache name, in seconds instead of host minutes at
    scale 26.  Needs a GPU."""
    name = f"rmat_s{scale}_ef{edge_factor}_{a}_{b}_{c}_seed{seed}"
    root = cache_dir() / name
    root.mkdir(parents=True, exist_ok=True)
    indptr, indices = root / "indptr.bin", root / "indices.bin"
    if indptr.exists() and indices.exists():
        return indptr, indices
    import horkxg_b200 as hb
    with hb.Context(device) as ctx:
        off, nbr, _ = ctx.generate_rmat(scale, edge_factor, a, b, c, seed)
    for path, arr in ((indptr, off), (indices, nbr)):
        tmp = path.with_suffix(".tmp")
        arr.tofile(tmp)
        tmp.rename(path)
    return indptr, indices


def rgg(n: int, mean_degree: float = 10.0, seed: int = 7) -> tuple[Path, Path]:
    radius = math.sqrt(mean_degree / (math.pi * n))
    return _run(f"rgg_n{n}_deg{mean_degree}_seed{seed}", _lib().gp_gen_rgg, n, radius, seed)


def write_csr(name: str, offsets, indices) -> tuple[Path, Path]:
    """Write an explicit int64 CSR (used for small hand-made fixtures)."""
    root = cache_dir() / name
    root.mkdir(parents=True, exist_ok=True)
    indptr, idx = root / "indptr.bin", root / "indices.bin"
    np.asarray(offsets, dtype=np.int64).tofile(indptr)
    np.asarray(indices, dtype=np.int64).tofile(idx)
    return indptr, idx


def load(indptr: Path, indices: Path) -> tuple[np.ndarray, np.ndarray]:
    """Memory-map an int64 CSR pair."""
    off = np.fromfile(indptr, dtype=np.int64)
    idx = np.memmap(indices, dtype=np.int64, mode="r") if os.path.getsize(indices) else np.zeros(0, np.int64)
    return off, idx


def _in_memory(make, *args) -> tuple[np.ndarray, np.ndarray]:
    """Run an in-memory generator: int64 offsets and int32 neighbours."""
    L = _lib()
    n, m = ctypes.c_int64(), ctypes.c_int64()
    h = make(*args, ctypes.byref(n), ctypes.byref(m))
    if not h:
        raise RuntimeError(L.gp_gen_last_error().decode())
    try:
        off = np.empty(n.value + 1, np.int64)
        nbr = np.empty(m.value, np.int32)
        if L.gp_gen_copy(h, off.ctypes.data, nbr.ctypes.data, 4) != 0:
            raise RuntimeError(L.gp_gen_last_error().decode())
    finally:
        L.gp_gen_free(h)
    return off, nbr


def rgg_csr(n: int, mean_degree: float = 10.0, seed: int = 7):
    radius = math.sqrt(mean_degree / (math.pi * n))
    return _in_memory(_lib().gp_gen_rgg_new, n, radius, seed)


def grid2d_csr(nx: int, ny: int):
    return _in_memory(_lib().gp_gen_grid2d_new, nx, ny)


def rmat_csr(scale: int, edge_factor: int = 16, seed: int = 1):
    return _in_memory(_lib().gp_gen_rmat_new, scale, edge_factor, 0.57, 0.19, 0.19, seed)


def rgg_batch(count: int = 512, seed: int = 7, n_lo: float = 1e3, n_hi: float = 1e6,
              mean_degree: float = 10.0, parts=(2, 4, 8, 16, 32)):
    """The batched workload: `count` random geometric graphs in the unit
    square, n log-uniform in [n_lo, n_hi], radius sqrt(mean_degree/(pi n)),
    each with k drawn uniformly from `parts`; all drawn from one seeded
    stream.  Returns (packed offsets int64, neighbours int32, vertex offsets,
    ks), cached on disk by parameters."""
    name = f"rgg_batch_{count}_{seed}_{n_lo:g}_{n_hi:g}_{mean_degree:g}"
    root = cache_dir() / name
    files = [root / f for f in ("off.npy", "nbr.npy", "vo.npy", "ks.npy")]
    if all(f.exists() for f in files):
        return tuple(np.load(f) for f in files)
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(math.log(n_lo), math.log(n_hi), count)).astype(np.int64)
    ks = rng.choice(np.asarray(parts, np.int32), count)
    offs, nbrs = [], []
    for i, n in enumerate(ns):
        off, nbr = rgg_csr(int(n), mean_degree, seed * 1_000_003 + i)
        offs.append(off)
        nbrs.append(nbr)
    vo = np.zeros(count + 1, np.int64)
    vo[1:] = np.cumsum(ns)
    packed_off = np.zeros(int(vo[-1]) + 1, np.int64)
    base = 0
    for i, off in enumerate(offs):
        packed_off[vo[i]:vo[i + 1] + 1] = off + base
        base += int(off[-1])
    nbr = np.concatenate(nbrs) if nbrs else np.zeros(0, np.int32)
    root.mkdir(parents=True, exist_ok=True)
    for f, a in zip(files, (packed_off, nbr, vo, ks)):
        np.save(f, a)
    return packed_off, nbr, vo, ks


def serving_mix(count: int, seed: int = 11, n_lo: float = 1e4, n_hi: float = 4e6):
    """Request graphs of the serving workload: each drawn uniformly from
    {2D grid, RGG mean degree 10, RMAT edge factor 16} with n log-uniform in
    [n_lo, n_hi] and k uniform in [2, 32].  A grid gets side round(sqrt(n)),
    an RMAT graph scale round(log2 n).  Returns a list of
    (kind, offsets, neighbours, k)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        kind = ("grid", "rgg", "rmat")[int(rng.integers(3))]
        n = float(np.exp(rng.uniform(math.log(n_lo), math.log(n_hi))))
        k = int(rng.integers(2, 33))
        if kind == "grid":
            side = max(2, int(round(math.sqrt(n))))
            off, nbr = grid2d_csr(side, side)
        elif kind == "rgg":
            off, nbr = rgg_csr(int(n), 10.0, seed * 1_000_003 + i)
        else:
            off, nbr = rmat_csr(max(2, int(round(math.log2(n)))), 16, seed * 1_000_003 + i)
        out.append((kind, off, nbr, k))
    return out


def by_name(name: str) -> tuple[Path, Path]:
    """Named workloads shared by tests, the golden-vector script and bench.py."""
    table = {
        "grid2d_256": lambda: grid2d(256, 256),
        "grid2d_64": lambda: grid2d(64, 64),
        "grid3d_24": lambda: grid3d(24, 24, 24),
        "grid3d_320": lambda: grid3d(320, 320, 320),
        "rmat12": lambda: rmat(12),
        "rmat14": lambda: rmat(14),
        "rmat16": lambda: rmat(16),
        "rmat20": lambda: rmat(20),
        "rmat22": lambda: rmat(22),
        "rmat24": lambda: rmat(24),
        "rmat26": lambda: rmat_device(26),
        "rgg_20k": lambda: rgg(20000),
        "cycle_hub_4096": cycle_hub,
    }
    return table[name]()


def cycle_hub(n: int = 4096, spokes: int = 512) -> tuple[Path, Path]:
    """4096-cycle plus a 512-spoke hub at vertex 0 with a hub self loop: the
    unit-weight form of the reference fixture in tests/test_uncoarsen.cu:233-285."""
    rows = [[] for _ in range(n)]
    for v in range(n):
        rows[v].append((v + 1) % n)
        rows[(v + 1) % n].append(v)
    for v in range(1, spokes + 1):
        rows[0].append(v)
        rows[v].append(0)
    rows[0].append(0)
    offsets = [0]
    indices = []
    for r in rows:
        r.sort()
        indices.extend(r)
        offsets.append(len(indices))
    return write_csr(f"cycle_hub_{n}_{spokes}", offsets, indices)


def main(argv=None) -> int:
    """``python -m horkxg_b200.graphs NAME...`` generates (or finds in the
    cache) the named workloads and prints one JSON object mapping each name to
    its [indptr, indices] paths, so that a caller can get the input files
    without loading the generator library into its own process."""
    import json
    import sys
    names = sys.argv[1:] if argv is None else argv
    out = {name: [str(p) for p in by_name(name)] for name in names}
    print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
