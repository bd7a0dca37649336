#!/usr/bin/env python3
"""Generate the golden vectors that pin the oracle and the B200 build.

Runs the reference's own sm_100a binaries (compiled from its sources by
``oracle/Makefile`` into ``oracle/_ref/``) on seeded synthetic fixtures and
records:

* per-level SHA-256 digests of the SCLP hierarchy (the reference's
  ``write_hierarchy`` byte layout, ``include/hierarchy.hpp:42-126``) for the
  production coarsening options of ``app/partition_main.cu:53-55`` and, for
  the cycle+hub fixture, the library defaults used by
  ``tests/test_uncoarsen.cu:233-285``;
* ``final_edge_cut`` and timings of ``gpart_partition_*`` for seeds 0-4.

Needs a GPU.  Usage: ``python tests/golden/make_golden.py --out DIR``; the JSON
written to DIR/reference_goldens.json is committed as
``tests/golden/reference_goldens.json``.  With ``--scale`` it records the
same digests for the configured sizes instead (RMAT-20 at seeds 0-2, RMAT-22
k=32, the 320^3 grid at big width) plus the RMAT-20 cuts at seeds 0-4, into
DIR/reference_goldens_scale.json (committed as
``tests/golden/reference_goldens_scale.json``); the hierarchy files, several
GB, are deleted after hashing.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import re
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from horkxg_b200 import graphs  # noqa: E402

REF = ROOT / "oracle" / "_ref"

HIERARCHY_CASES = [
    # fixture, parts, seed, beta (-1 = production), pack_isolated, variant
    ("grid2d_256", 4, 0, -1, 1, "standard"),
    ("grid2d_256", 4, 1, -1, 1, "standard"),
    ("grid2d_256", 4, 2, -1, 1, "standard"),
    ("grid2d_64", 2, 0, -1, 1, "standard"),
    ("grid2d_64", 8, 3, -1, 1, "standard"),
    ("grid3d_24", 8, 0, -1, 1, "standard"),
    ("grid3d_24", 8, 0, -1, 1, "big"),
    ("rmat12", 8, 0, -1, 1, "standard"),
    ("rmat14", 32, 0, -1, 1, "standard"),
    ("rmat14", 4, 5, -1, 1, "big"),
    ("rmat16", 32, 0, -1, 1, "standard"),
    ("rgg_20k", 8, 0, -1, 1, "standard"),
    ("rgg_20k", 16, 4, -1, 0, "standard"),
    ("cycle_hub_4096", 4, 0, 256, 0, "standard"),
    ("cycle_hub_4096", 4, 0, 256, 0, "big"),
]

SCALE_HIERARCHY_CASES = [
    ("rmat20", 32, 0, -1, 1, "standard"),
    ("rmat20", 32, 1, -1, 1, "standard"),
    ("rmat20", 32, 2, -1, 1, "standard"),
    ("rmat22", 32, 0, -1, 1, "standard"),
    ("grid3d_320", 8, 0, -1, 1, "big"),
]

SCALE_PARTITION_CASES = [
    ("rmat20", 32, "standard"),
]

PARTITION_CASES = [
    ("grid2d_256", 4, "standard"),
    ("grid3d_24", 8, "standard"),
    ("rmat14", 32, "standard"),
    ("rmat16", 32, "standard"),
    ("rgg_20k", 8, "standard"),
]


def level_digests(path: Path) -> list[dict]:
    data = np.memmap(path, dtype=np.int32, mode="r")
    pos = 1
    out = []
    for level in range(int(data[0])):
        n, m = int(data[pos]), int(data[pos + 1])
        size = 2 + (n + 1) + m + m + n + (n_prev if level > 0 else 0)
        h = hashlib.sha256()
        for at in range(pos, pos + size, 1 << 26):        # in pieces: level files reach GBs
            h.update(np.ascontiguousarray(data[at:min(pos + size, at + (1 << 26))]).tobytes())
        out.append({"n": n, "m": m, "sha256": h.hexdigest()})
        pos += size
        n_prev = n
    if pos != len(data):
        raise ValueError(f"trailing data in {path}")
    return out


def file_sha256(path: Path) -> str:
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for block in iter(lambda: f.read(1 << 26), b""):
            h.update(block)
    return h.hexdigest()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", type=Path, required=True)
    ap.add_argument("--keep", action="store_true", help="keep hierarchy files under --out")
    ap.add_argument("--scale", action="store_true", help="the configured sizes instead of the small fixtures")
    args = ap.parse_args()
    args.out.mkdir(parents=True, exist_ok=True)
    hierarchy_cases = SCALE_HIERARCHY_CASES if args.scale else HIERARCHY_CASES
    partition_cases = SCALE_PARTITION_CASES if args.scale else PARTITION_CASES
    result = {"fixtures": {}, "hierarchies": [], "partitions": []}
    names = sorted({c[0] for c in hierarchy_cases} | {c[0] for c in partition_cases})
    for name in names:
        indptr, indices = graphs.by_name(name)
        result["fixtures"][name] = {
            "n": int(indptr.stat().st_size // 8 - 1),
            "m": int(indices.stat().st_size // 8),
            "sha256_indptr": file_sha256(indptr),
            "sha256_indices": file_sha256(indices),
        }
    for name, parts, seed, beta, pack, variant in hierarchy_cases:
        indptr, indices = graphs.by_name(name)
        out = args.out / f"hier_{name}_k{parts}_s{seed}_b{beta}_p{pack}_{variant}.bin"
        cmd = [str(REF / f"ref_hierarchy_{variant}"), str(indptr), str(indices), str(parts), str(seed),
               str(beta), str(pack), str(out)]
        log = subprocess.run(cmd, capture_output=True, text=True, check=True).stdout
        stop = re.findall(r"stop_reason=(\S+)", log)
        result["hierarchies"].append({
            "fixture": name, "parts": parts, "seed": seed, "beta": beta, "pack_isolated": pack,
            "variant": variant, "stop_reason": stop[-1] if stop else None,
            "levels": level_digests(out)})
        if not args.keep or out.stat().st_size > (3 << 20):
            out.unlink()
        print("hierarchy", name, parts, seed, variant, len(result["hierarchies"][-1]["levels"]), flush=True)
    for name, parts, variant in partition_cases:
        indptr, indices = graphs.by_name(name)
        for seed in range(5):
            part = Path("/tmp") / f"gp_golden_{name}_{parts}_{seed}.part"
            cmd = [str(REF / f"gpart_partition_{variant}"), str(indptr), str(indices), str(parts), str(part),
                   "1.03", str(seed)]
            t0 = time.time()
            text = subprocess.run(cmd, capture_output=True, text=True, check=True).stdout
            wall = time.time() - t0
            cut = int(re.findall(r"^final_edge_cut=(\d+)$", text, re.M)[-1])
            algo = float(re.findall(r"algorithm_total_seconds=([0-9.e+-]+)", text)[-1])
            labels = np.fromfile(part, dtype=np.int32)
            loads = np.bincount(labels, minlength=parts)
            result["partitions"].append({
                "fixture": name, "parts": parts, "variant": variant, "seed": seed, "ratio": 1.03,
                "cut": cut, "max_load": int(loads.max()), "algorithm_total_seconds": algo,
                "process_seconds": wall})
            print("partition", name, parts, seed, cut, algo, flush=True)
    target = "reference_goldens_scale.json" if args.scale else "reference_goldens.json"
    (args.out / target).write_text(json.dumps(result, indent=1) + "\n")


if __name__ == "__main__":
    main()
