"""Build recipe of the B200 partitioner (in-tree, no JIT cache).

Artifacts (all inside the package directory so they travel with the tree):
  libgpart_b200.so              CUDA library, C ABI of include/gpart_b200.h
  bin/gpart_partition_standard  drop-in drivers (app/partition_main.cu)
  bin/gpart_partition_big
  bin/gpart_coarsen_standard    hierarchy export (app/coarsen_main.cu)
  bin/gpart_coarsen_big
  libgpgen.so                   synthetic workload generators
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC"]


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _stale(target: Path, sources: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources)


def build(force: bool = False) -> None:
    headers = sorted(CSRC.glob("*.cuh")) + [ROOT / "include" / "gpart_b200.h"]
    lib = PKG / "libgpart_b200.so"
    sources = [CSRC / "gp_pipeline.cu", CSRC / "gp_serve.cpp"]
    if force or _stale(lib, [*sources, *headers]):
        _run([NVCC, *NVFLAGS, "-shared", "-I", str(ROOT / "include"), "-o", str(lib), *map(str, sources)])
    bindir = PKG / "bin"
    bindir.mkdir(exist_ok=True)
    for width, macro in (("standard", "GP_WIDTH_STANDARD"), ("big", "GP_WIDTH_BIG")):
        exe = bindir / f"gpart_partition_{width}"
        if force or _stale(exe, [CSRC / "gp_cli.cpp", lib]):
            _run([NVCC, "-O2", "-std=c++17", *ARCH, f"-DGP_DRIVER_WIDTH={macro}", "-o", str(exe),
                  str(CSRC / "gp_cli.cpp"), "-L", str(PKG), "-lgpart_b200", "-Xlinker", "-rpath=$ORIGIN/.."])
        coarsen = bindir / f"gpart_coarsen_{width}"
        if force or _stale(coarsen, [exe]):
            shutil.copy2(exe, coarsen)
    gen = PKG / "libgpgen.so"
    if force or _stale(gen, [CSRC / "gen.cpp"]):
        _run(["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-pthread", "-o", str(gen), str(CSRC / "gen.cpp")])


def build_oracle() -> None:
    """The CPU oracle (test infrastructure) and, where the reference sources
    are present, its sm_100a build under oracle/_ref."""
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "liboracle.so"], check=True)
    # the recipe builds the reference only where its sources are present
    subprocess.run(["make", "-s", "-j8", "-C", str(ROOT / "oracle"), "ref-if-present"], check=True)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
    build_oracle()
