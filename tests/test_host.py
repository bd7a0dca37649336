"""Host-side logic that needs no GPU: the bench's roofline arithmetic and workloads, and the
caching allocator's policy over a fake driver."""
import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))


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


def test_secondary_configs_are_known_workloads():
    """Both arms measure the same secondary workloads (the configured 320^3
    grid, big width, k=8 and k=32) after the main one."""
    import bench
    assert bench.OTHER_CONFIGS == ("grid3d_320_k8", "grid3d_320_k32")
    for name in bench.OTHER_CONFIGS:
        graph, parts, width, _ = bench.WORKLOADS[name]
        assert graph == "grid3d_320" and width == "big" and parts in (8, 32)


def test_allocator_policy_on_a_fake_device(tmp_path):
    """The caching allocator's reuse rules (exact class, a cached block up to
    25% larger, exact classes only under memory pressure) and its
    out-of-memory path (evict the smallest sufficient cached block, retry,
    else GP_ENOMEM), run by tests/alloc_policy.cu over a fake driver: no GPU."""
    import shutil
    import subprocess
    import pytest
    root = Path(__file__).resolve().parents[1]
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(nvcc).exists():
        pytest.skip("nvcc not available")
    exe = tmp_path / "alloc_policy"
    subprocess.run([nvcc, "-std=c++17", "-O1", "-gencode", "arch=compute_100a,code=sm_100a", "-I",
                    str(root / "include"), "-o", str(exe), str(root / "tests" / "alloc_policy.cu")],
                   check=True, capture_output=True, timeout=600)
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, run.stdout + run.stderr
    assert "all checks passed" in run.stdout
