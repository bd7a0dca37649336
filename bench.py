#!/usr/bin/env python3
"""Benchmark: edges/s partitioned (directed CSR entries / partition time).

Default workload: RMAT scale 22, edge factor 16 (a=.57 b=.19 c=.19), seed 1,
symmetrised, self loops and duplicates removed, unit weights, k=32,
imbalance 1.03, seed 0, standard (32-bit) width -- generated here (synthetic,
no dataset).  One step = one full partition (coarsen -> initial -> refine) of
that graph.

  python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

* value: K steps with the CSR already resident in HBM (device arrays passed
  in place), timed with CUDA events on the library's stream, max over ranks.
  The graph (~0.5 GB) is larger than L2, so no L2 flush is done.
* e2e: the same call with host buffers: int64 indptr/indices in pinned host
  memory (the reference driver's input format), H2D + GPU narrowing and
  validation + partition + D2H of the labels inside the timed region.
* --impl reference: the reference's own partitioner (its CUDA sources
  compiled for sm_100a into oracle/_ref by oracle/Makefile) run through its
  own CLI on the same files; its algorithm_total_seconds scope is the step.
* N > 1 GPUs: independent replicas (one graph per GPU, no collective).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
# one hardware work queue per server slot stream (read at CUDA context creation)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

WORKLOADS = {
    # name: (graph, parts, width, description)
    "rmat22_k32": ("rmat22", 32, "standard",
                   "RMAT scale 22 ef16 (0.57,0.19,0.19) seed 1, symmetrised, k=32, imbalance 1.03, standard"),
    "grid2d_256_k4": ("grid2d_256", 4, "standard", "2D 5-point grid 256x256, k=4, imbalance 1.03, standard"),
    "rmat24_k32": ("rmat24", 32, "standard", "RMAT scale 24 ef16 seed 1, k=32, standard"),
    # profiling-size case of the default workload (same generator, 1/4 the vertices)
    "rmat20_k32": ("rmat20", 32, "standard", "RMAT scale 20 ef16 (0.57,0.19,0.19) seed 1, symmetrised, k=32, standard"),
    "grid3d_320_k32": ("grid3d_320", 32, "big", "3D 7-point grid 320^3, k=32, big"),
    "grid3d_320_k8": ("grid3d_320", 8, "big", "3D 7-point grid 320^3, k=8, big"),
}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, world, local


class Dist:
    def __init__(self, world: int):
        self.world = world
        self.pg = None
        if world > 1:
            import torch.distributed as td
            from datetime import timedelta
            td.init_process_group("gloo", timeout=timedelta(seconds=600))
            self.td = td

    def barrier(self):
        if self.world > 1:
            self.td.barrier()

    def max(self, x: float) -> float:
        if self.world == 1:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64)
        self.td.all_reduce(t, op=self.td.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.td.destroy_process_group()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def load_workload(name: str, rank: int, dist: Dist | None):
    from horkxg_b200 import graphs
    gname, parts, width, desc = WORKLOADS[name]
    if rank == 0:
        graphs.by_name(gname)
    if dist is not None:
        dist.barrier()
    indptr, indices = graphs.by_name(gname)
    off = np.fromfile(indptr, dtype=np.int64)
    idx = np.fromfile(indices, dtype=np.int64)
    return indptr, indices, off, idx, parts, width, desc


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


# DRAM bytes per algorithmic byte, measured with ncu (dram__bytes_read.sum +
# dram__bytes_write.sum over every launch of the kernel in one timed
# partition of RMAT-20 ef16, k=32, against the library's algorithmic bytes for
# the same launches).  The traffic of a launch here is that ratio times its
# algorithmic bytes.
DRAM_PER_ALGORITHMIC_BYTE = {"hub_insert_kernel": 1.745, "segment_smem_kernel": 0.555}


# Algorithmic bytes per launch of the dominant kernels are recorded by the
# library itself (gp_profile_dump); this picks the kernel with the largest
# total time that has a traffic model.
def roofline(profile: dict, hbm_gbs: float, src: str):
    ranked = sorted(profile.items(), key=lambda kv: -kv[1]["ms"])
    total_ms = sum(v["ms"] for v in profile.values()) or 1.0
    for name, v in ranked:
        if v["bytes"] > 0 and v["ms"] > 0:
            achieved = v["bytes"] / (v["ms"] * 1e-3) / 1e9
            per_launch = v["bytes"] / max(1, v["launches"])
            ratio = DRAM_PER_ALGORITHMIC_BYTE.get(name)
            return {"kernel": name, "bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_gbs,
                    "peak_source": src, "unit": "GB/s", "frac": round(achieved / hbm_gbs, 4),
                    "traffic": round(ratio * per_launch) if ratio else None,
                    "traffic_source": ("ncu DRAM bytes per algorithmic byte of this kernel on RMAT-20 "
                                       f"({ratio}) x the algorithmic bytes per launch here") if ratio else None,
                    "share_of_gpu_time": round(v["ms"] / total_ms, 4), "launches": v["launches"],
                    "algorithmic_bytes_per_launch": per_launch}
    return None


def host_cpu() -> str:
    model = "unknown"
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return f"{model}, {os.cpu_count()} logical cores"


def analyzer_baseline(indptr: Path, indices: Path, labels: np.ndarray, parts: int, m: int, cut: int):
    """The reference's CPU analyzer (graph_untils/analyze_partition.cpp, single
    threaded, built from its source by oracle/Makefile) on the timed result:
    one instance timed three times (median), then eight concurrent instances.
    The int32 labels are written as text first, untimed, because the analyzer
    reads text labels (analyze_partition.cpp:145-155)."""
    exe = ROOT / "oracle" / "_ref" / "analyze_partition"
    if not exe.exists():
        return None
    txt = Path("/tmp") / f"gp_labels_{os.getpid()}.txt"
    txt.write_text("\n".join(map(str, labels.tolist())) + "\n")
    cmd = [str(exe), "--partition", str(txt), "--indptr", str(indptr), "--indices", str(indices),
           "--parts", str(parts)]
    times, directed = [], None
    for _ in range(3):
        t0 = time.perf_counter()
        out = subprocess.run(cmd, capture_output=True, text=True, check=True).stdout
        times.append(time.perf_counter() - t0)
        for line in out.splitlines():
            f = line.split()
            if len(f) >= 3 and f[0] == str(txt):
                directed = int(f[2])
    t0 = time.perf_counter()
    procs = [subprocess.Popen(cmd, stdout=subprocess.DEVNULL) for _ in range(8)]
    rcs = [p.wait() for p in procs]
    conc = time.perf_counter() - t0
    txt.unlink(missing_ok=True)
    if directed != 2 * cut or any(rcs):
        raise RuntimeError(f"analyzer disagrees: directed cut {directed} vs 2x{cut}, exit codes {rcs}")
    one = statistics.median(times)
    return {"value": m / one, "unit": "edges/s", "cores": 1, "kind": "reference",
            "sample": f"reference CPU analyzer (analyze_partition, g++ -O2, one thread) over the full timed "
                      f"result ({m} directed entries; whole process incl. reading the int64 CSR), median of 3: "
                      f"{one:.2f} s; its directed cut {directed} = 2 x the reported cut",
            "concurrent8_value": 8 * m / conc, "host": host_cpu()}


def cpu_baseline(sample_scale: int = 17, parts: int = 32):
    """The oracle's CPU restatement of the whole partitioner (single thread)
    on a bounded sample: RMAT scale `sample_scale` (same generator, seed 1)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle as O
    from horkxg_b200 import graphs
    off, idx = graphs.load(*graphs.rmat(sample_scale))
    g = O.Graph(off, np.asarray(idx))
    t0 = time.perf_counter()
    _, cut = O.partition(g, parts, 1.03, 0)
    dt = time.perf_counter() - t0
    return {"value": len(idx) / dt, "unit": "edges/s", "cores": 1, "kind": "port",
            "sample": f"RMAT scale {sample_scale} ef16 seed 1 (m={len(idx)}), k={parts}, one full partition "
                      f"({dt:.1f} s, cut {cut}) by the oracle's C++ restatement"}


def pinned_numpy(a: np.ndarray) -> np.ndarray:
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()


def recount_ok(off, nbr, labels, cut) -> bool:
    src = np.repeat(np.arange(len(off) - 1, dtype=np.int64), np.diff(off))
    return int(np.count_nonzero(labels[src] != labels[nbr])) == 2 * cut


def run_batched(local: int, slots: int, passes: int = 5):
    """Batched workload: 512 random geometric graphs (n log-uniform in
    [1e3, 1e6], mean degree 10, k uniform in {2,4,8,16,32}, seed 7) in one
    packed CSR in pinned host memory.  "plain" partitions them one by one on
    one context (gp_partition_range per instance); "batched" hands the packed
    CSR to gp_partition_batch on a server with `slots` slots.  Host wall
    clock around each synchronous pass (the calls return with labels on the
    host), median of `passes` passes of each; the batched pass runs once
    untimed first so its slots are warm, as the plain context is."""
    import horkxg_b200 as hb
    from horkxg_b200 import graphs
    t0 = time.perf_counter()
    off, nbr, vo, ks = graphs.rgg_batch()
    gen_s = time.perf_counter() - t0
    packed = hb.PackedGraph(pinned_numpy(off), pinned_numpy(nbr), vo)
    count = packed.count
    opts = [hb.default_options(parts=int(k)) for k in ks]
    with hb.Context(local) as ctx:
        ctx.partition_range(packed, int(np.argmax(np.diff(vo))), opts[0])   # warm the context
        plain_times = []
        for _ in range(passes):
            t0 = time.perf_counter()
            plain_cuts = [ctx.partition_range(packed, i, opts[i])[1].cut for i in range(count)]
            plain_times.append(time.perf_counter() - t0)
    with hb.Server(local, slots=slots, memory_budget=120 << 30) as srv:
        srv.partition_batch(packed, opts)
        batch_times = []
        for _ in range(passes):
            t0 = time.perf_counter()
            labels, reps = srv.partition_batch(packed, opts)
            batch_times.append(time.perf_counter() - t0)
    plain_s = statistics.median(plain_times)
    batch_s = statistics.median(batch_times)
    bad = 0
    worst_ratio = 0.0
    for i in range(count):
        a, b = int(vo[i]), int(vo[i + 1])
        o, x = packed.instance(i)
        lab = labels[a:b]
        k = int(ks[i])
        loads = np.bincount(lab, minlength=k)
        if not recount_ok(o, x, lab, reps[i].cut) or loads.max() > hb.capacity(b - a, k, 1.03):
            bad += 1
        if plain_cuts[i]:
            worst_ratio = max(worst_ratio, reps[i].cut / plain_cuts[i])
    if bad:
        raise RuntimeError(f"{bad} batched instances failed the recount or capacity check")
    return {"workload": "512 RGG, n log-uniform [1e3,1e6], mean degree 10, k in {2,4,8,16,32}, seed 7",
            "graphs": count, "vertices": int(vo[-1]), "edges": int(packed.m), "slots": slots,
            "plain_graphs_per_s": count / plain_s, "batched_graphs_per_s": count / batch_s,
            "speedup": plain_s / batch_s, "plain_seconds": plain_s, "batched_seconds": batch_s,
            "batched_edges_per_s": packed.m / batch_s, "generation_seconds": gen_s,
            "checked": "every instance: exact recount == reported cut, max part <= capacity",
            "max_cut_ratio_batched_vs_plain": worst_ratio,
            "plain_seconds_passes": plain_times, "batched_seconds_passes": batch_times,
            "timing": f"host wall clock, synchronous calls, median of {passes} passes each"}


def run_serving(local: int, slots: int, seconds: float, rate: float = 200.0, pool_size: int = 32):
    """Serving workload: Poisson arrivals at `rate`/s for `seconds` s (seed
    11); each request is a graph of the serving mix ({2D grid, RGG deg 10,
    RMAT ef 16}, n log-uniform [1e4, 4e6], k uniform [2, 32]).  The mix is
    pre-generated as `pool_size` distinct graphs that the arrivals draw from
    uniformly (each request is partitioned in full).  Latency is measured by
    the server from submission to labels on the host."""
    import horkxg_b200 as hb
    from horkxg_b200 import graphs
    t0 = time.perf_counter()
    pool = [(kind, hb.HostGraph(pinned_numpy(off), pinned_numpy(nbr)), k)
            for kind, off, nbr, k in graphs.serving_mix(pool_size, seed=11)]
    gen_s = time.perf_counter() - t0
    rng = np.random.default_rng(11)
    arrivals, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= seconds:
            break
        arrivals.append((t, int(rng.integers(pool_size))))
    import queue
    done_q: "queue.Queue" = queue.Queue()
    infos = []
    with hb.Server(local, slots=slots, memory_budget=120 << 30) as srv:
        for _, g, k in pool:                    # warm every slot's memory pool
            srv.wait(srv.submit(g, parts=k))

        def waiter():
            while True:
                item = done_q.get()
                if item is None:
                    return
                ticket, idx = item
                labels, rep, info = srv.wait(ticket)
                infos.append((info.latency_seconds, info.queued_seconds, info.service_seconds, rep.cut, idx))

        th = threading.Thread(target=waiter, daemon=True)
        th.start()
        start = time.perf_counter()
        for at, idx in arrivals:
            delay = start + at - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            _, g, k = pool[idx]
            done_q.put((srv.submit(g, parts=k), idx))
        done_q.put(None)
        th.join()
        total = time.perf_counter() - start
    lat = np.array([x[0] for x in infos]) * 1e3
    edges = sum(pool[x[4]][1].m for x in infos)
    return {"workload": f"Poisson {rate:g}/s for {seconds:g} s, seed 11; grid / RGG deg 10 / RMAT ef16, "
                        f"n log-uniform [1e4,4e6], k uniform [2,32]; {pool_size} pre-generated graphs",
            "requests": len(infos), "slots": slots, "memory_budget_gb": 120,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_queue_ms": float(np.mean([x[1] for x in infos]) * 1e3),
            "mean_service_ms": float(np.mean([x[2] for x in infos]) * 1e3),
            "offered_graphs_per_s": rate, "achieved_graphs_per_s": len(infos) / total,
            "achieved_edges_per_s": edges / total, "wall_seconds": total, "generation_seconds": gen_s}


def run_ours(args, rank, world, local, dist):
    import torch
    import horkxg_b200 as hb
    torch.cuda.set_device(local)
    indptr, indices, off64, idx64, parts, width, desc = load_workload(args.workload, rank, dist)
    n, m = len(off64) - 1, len(idx64)
    ctx = hb.Context(local)
    wcode = hb.STANDARD if width == "standard" else hb.BIG
    odt = torch.int32 if width == "standard" else torch.int64
    d_off = torch.from_numpy(off64).to(device=f"cuda:{local}", dtype=odt)
    d_nbr = torch.from_numpy(idx64).to(device=f"cuda:{local}", dtype=torch.int32)
    d_lab = torch.empty(n, dtype=torch.int32, device=f"cuda:{local}")
    ddesc = hb.GraphDesc()
    ddesc.n, ddesc.m, ddesc.width, ddesc.memory, ddesc.index64 = n, m, wcode, hb.DEVICE, 0
    ddesc.offsets, ddesc.neighbors = d_off.data_ptr(), d_nbr.data_ptr()
    opts = hb.default_options(parts=parts, seed=0)
    stream = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{local}")
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        ctx.partition_desc(ddesc, d_lab.data_ptr(), opts)
    torch.cuda.synchronize()
    dist.barrier()
    launches0 = ctx.launches
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reports = []
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.nvtx.range_push("timed")  # lets ncu --nvtx-include "timed/" select these launches
        start.record(stream)
        for _ in range(args.steps):
            reports.append(ctx.partition_desc(ddesc, d_lab.data_ptr(), opts))
        stop.record(stream)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        dist.barrier()
    launches = (ctx.launches - launches0) // max(1, args.steps)
    elapsed = start.elapsed_time(stop) * 1e-3
    t_max = dist.max(elapsed)
    cuts = [r.cut for r in reports]
    labels = d_lab.cpu().numpy()
    # correctness of the timed result: exact recount + capacity
    loads = np.bincount(labels, minlength=parts)
    cap = hb.capacity(n, parts, 1.03)
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(off64))
    directed = int(np.count_nonzero(labels[src] != labels[idx64]))
    assert directed // 2 == reports[-1].cut and loads.max() <= cap, "timed result failed the recount"

    # end to end through the public API with host buffers
    pin_off = torch.from_numpy(off64).pin_memory()
    pin_idx = torch.from_numpy(idx64).pin_memory()
    pin_lab = torch.empty(n, dtype=torch.int32).pin_memory()
    hdesc = hb.GraphDesc()
    hdesc.n, hdesc.m, hdesc.width, hdesc.memory, hdesc.index64 = n, m, wcode, hb.HOST, 1
    hdesc.offsets, hdesc.neighbors = pin_off.data_ptr(), pin_idx.data_ptr()
    ctx.partition_desc(hdesc, pin_lab.data_ptr(), opts)
    torch.cuda.synchronize()
    dist.barrier()
    e_start, e_stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    e_steps = max(1, min(args.steps, 5))
    for _ in range(e_steps):
        ctx.partition_desc(hdesc, pin_lab.data_ptr(), opts)
    e_stop.record(stream)
    torch.cuda.synchronize()
    e_elapsed = dist.max(e_start.elapsed_time(e_stop) * 1e-3)

    # final cut over seeds 0..4 (untimed), for the cut-quality comparison
    # with the reference's median over the same seeds
    seed_cuts = []
    for sd in range(args.cut_seeds):
        seed_cuts.append(int(ctx.partition_desc(ddesc, d_lab.data_ptr(), hb.default_options(parts=parts, seed=sd)).cut))

    # per-kernel profile of one more step (outside the timed region)
    ctx.profile(True)
    ctx.partition_desc(ddesc, d_lab.data_ptr(), opts)
    prof = ctx.profile_dump()
    ctx.profile(False)
    if args.profile_out is not None and rank == 0:
        args.profile_out.parent.mkdir(parents=True, exist_ok=True)
        args.profile_out.write_text(json.dumps(prof, indent=1, sort_keys=True))
    hbm, src_peak = peaks()
    result = None
    if rank == 0:
        value = world * m * args.steps / t_max
        line = {
            "metric": "edges/s partitioned", "value": value, "unit": "edges/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic",
            "config": {"workload": desc, "graph": WORKLOADS[args.workload][0], "vertices": n, "edges": m,
                       "parts": parts, "width": width, "parallelism": f"replicas{world}",
                       "l2": "inputs larger than L2 (0.5 GB CSR), no flush"},
            "cut": int(statistics.median(cuts)), "max_part_weight": int(loads.max()), "capacity": int(cap),
            "cut_seeds": seed_cuts, "cut_median_seeds": int(statistics.median(seed_cuts)) if seed_cuts else None,
            "algorithm_seconds_median": statistics.median(r.algorithm_seconds for r in reports),
            "stage_seconds": {"coarsen": reports[-1].coarsen_seconds, "initial": reports[-1].initial_seconds,
                              "uncoarsen": reports[-1].uncoarsen_seconds, "free": reports[-1].free_seconds},
            "levels": reports[-1].levels, "coarsest_n": reports[-1].coarsest_n,
            "e2e": {"value": world * m * e_steps / e_elapsed, "unit": "edges/s",
                    "h2d_bytes_per_step": (n + 1) * 8 + m * 8, "d2h_bytes_per_step": n * 4},
            "gpu_launches": int(launches),
            "roofline": roofline(prof, hbm, src_peak),
            "clocks": clocks.summary(),
            "kernel_profile_ms": {k: round(v["ms"], 4) for k, v in sorted(prof.items(), key=lambda kv: -kv[1]["ms"])[:12]},
        }
        if world == 1 and not args.no_batched:
            line["batched"] = run_batched(local, args.slots)
        if world == 1 and args.serve_seconds > 0:
            line["serving"] = run_serving(local, args.slots, args.serve_seconds)
        if not args.no_cpu_baseline and world == 1:
            # the reference's CPU analyzer on the timed result, and the
            # oracle's single-thread restatement of the partitioner on a sample
            port = cpu_baseline()
            line["cpu_baseline"] = analyzer_baseline(indptr, indices, labels, parts, m, reports[-1].cut) or port
            line["cpu_port_partition"] = port
        result = line
    ctx.close()
    return result


def run_reference(args, rank, world, local, dist):
    if rank != 0:
        return None
    indptr, indices, off64, idx64, parts, width, desc = load_workload(args.workload, rank, None)
    n, m = len(off64) - 1, len(idx64)
    exe = ROOT / "oracle" / "_ref" / f"gpart_partition_{width}"
    if not exe.exists():
        return {"impl": "reference", "unavailable": f"{exe} not built (oracle/Makefile ref target)"}
    env = dict(os.environ, CUDA_VISIBLE_DEVICES=os.environ.get("CUDA_VISIBLE_DEVICES", str(local)))
    out = Path("/tmp") / f"gp_ref_{args.workload}.part"
    algo, walls, cuts = [], [], []

    def once(seed=0):
        t0 = time.perf_counter()
        text = subprocess.run([str(exe), str(indptr), str(indices), str(parts), str(out), "1.03", str(seed)],
                              capture_output=True, text=True, check=True, env=env).stdout
        wall = time.perf_counter() - t0
        a = float(re.findall(r"algorithm_total_seconds=([0-9.e+-]+)", text)[-1])
        c = int(re.findall(r"^final_edge_cut=(\d+)$", text, re.M)[-1])
        return a, wall, c

    for _ in range(args.warmup):
        once()
    with ClockSampler(local) as clocks:
        for i in range(args.steps):
            a, w, c = once(i % 5)   # seeds 0..4 in turn (the timing does not depend on the seed)
            algo.append(a)
            walls.append(w)
            cuts.append(c)
    seed_cuts = cuts[:5]
    for sd in range(len(seed_cuts), min(5, args.cut_seeds)):
        seed_cuts.append(once(sd)[2])
    total = sum(algo)
    value = m * args.steps / total
    return {
        "impl": "reference", "metric": "edges/s partitioned", "value": value, "unit": "edges/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": desc, "graph": WORKLOADS[args.workload][0], "vertices": n, "edges": m,
                   "parts": parts, "width": width, "parallelism": "replicas1"},
        "cut": int(statistics.median(cuts)),
        "cut_seeds": seed_cuts, "cut_median_seeds": int(statistics.median(seed_cuts)) if seed_cuts else None,
        "process_seconds_median": statistics.median(walls),
        "e2e": {"value": value, "unit": "edges/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "cpu_baseline": {"value": value, "unit": "edges/s", "cores": 0, "kind": "reference",
                         "sample": "the reference's own partitioner is CUDA code (no CPU implementation exists); "
                                   "this arm runs its sm_100a build from oracle/_ref on the GPU, algorithm_total_seconds scope"},
        "clocks": clocks.summary(),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="rmat22_k32")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-out", type=Path, default=None, help="write the full per-kernel profile (JSON)")
    ap.add_argument("--no-batched", action="store_true", help="skip the 512-graph batched workload")
    ap.add_argument("--serve-seconds", type=float, default=10.0,
                    help="length of the Poisson request stream (the serving workload is 60 s; 0 skips it)")
    ap.add_argument("--slots", type=int, default=8, help="server slots for the batched and serving workloads")
    ap.add_argument("--cut-seeds", type=int, default=5, help="untimed partitions with seeds 0..N-1 for the cut median")
    args = ap.parse_args()
    rank, world, local = dist_env()
    dist = Dist(world)
    try:
        if args.impl == "reference":
            line = run_reference(args, rank, world, local, dist)
        else:
            line = run_ours(args, rank, world, local, dist)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
