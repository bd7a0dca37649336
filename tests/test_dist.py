"""The multi-GPU bench path on the CPU: `bench.py --gpus N` runs one process
per GPU as independent replicas (no data-path collective); the ranks only
meet at barriers and take the maximum of their timings over a gloo process
group.  Two ranks on 127.0.0.1 check both."""
import multiprocessing as mp
import os
import socket
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank: int, world: int, port: int, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import bench
    r, w, local = bench.dist_env()
    dist = bench.Dist(w)
    dist.barrier()
    worst = dist.max(1.5 + r)          # each rank's "timing"
    dist.barrier()
    dist.close()
    out.put((r, w, local, worst))


def test_two_rank_barrier_and_max_over_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [(r, w, l) for r, w, l, _ in results] == [(0, 2, 0), (1, 2, 1)]
    assert all(m == 2.5 for *_, m in results)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    d = bench.Dist(1)
    d.barrier()
    assert d.max(3.0) == 3.0
    d.close()
