"""The multi-process plumbing of bench.py on CPU: two gloo ranks on 127.0.0.1 (the max-over-ranks
timing every N > 1 run reports), and the reference arm's rank handling (rank 0 alone runs the CPU
oracle and prints; other ranks exit without work)."""
import json
import os
import socket
import subprocess
import sys
from datetime import timedelta
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, queue):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        sys.path.insert(0, str(ROOT))
        import bench
        value = bench.reduce_max(0.5 * (rank + 1), dist)
        alone = bench.reduce_max(3.0, None)
        dist.barrier()
        queue.put((rank, value, alone))
    finally:
        dist.destroy_process_group()


def test_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, queue)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(queue.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == [(0, 1.0, 3.0), (1, 1.0, 3.0)]


def _bench(*args, rank="0"):
    env = dict(os.environ, RANK=rank, WORLD_SIZE="2", LOCAL_RANK=rank)
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], cwd=ROOT, env=env,
                          capture_output=True, text=True, timeout=600)


def test_reference_arm_rank_handling():
    small = ("--impl", "reference", "--gpus", "2", "--particles", "20000", "--resolution", "64",
             "--steps", "2", "--warmup", "1")
    other = _bench(*small, rank="1")
    assert other.returncode == 0 and other.stdout.strip() == ""
    first = _bench(*small, rank="0")
    assert first.returncode == 0, first.stderr[-2000:]
    line = json.loads(first.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["e2e"]["h2d_bytes_per_step"] == 0
