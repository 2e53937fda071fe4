"""The multi-process plumbing of bench.py on the CPU (world size 2, gloo, 127.0.0.1): every rank
gets the largest rank's time, and the reference arm runs on rank 0 only (the other ranks exit
without output)."""

import os
import socket
import subprocess
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, values, out):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out[rank] = bench.max_over_ranks(values[rank], world, device="cpu")
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    world = 2
    values = [3.25, 7.5]
    with mp.Manager() as manager:
        out = manager.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), values, out), nprocs=world, join=True)
        assert dict(out) == {0: 7.5, 1: 7.5}
    assert __import__("bench").max_over_ranks(4.0, 1) == 4.0


def test_reference_arm_prints_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "0"],
                       capture_output=True, text=True, env=env, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
