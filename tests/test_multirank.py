"""The multi-rank path of bench.py on the CPU, world size 2 over gloo: the max-over-ranks timing and barrier that every
multi-GPU line uses, and the reference arm under torchrun (rank 0 alone runs the host-core oracle and prints the one
JSON line; the other rank exits 0 without work).  The GPU arm's ranks are independent replicas (no data-path
collective), so these are its only cross-rank steps."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        value = bench.max_over_ranks(1.0 + rank, world)  # each rank's own time; the line takes the slowest
        bench.barrier(world)
        Path(out_dir, f"rank{rank}.txt").write_text(repr(value))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_barrier_with_gloo(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    assert [float(Path(tmp_path, f"rank{r}.txt").read_text()) for r in range(2)] == [2.0, 2.0]


def test_reference_arm_under_torchrun_two_ranks():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1",
           "--warmup", "1"]
    r = subprocess.run(cmd, cwd=str(ROOT), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
