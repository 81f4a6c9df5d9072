"""One reconstruction sharded over two ranks (``cubokit_b200.sharded``) against one plan over all positions: the same
iterations with the gradient sums, weights and errors added band by band, so the same results up to the order of the
sums (FP64 1e-11, FP32 1e-5 of max(1, max|b|)), and bit-identical results on both ranks.  The two ranks run as two
processes on one GPU over gloo (their kernels never wait on one another); on a multi-GPU node the same code runs one
rank per GPU over NCCL."""
import os
import socket
from pathlib import Path

import numpy as np
import pytest

from tests import golden_cases as gc
from tests import scenes

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
KW = dict(iterations=3, step_size=0.5, normalization_minimum=0.8, fix_probe_center_of_mass=True)


def _scene():
    s = scenes.raster_scene(scan=6, det=32, step=4, seed=5)
    return s, s["positions"] + np.array([0.25, -0.3])


def _rank_main(rank, world, port, out_dir, precision, states):
    import sys
    sys.path.insert(0, str(ROOT))
    import torch
    import torch.distributed as dist
    from cubokit_b200 import MixedstatePtychography, sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        torch.cuda.set_device(0)
        s, start = _scene()
        extra = {}
        probe = s["probe"]
        if states > 1:
            probe = MixedstatePtychography.initial_probes(s["probe"] / np.sqrt(states), states, seed=3)
            extra["mixed_states"] = states
        r = sharded.reconstruct(s["amplitudes"], start, s["object"], probe, precision=precision, device=0, **KW,
                                **extra)
        np.savez(Path(out_dir, f"rank{rank}.npz"), object=r.object, probe=r.probe, errors=r.errors)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as sock:
        sock.bind(("127.0.0.1", 0))
        return sock.getsockname()[1]


def _run_two_ranks(tmp_path, precision, states):
    import torch.multiprocessing as mp
    mp.start_processes(_rank_main, args=(2, _free_port(), str(tmp_path), precision, states), nprocs=2,
                       start_method="spawn", join=True)
    return [dict(np.load(Path(tmp_path, f"rank{r}.npz"))) for r in range(2)]


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("fp32", 1e-5)])
def test_two_bands_equal_one_plan(tmp_path, precision, tol):
    import cubokit_b200 as cb
    a, b = _run_two_ranks(tmp_path, precision, 1)
    for key in ("object", "probe", "errors"):
        assert np.array_equal(a[key], b[key]), key  # every rank applies the same sums
    s, start = _scene()
    one = cb.SingleslicePtychography.reconstruct(s["amplitudes"], start, s["object"], s["probe"], precision=precision,
                                                 **KW)
    assert max(gc.complex_gap(a["object"], one.object), gc.complex_gap(a["probe"], one.probe),
               gc.gap(a["errors"], one.errors)) < tol


def test_two_bands_of_a_mixed_state_plan(tmp_path):
    import cubokit_b200 as cb
    a, b = _run_two_ranks(tmp_path, "fp64", 2)
    assert np.array_equal(a["object"], b["object"]) and np.array_equal(a["probe"], b["probe"])
    s, start = _scene()
    probes = cb.MixedstatePtychography.initial_probes(s["probe"] / np.sqrt(2), 2, seed=3)
    one = cb.MixedstatePtychography.reconstruct(s["amplitudes"], start, s["object"], probes, **KW)
    assert max(gc.complex_gap(a["object"], one.object), gc.gap(a["errors"], one.errors),
               gc.complex_gap(gc.align_phases(a["probe"], one.probes), one.probes)) < 1e-11


def test_two_runs_at_two_ranks_agree_bit_for_bit(tmp_path):
    """The sum over the bands has a fixed order (every rank adds the all-gathered band sums in rank order), so two runs
    with the same number of ranks give the same bits."""
    (tmp_path / "a").mkdir()
    (tmp_path / "b").mkdir()
    first = _run_two_ranks(tmp_path / "a", "fp32", 1)
    second = _run_two_ranks(tmp_path / "b", "fp32", 1)
    for key in ("object", "probe", "errors"):
        assert np.array_equal(first[0][key], second[0][key]), key


def test_bench_sharded_line_with_two_ranks():
    """bench.py --gpus 2 under torchrun: one reconstruction of a 16 x 16 scan in two position bands (the ranks share this
    GPU over gloo here; on a multi-GPU node each rank has its own GPU and NCCL), one JSON line from rank 0 with the
    whole job's rate, strong scaling."""
    import json
    import subprocess
    import sys
    env = dict(os.environ, CUBO_BENCH_BACKEND="gloo")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--gpus", "2", "--scan", "16", "--steps", "2",
           "--warmup", "1", "--no-e2e"]
    r = subprocess.run(cmd, cwd=str(ROOT), capture_output=True, text=True, timeout=900, env=env)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-3000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = lines[0]
    assert line["n_gpus"] == 2 and line["scaling"] == "strong" and line["value"] > 0 and line["gpu_launches"] > 0
    assert "position bands" in line["config"]["parallelism"]
