"""The fixed-order sum over ranks of a sharded reconstruction (``cubokit_b200.sharded.OrderedSum``), world size 2 over
gloo on the CPU: every rank ends with the same buffers, equal bit for bit to the sum of the ranks' buffers taken in rank
order, whether whole buffers are exchanged or only the object rows each rank's windows cover (the halo exchange);
``touched_rows`` gives those rows with the engine's rounding and wrap."""
import os
import socket
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
OR, OC, N = 24, 10, 12


def _free_port():
    with socket.socket() as sock:
        sock.bind(("127.0.0.1", 0))
        return sock.getsockname()[1]


def _rank_buffers(rank, rows):
    """Rank `rank`'s gradient buffers: random in its rows (FP32, as the FP32 and split-BF16 forms keep them), zero in
    every other object row; random probe sums and loss."""
    rng = np.random.default_rng(100 + rank)
    grad = np.zeros((OR, OC, 2), np.float32)
    weight = np.zeros((OR, OC), np.float32)
    grad[rows] = rng.standard_normal((len(rows), OC, 2)).astype(np.float32)
    weight[rows] = rng.random((len(rows), OC)).astype(np.float32)
    return {"grad_object": grad.reshape(-1, 2), "weight_object": weight.reshape(-1),
            "grad_probe": rng.standard_normal((N, 2)), "weight_probe": rng.random(N), "loss": rng.random(1)}


def _rows(world):
    from cubokit_b200.sharded import band_bounds, touched_rows
    positions = np.array([[r, 3.0] for r in np.arange(0.5, 40.0, 1.5)])  # ties round to even
    return positions, [touched_rows(positions[slice(*band_bounds(len(positions), world, r))], 6, OR)
                       for r in range(world)]


def _rank_main(rank, world, port, out_dir):
    import sys
    sys.path.insert(0, str(ROOT))
    import torch
    import torch.distributed as dist
    from cubokit_b200.sharded import OrderedSum
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        _, rows = _rows(world)
        out = {}
        for mode in ("halo", "full"):
            views = {k: torch.from_numpy(v.copy()) for k, v in _rank_buffers(rank, rows[rank]).items()}
            OrderedSum(views, (OR, OC), rows if mode == "halo" else None).sum()
            out.update({f"{mode}_{k}": v.numpy() for k, v in views.items()})
        np.savez(Path(out_dir, f"rank{rank}.npz"), **out)
    finally:
        dist.destroy_process_group()


def test_touched_rows_follow_the_engine_rounding_and_wrap():
    from cubokit_b200.sharded import touched_rows
    # centre 2.5 rounds to 2 (ties to even), window rows -3..2 around it, wrapped into 24 rows
    assert list(touched_rows(np.array([[2.5, 0.0]]), 6, 24)) == [0, 1, 2, 3, 4, 23]
    assert list(touched_rows(np.array([[3.5, 0.0]]), 6, 24)) == [1, 2, 3, 4, 5, 6]


def test_ordered_sum_is_the_rank_order_sum_on_every_rank(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn",
                       join=True)
    got = [dict(np.load(Path(tmp_path, f"rank{r}.npz"))) for r in range(world)]
    _, rows = _rows(world)
    parts = [_rank_buffers(r, rows[r]) for r in range(world)]
    for key in parts[0]:
        expected = parts[0][key].copy()
        for r in range(1, world):
            expected = expected + parts[r][key]
        for r in range(world):
            for mode in ("halo", "full"):
                assert np.array_equal(got[r][f"{mode}_{key}"], expected), (key, r, mode)
