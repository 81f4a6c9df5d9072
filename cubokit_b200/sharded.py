"""One reconstruction sharded over GPUs: each rank of a ``torch.distributed`` group (NCCL over NVLink, one process per
GPU) holds a contiguous band of the scan positions and the whole object and probe.  Every iteration runs the band's
position pass and gathers (``cubo_ptycho_plan_enqueue_gradients``), sums the bands' gradient sums, weights and squared
errors, and applies the same update on every rank (``cubo_ptycho_plan_apply_gradients``).  No counterpart in
CuboPtycho, whose engine runs on one CPU thread (``Ptychography.swift:298-359``).

The sum over the bands has a fixed order: every rank receives every band's buffers (an all-gather) and adds them in
rank order itself, so the result does not depend on the collective's algorithm, protocol or topology and two runs
with the same number of ranks agree bit for bit.  It equals one plan over all positions up to the order of the sums
(each band sums its positions, then the bands are added).  With ``exchange="halo"`` (the default) a rank sends only
the object rows its windows cover (its band's rows plus half a window either side), the other rows of its object
sums being zero; ``exchange="full"`` sends whole buffers.
"""
from typing import Optional

import numpy as np

from .ptycho import Plan, PtychographyError, Result, context


def band_bounds(count: int, world: int, rank: int):
    """The contiguous band of positions [lo, hi) rank `rank` of `world` takes."""
    return rank * count // world, (rank + 1) * count // world


def touched_rows(positions, window_rows: int, object_rows: int) -> np.ndarray:
    """The object rows, ascending, that the windows of these positions cover: the rounded centre (nearest, ties to
    even, as the engine's ``Ptychography.swift:301``) plus the corner-centred window offsets, wrapped."""
    if len(positions) == 0:
        return np.zeros(0, np.int64)
    rr = np.unique(np.rint(np.asarray(positions, np.float64).reshape(-1, 2)[:, 0]).astype(np.int64))
    off = np.arange(window_rows)
    off = np.where(off < (window_rows + 1) // 2, off, off - window_rows)
    mask = np.zeros(object_rows, bool)
    mask[np.mod(rr[:, None] + off[None, :], object_rows).ravel()] = True
    return np.flatnonzero(mask)


def _all_gather(t, group):
    """[world, *t.shape]: every rank's `t`, in rank order.  NCCL gathers on the device; other backends through host
    memory (gloo has no device all-gather)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    if dist.get_backend(group) == "nccl":
        out = torch.empty((world,) + tuple(t.shape), dtype=t.dtype, device=t.device)
        dist.all_gather_into_tensor(out, t.contiguous(), group=group)
        return out
    host = t.detach().cpu().contiguous()
    parts = [torch.empty_like(host) for _ in range(world)]
    dist.all_gather(parts, host, group=group)
    return torch.stack(parts).to(t.device)


class OrderedSum:
    """Adds the bands' gradient buffers over the ranks in rank order, in place.

    ``views`` are the plan's buffers (``Plan.gradient_tensors()``): ``grad_object`` (objects x 2), ``weight_object``
    (objects), ``grad_probe``, ``weight_probe`` and ``loss``.  ``rows_by_rank`` lists, per rank, the object rows its
    object sums can be non-zero in (``None``: every row)."""

    def __init__(self, views, object_shape, rows_by_rank, group=None):
        import torch
        import torch.distributed as dist
        self.views = views
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.object_rows, self.object_columns = object_shape[-2:]
        dev = views["grad_object"].device
        if rows_by_rank is None:
            rows_by_rank = [np.arange(self.object_rows)] * self.world
        self.rows = [torch.as_tensor(np.asarray(r, np.int64), device=dev) for r in rows_by_rank]
        self.width = max(1, max(len(r) for r in rows_by_rank))

    def sum(self):
        import torch
        v = self.views
        OR, OC = self.object_rows, self.object_columns
        grad = v["grad_object"].view(OR, OC, 2)
        weight = v["weight_object"].view(OR, OC)
        # this rank's touched rows of (grad re, grad im, weight), padded to the widest rank's row count
        mine = self.rows[self.rank]
        send = torch.zeros((self.width, OC, 3), dtype=grad.dtype, device=grad.device)
        send[:len(mine), :, :2] = grad.index_select(0, mine)
        send[:len(mine), :, 2] = weight.index_select(0, mine)
        recv = _all_gather(send, self.group)
        acc = torch.zeros((OR, OC, 3), dtype=grad.dtype, device=grad.device)
        for r in range(self.world):  # rank order; each rank's rows are distinct, so every element is added once
            rows = self.rows[r]
            acc[rows] = acc[rows] + recv[r, :len(rows)]
        grad.copy_(acc[..., :2])
        weight.copy_(acc[..., 2])
        for key in ("grad_probe", "weight_probe", "loss"):
            parts = _all_gather(v[key], self.group)
            total = parts[0].clone()
            for r in range(1, self.world):
                total += parts[r]
            v[key].copy_(total)


def reconstruct(amplitudes, positions, object, probe, iterations: int = 8, precision: str = "fp32", group=None,
                device: Optional[int] = None, error_normalization="suppliedAmplitudeEnergy", exchange: str = "halo",
                **options) -> Result:
    """``SingleslicePtychography.reconstruct`` over the ranks of ``group`` (every rank passes the same arguments and
    gets the same result).  ``options`` are the engine's other parameters (``step_size``, ``normalization_minimum``,
    constraints, ``mixed_states`` ...); position correction is refused, as the sharded iteration does not move
    positions.  ``exchange``: "halo" (each rank sends the object rows its band covers) or "full"."""
    if exchange not in ("halo", "full"):
        raise PtychographyError("exchange: 'halo' or 'full'")
    run = ShardedRun(amplitudes, positions, object, probe, precision=precision, group=group, device=device,
                     error_normalization=error_normalization, exchange=exchange, **options)
    try:
        run.iterate(int(iterations))
        return run.result()
    finally:
        run.close()


class ShardedRun:
    """The state of a sharded reconstruction on this rank: its band's plan and the ordered sum over the ranks.
    ``enqueue(k)`` queues k iterations on the plan's stream without waiting (NCCL) — what the benchmark times."""

    def __init__(self, amplitudes, positions, object, probe, precision: str = "fp32", group=None,
                 device: Optional[int] = None, error_normalization="suppliedAmplitudeEnergy", exchange: str = "halo",
                 **options):
        import torch
        import torch.distributed as dist
        if options.get("position_correction") is not None:
            raise PtychographyError("position correction in a sharded reconstruction")
        world, rank = dist.get_world_size(group), dist.get_rank(group)
        self.group = group
        positions = np.asarray(positions, np.float64).reshape(-1, 2)
        count = len(positions)
        if count < world:
            raise PtychographyError("fewer positions than ranks")
        obj, prb = np.asarray(object), np.asarray(probe)
        rows, columns = prb.shape[-2:]
        self.positions = positions
        lo, hi = band_bounds(count, world, rank)
        if device is None:
            device = torch.cuda.current_device()
        self.ctx = context(device)
        self.dev = torch.device("cuda", device)
        band = np.asarray(amplitudes, np.float32).reshape(count, rows, columns)[lo:hi]
        # the error normalisation of all positions (Ptychography.swift:30-48): the amplitude energy summed over the
        # bands in rank order, or the mean intensity times the number of positions
        if isinstance(error_normalization, tuple):
            self.divisor = float(error_normalization[1]) * count
        else:
            energy = torch.tensor([float(np.sum(band.astype(np.float64) ** 2))], dtype=torch.float64, device=self.dev)
            parts = _all_gather(energy, group)
            self.divisor = float(sum(float(parts[r, 0].item()) for r in range(world)))
        self.plan = Plan(band, positions[lo:hi], obj.shape, prb.shape[-2:], ctx=self.ctx, precision=precision,
                         error_normalization=error_normalization, **options)
        self.plan.set_state(obj, prb)
        self.stream = torch.cuda.ExternalStream(self.ctx.stream, device=self.dev)
        self.exchange = exchange
        self.window_rows = rows
        self.object_shape = obj.shape
        self.summer = None
        self.losses = []

    def enqueue(self, iterations: int):
        import torch
        import torch.distributed as dist
        for _ in range(int(iterations)):
            self.plan.enqueue_gradients()
            if self.summer is None:
                world = dist.get_world_size(self.group)
                rows = None
                if self.exchange == "halo":
                    rows = [touched_rows(self.positions[slice(*band_bounds(len(self.positions), world, r))],
                                         self.window_rows, self.object_shape[-2]) for r in range(world)]
                self.summer = OrderedSum(self.plan.gradient_tensors(), self.object_shape, rows, self.group)
            with torch.cuda.stream(self.stream):  # ordered after this band's gathers, and before its update
                self.summer.sum()
                self.losses.append(self.summer.views["loss"].clone())
            self.plan.apply_gradients()

    def iterate(self, iterations: int):
        self.enqueue(iterations)
        self.ctx.synchronize()

    def result(self) -> Result:
        self.ctx.synchronize()
        errors = np.array([float(l.item()) for l in self.losses]) / self.divisor
        o, p = self.plan.get_state()
        return Result(o, p, errors, self.positions.copy())

    def close(self):
        if getattr(self, "plan", None) is not None:
            self.plan.close()
            self.plan = None
