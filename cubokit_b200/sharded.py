"""One reconstruction sharded over GPUs: each rank of a ``torch.distributed`` group (NCCL over NVLink, one process per
GPU) holds a contiguous band of the scan positions and the whole object and probe, and every iteration sums the bands'
gradient sums, weights and squared errors with one all-reduce each before every rank applies the same update
(``cubo_ptycho_plan_enqueue_gradients`` / ``_gradient_buffers`` / ``_apply_gradients``).  The result equals one plan
over all positions up to the order of the sums (the object and probe sums are per pixel over positions; here each
band sums its positions, then the bands are added).  No counterpart in CuboPtycho, whose engine runs on one CPU
thread (``Ptychography.swift:298-359``)."""
from typing import Optional

import numpy as np

from .ptycho import Plan, PtychographyError, Result, context

_SUMMED = ("grad_object", "weight_object", "grad_probe", "weight_probe", "loss")


def reconstruct(amplitudes, positions, object, probe, iterations: int = 8, precision: str = "fp32", group=None,
                device: Optional[int] = None, error_normalization="suppliedAmplitudeEnergy", **options) -> Result:
    """``SingleslicePtychography.reconstruct`` over the ranks of ``group`` (every rank passes the same arguments and
    gets the same result).  ``options`` are the engine's other parameters (``step_size``, ``normalization_minimum``,
    constraints, ``mixed_states`` ...); position correction is refused, as the sharded iteration does not move
    positions."""
    import torch
    import torch.distributed as dist
    if options.get("position_correction") is not None:
        raise PtychographyError("position correction in a sharded reconstruction")
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    positions = np.asarray(positions, np.float64).reshape(-1, 2)
    count = len(positions)
    if count < world:
        raise PtychographyError("fewer positions than ranks")
    obj, prb = np.asarray(object), np.asarray(probe)
    rows, columns = prb.shape[-2:]
    amps = np.asarray(amplitudes, np.float32).reshape(count, rows, columns)
    lo, hi = rank * count // world, (rank + 1) * count // world
    if device is None:
        device = torch.cuda.current_device()
    ctx = context(device)
    dev = torch.device("cuda", device)
    # the error normalisation of all positions (Ptychography.swift:30-48): the amplitude energy summed over the bands,
    # or the mean intensity times the number of positions
    if isinstance(error_normalization, tuple):
        divisor = float(error_normalization[1]) * count
    else:
        energy = torch.tensor([float(np.sum(amps[lo:hi].astype(np.float64) ** 2))], dtype=torch.float64, device=dev)
        dist.all_reduce(energy, group=group)
        divisor = float(energy.item())
    plan = Plan(amps[lo:hi], positions[lo:hi], obj.shape, prb.shape[-2:], ctx=ctx, precision=precision,
                error_normalization=error_normalization, **options)
    try:
        plan.set_state(obj, prb)
        stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
        losses = []
        views = None
        for _ in range(int(iterations)):
            plan.enqueue_gradients()
            if views is None:
                views = plan.gradient_tensors()
            with torch.cuda.stream(stream):  # ordered after this band's gathers, and before its update
                for key in _SUMMED:
                    dist.all_reduce(views[key], group=group)
                losses.append(views["loss"].clone())
            plan.apply_gradients()
        ctx.synchronize()
        errors = np.array([float(l.item()) for l in losses]) / divisor
        o, p = plan.get_state()
    finally:
        plan.close()
    return Result(o, p, errors, positions.copy())
