"""Autotuner for the object-gather tile shape.

For a problem (detector, object and scan sizes, form) every candidate tile (32 x 8, 16 x 16, 64 x 4 pixels, along the
residual's contiguous axis) is timed on the problem itself: one plan per candidate, a warm-up iteration, then the
object-gather kernel's device time over a few iterations from the plan's CUDA-event kernel statistics.  The fastest
candidate is cached in a JSON file keyed by (detector, object, positions, form, GPU name), so the timing runs once per
shape per machine.  The tile choice never changes results: every object pixel sums the same positions in the same
order.
"""
from __future__ import annotations

import json
import os
from pathlib import Path

import numpy as np

from .ptycho import Plan, context

CANDIDATES = (1, 2, 3)  # 32 x 8, 16 x 16, 64 x 4
NAMES = {0: "default", 1: "32x8", 2: "16x16", 3: "64x4"}


def cache_path() -> Path:
    root = os.environ.get("CUBOKIT_B200_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "cubokit_b200")
    return Path(root) / "autotune.json"


def _load():
    try:
        return json.loads(cache_path().read_text())
    except Exception:
        return {}


def _store(table):
    path = cache_path()
    try:
        path.parent.mkdir(parents=True, exist_ok=True)
        tmp = path.with_suffix(".tmp")
        tmp.write_text(json.dumps(table, indent=1, sort_keys=True))
        os.replace(tmp, path)
    except OSError:
        pass  # a read-only home: tune again next time


def key(probe_shape, object_shape, positions, precision, device_name):
    return f"{probe_shape[0]}x{probe_shape[1]}|{object_shape[0]}x{object_shape[1]}|{positions}|{precision}|{device_name}"


def device_name(device=0):
    try:
        import torch
        return torch.cuda.get_device_name(device)
    except Exception:
        return "cuda"


def tune(amplitudes, positions, obj, probe, precision="fp32", iterations=3, device=0, use_cache=True):
    """The fastest gather tile for this problem (and the timings, ms per object-gather launch, by candidate)."""
    obj = np.asarray(obj)
    probe = np.asarray(probe)
    k = key(probe.shape, obj.shape, len(positions), precision, device_name(device))
    table = _load() if use_cache else {}
    if k in table:
        return table[k]["tile"], table[k]["ms"]
    ctx = context(device)
    timings = {}
    for cand in CANDIDATES:
        plan = Plan(amplitudes, positions, obj.shape, probe.shape, ctx=ctx, precision=precision, gather_tile=cand)
        plan.set_state(obj, probe)
        plan.iterate(1)
        plan.set_timing(True)
        plan.enqueue(iterations)
        ms, launches = plan.kernel_stats()["object_gather"]
        plan.close()
        timings[NAMES[cand]] = ms / max(launches, 1)
    best = min(CANDIDATES, key=lambda c: timings[NAMES[c]])
    if use_cache:
        table = _load()
        table[k] = {"tile": best, "ms": timings}
        _store(table)
    return best, timings
