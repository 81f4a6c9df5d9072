"""Autotuner for the object-gather tile and the position-pass CTA shape.

For a problem (detector, object and scan sizes, form) every candidate is timed on the problem itself: one plan per
candidate, a warm-up iteration, then the kernel's device time over a few iterations from the plan's CUDA-event kernel
statistics.  `tune` picks the object-gather tile (32 x 8, 16 x 16, 64 x 4 pixels, along the residual's contiguous
axis); `tune_pass` the CTA shape of the shared-memory position pass at the detectors it runs with a compile-time radix
plan or the FP32 register-line kernel (64 x 64 and 96 x 96).  The fastest candidate is cached in a JSON file keyed by
(what, detector, object, positions, form, GPU name), so the timing runs once per shape per machine.  Neither choice
changes the object: every object pixel sums the same positions in the same order whatever the tile, and every
butterfly computes the same values whatever the shared-memory CTA shape; the FP32 register-line kernel agrees with
those to FP32 round-off.
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


def _time(amplitudes, positions, obj, probe, precision, iterations, device, kernel, option, candidates, names):
    ctx = context(device)
    timings = {}
    for cand in candidates:
        plan = Plan(amplitudes, positions, obj.shape, probe.shape, ctx=ctx, precision=precision, **{option: cand})
        plan.set_state(obj, probe)
        plan.iterate(1)
        plan.set_timing(True)
        plan.enqueue(iterations)
        ms, launches = plan.kernel_stats()[kernel]
        plan.close()
        timings[names[cand]] = ms / max(launches, 1)
    return min(candidates, key=lambda c: timings[names[c]]), timings


def _tuned(what, amplitudes, positions, obj, probe, precision, iterations, device, use_cache, kernel, option,
           candidates, names):
    obj = np.asarray(obj)
    probe = np.asarray(probe)
    k = what + "|" + key(probe.shape, obj.shape, len(positions), precision, device_name(device))
    table = _load() if use_cache else {}
    if k in table:
        return table[k]["choice"], table[k]["ms"]
    best, timings = _time(amplitudes, positions, obj, probe, precision, iterations, device, kernel, option, candidates,
                          names)
    if use_cache:
        table = _load()
        table[k] = {"choice": best, "ms": timings}
        _store(table)
    return best, timings


def tune(amplitudes, positions, obj, probe, precision="fp32", iterations=3, device=0, use_cache=True):
    """The fastest gather tile for this problem (and the timings, ms per object-gather launch, by candidate)."""
    return _tuned("gather", amplitudes, positions, obj, probe, precision, iterations, device, use_cache,
                  "object_gather", "gather_tile", CANDIDATES, NAMES)


PASS_CANDIDATES = {("fp32", 64): (0, 1, 2, 3), ("fp32", 96): (0, 2, 3), ("fp64", 64): (1, 2, 3), ("fp64", 96): (3,)}
PASS_NAMES = {0: "default", 1: "shared memory, 128 threads", 2: "shared memory, 256 threads",
              3: "shared memory, 512 threads"}


def tune_pass(amplitudes, positions, obj, probe, precision="fp32", iterations=3, device=0, use_cache=True):
    """The fastest position-pass CTA shape for this problem (and the timings, ms per position-pass launch, by
    candidate); (0, {}) for detectors without a choice (every size but 64 x 64 and 96 x 96)."""
    rows, columns = np.asarray(probe).shape
    if rows != columns or (precision, rows) not in PASS_CANDIDATES:
        return 0, {}
    return _tuned("pass", amplitudes, positions, obj, probe, precision, iterations, device, use_cache,
                  "position_pass", "pass_shape", PASS_CANDIDATES[(precision, rows)], PASS_NAMES)
