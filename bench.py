"""Benchmark of the single-slice ptychography GD engine on B200.

Workload (the precision-form configuration): 256 x 256 raster scan, step 4 px, 128 x 128 detector, object 1152 x 1152,
Float32 amplitudes at 1e5 e/pattern, seeded synthetic data (cubokit_b200.synthetic).  One step = one full-batch GD
iteration over all 65,536 positions.  Metric: positions * iterations / s.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--form both|fp32|split_bf16] [--impl ours|reference]

The headline form is split-BF16 (the DFT-matrix products on the tensor cores); the FP32 form runs on the same data in
the same invocation and the line reports both, their ratio and the relative L2 difference of their objects.

`value` is device-timed (CUDA events on the engine's stream) with amplitudes resident in HBM; the 4.3 GB amplitude
stack and the 8.6 GB residual buffer are far larger than L2, so no flush is needed.  `e2e` is one
SingleslicePtychography.reconstruct call (the public API) of K iterations from pinned host buffers, host<->device
copies, validation and plan set-up included, timed by the wall clock around the blocking call.  With --gpus N > 1
(torchrun), every rank runs an independent replica on its own GPU (the path has no cross-GPU exchange: "replicas
only"); value = sum over ranks, time = max over ranks.  --impl reference times the FP64 C restatement of CuboPtycho's
Double CPU path (oracle/, OpenMP over all host cores) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "positions*iter/s, 128^2 det GD: split-BF16 vs FP32 at <=1e-4 object err"
UNIT = "positions*iter/s"
SCAN, DET, STEP, DOSE = 256, 128, 4, 1e5


def algorithmic(P, n, objects):
    """Per-iteration algorithmic bytes and flops of the path (amplitudes read once; object and probe complex64 read
    and written once; two n-point 2-D FFTs and 40 flops per pixel per position)."""
    bytes_iter = P * 4 * n + 16 * objects + 16 * n
    flops_iter = P * (10 * n * math.log2(n) + 40 * n)
    return bytes_iter, flops_iter


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = [l.split(",") for l in open(self.path).read().strip().splitlines() if l.strip()]
        os.unlink(self.path)
        sm, mx, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1])); mx.append(float(r[2])); power.append(float(r[3]))
            except (ValueError, IndexError):
                continue
            for name, v in zip(names, r[5:9]):
                if v.strip() == "Active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "power_w_max": max(power),
                "samples": len(sm), "reasons": sorted(reasons)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d["hbm_gbs"], d.get("bf16_tflops"), "measured"
    return 6650.0, 1590.0, "fallback"


def fma_peaks(ctx):
    """This device's FP32 and FP64 CUDA-core FMA rates, TFLOP/s (measured by the library's FMA-chain kernel)."""
    f32, f64 = ctx.measure_peaks()
    return {"fp32_tflops": f32, "fp64_tflops": f64, "kind": "measured (FMA chains)"}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        backend = "gloo" if args.impl == "reference" else "nccl"
        dist.init_process_group(backend, timeout=timedelta(seconds=600))
    return world, rank, local


def max_over_ranks(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_oracle_sample(ds, threads, target_s=12.0):
    """The FP64 C restatement of the Double path on a contiguous subset of the positions (whole detector, whole
    object), one iteration, sized to about `target_s` seconds; returns positions*iter/s and the sample."""
    from oracle import c_oracle
    P = len(ds.positions)
    amps = ds.amplitudes.reshape(P, -1)

    def run(count):
        t0 = time.perf_counter()
        c_oracle.reconstruct(amps[:count].astype(np.float64), ds.positions[:count], ds.object_start, ds.probe,
                             iterations=1, step_size=0.5, threads=threads)
        return time.perf_counter() - t0

    count = max(threads, 16)
    t = run(count)
    count = int(min(P, max(count, count * target_s / max(t, 1e-3))))
    t = run(count)
    return count / t, f"{count} of {P} positions, 1 iteration, full 128x128 detector and 1152x1152 object"


def run_reference(args, world, rank):
    if rank != 0:
        return
    from cubokit_b200 import synthetic
    from oracle import c_oracle
    threads = c_oracle.host_cores()
    ds = synthetic_dataset_cpu()
    P = len(ds.positions)
    amps = ds.amplitudes.reshape(P, -1)
    # one step = a bounded sample of the iteration: a fixed subset of positions, scaled to positions*iter/s
    sample = min(2048, max(threads * 8, 256))
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        c_oracle.reconstruct(amps[:sample].astype(np.float64), ds.positions[:sample], ds.object_start, ds.probe,
                             iterations=1, step_size=0.5, threads=threads)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
    mean = sum(times) / len(times)
    value = sample / mean
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": mean * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"{SCAN}x{SCAN} scan, {DET}x{DET} detector, object 1152x1152, dose 1e5, GD",
                       "form": "CuboPtycho Double CPU path (FP64 C restatement, OpenMP)",
                       "sample_positions_per_step": sample, "l2": "n/a (CPU)"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{sample} of {P} positions per step, 1 iteration each"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def synthetic_dataset_cpu():
    """The same workload's inputs without a GPU: probe and amplitudes from the NumPy oracle (for the CPU arm only)."""
    from cubokit_b200 import synthetic
    from oracle import numpy_oracle
    import cubokit_b200.ptycho as cp
    n = DET
    wavelength = cp.electron_wavelength(300e3)
    dk = 64.0 / n * 1e-3
    sampling = wavelength / (dk * n)
    p = numpy_oracle.probe_build(n, n, sampling, sampling, wavelength, 0.020, 0.002, 100.0)
    p = p * np.sqrt(DOSE / (n * n * np.sum(np.abs(p) ** 2)))
    size = SCAN * STEP + n
    truth = np.exp(1j * synthetic.phase_field(size, size, 1))
    positions = synthetic.raster(SCAN, n, STEP)
    # a sample of rows of the raster is enough for the CPU arm; synthesise only what it reads
    count = 2048
    idx = numpy_oracle.patch_indices(n, n, size, size, positions[:count, 0].astype(np.int64),
                                     positions[:count, 1].astype(np.int64))
    f = np.fft.fft2((p.reshape(1, -1) * truth.reshape(-1)[idx]).reshape(count, n, n))
    rng = np.random.default_rng(2)
    amps = np.sqrt(rng.poisson(np.abs(f) ** 2)).astype(np.float32)
    full = np.zeros((len(positions), n, n), np.float32)
    full[:count] = amps
    start = np.exp(1j * np.random.default_rng(3).normal(0, 0.02, (size, size)))
    return synthetic.Dataset(full, positions, start, p, truth, {})


def run_batched(args, world, rank, local):
    """64 independent reconstructions: scan sides uniform in 24..96 (step 4 px), detectors from {64, 96, 128}^2, each
    with its own seeded phase field (seed 1000 + i) and probe defocus uniform in 50..200 A; FP32 form; gather tiles
    picked by the autotuner per detector size; one graph replay per iteration, `steps` iterations timed."""
    import torch
    import cubokit_b200 as cb
    from cubokit_b200 import autotune, synthetic
    rng = np.random.default_rng(7)
    items, sizes = [], []
    for i in range(64):
        scan = int(rng.integers(24, 97))
        det = int(rng.choice([64, 96, 128]))
        defocus = float(rng.uniform(50, 200))
        ds = synthetic.dataset(scan, det, dose=DOSE, step=STEP, seed_object=1000 + i, seed_noise=2000 + i,
                               seed_start=3000 + i, defocus=defocus, device=local)
        items.append(dict(amplitudes=ds.amplitudes, positions=ds.positions, object=ds.object_start, probe=ds.probe,
                          step_size=0.5, precision="fp32"))
        sizes.append((scan, det))
    tiles = {}
    for it, (scan, det) in zip(items, sizes):
        if det not in tiles:
            tiles[det] = autotune.tune(it["amplitudes"], it["positions"], it["object"], it["probe"], device=local)[0]
        it["gather_tile"] = tiles[det]
    ctx = cb.context(local)
    batch = cb.Batch(items, ctx=ctx)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))
    batch.run(args.warmup)
    barrier(world)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        start.record(stream)
        batch.run(args.steps, synchronize=False)
        stop.record(stream)
        stop.synchronize()
    ms = max_over_ranks(start.elapsed_time(stop), world)
    total_positions = sum(len(it["positions"]) for it in items)
    value = total_positions * args.steps / (ms * 1e-3) * world
    if rank == 0:
        print(json.dumps({
            "metric": "positions*iter/s, 64 independent reconstructions in one captured graph", "value": value,
            "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "batched: 64 reconstructions, scans 24..96 (step 4), detectors {64,96,128}^2, "
                                   "defocus 50..200 A, seeds 1000+i", "positions_total": total_positions,
                       "detectors": {str(d): sum(1 for s in sizes if s[1] == d) for d in (64, 96, 128)},
                       "gather_tiles": {str(d): autotune.NAMES[t] for d, t in tiles.items()}},
            "gpu_launches": batch.launches_per_iteration * args.steps, "graph_launches": args.steps,
            "clocks": clocks.summary()}), flush=True)
    batch.close()


def run_preprocess(args, world, rank, local):
    """Amplitude preprocessing (PtychographyPreparation.amplitudes) over the precision workload's cube: 65,536 patterns
    of 128 x 128 Float32 intensities (the synthetic dataset's squared amplitudes) shifted by a uniform fractional origin
    (0.3, -0.45 px) with the periodic cubic B-spline (py4DSTEM's default order), square-rooted, with both mean
    intensities; one step = one pass over the cube, device-resident in and out.  `e2e` is the host-to-host call."""
    import torch
    import cubokit_b200 as cb
    from cubokit_b200 import synthetic
    ds = synthetic.dataset(args.scan, DET, dose=DOSE, step=STEP, pinned=True, device=local)
    cube_host = (ds.amplitudes.astype(np.float64) ** 2).astype(np.float32)
    count = cube_host.shape[0]
    n = cube_host.shape[1] * cube_host.shape[2]
    origins = (0.3, -0.45)
    ctx = cb.context(local)
    dev = torch.device("cuda", local)
    cube = torch.from_numpy(cube_host).to(dev)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    result = torch.empty_like(cube)  # the amplitudes, written in place every step
    for _ in range(args.warmup):
        out = cb.PtychographyPreparation.amplitudes(cube, origins, ctx=ctx, out=result)
    barrier(world)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ctx.set_timing(True)  # events around each kernel launch, on the stream it is launched on
    with ClockSampler(local) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            out = cb.PtychographyPreparation.amplitudes(cube, origins, ctx=ctx, out=result)
        stop.record(stream)
        stop.synchronize()
    kernel_ms, kernel_launches = ctx.prepare_kernel_stats()
    ctx.set_timing(False)
    ms = max_over_ranks(start.elapsed_time(stop), world)
    value = count * args.steps / (ms * 1e-3) * world
    hbm_peak, _, peak_kind = measured_peaks()
    bytes_step = count * n * 8  # Float32 intensities in, Float32 amplitudes out
    launch_ms = kernel_ms / max(1, kernel_launches)
    e2e = None
    if not args.no_e2e:
        t0 = time.perf_counter()
        host = cb.PtychographyPreparation.amplitudes(cube_host, origins, ctx=ctx)
        e2e_s = max_over_ranks(time.perf_counter() - t0, world)
        e2e = {"value": count / e2e_s * world, "unit": "patterns/s", "seconds": e2e_s,
               "h2d_bytes_per_step": count * n * 4 + count * 16, "d2h_bytes_per_step": count * n * 4 + 16,
               "matches_device": bool(np.array_equal(host.values, out.values.cpu().numpy()))}
    cpu = None
    if rank == 0 and not args.no_cpu:
        from oracle import numpy_oracle
        sample = 64
        t0 = time.perf_counter()
        numpy_oracle.prepare_amplitudes(cube_host[:sample], np.full(sample, origins[0]), np.full(sample, origins[1]),
                                        "cubicSpline")
        cpu = {"value": sample / (time.perf_counter() - t0), "unit": "patterns/s", "cores": 1, "kind": "port",
               "sample": f"{sample} of {count} patterns, NumPy FP64 restatement (FFT prefilter as the reference)"}
    if rank == 0:
        print(json.dumps({
            "metric": "patterns/s, amplitude preprocessing (cubic-spline origin shift, sqrt, mean intensities)",
            "value": value, "unit": "patterns/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 (f32 in and out)", "data": "synthetic",
            "config": {"workload": f"preprocess: {count} patterns of {DET}x{DET}, cubic spline, uniform origin "
                                   f"{origins}", "l2": "cube and amplitudes (4.3 GB each) far larger than L2"},
            "roofline": {"kernel": "prepare_kernel<cubic, 128, 128>", "bound": "hbm",
                         "achieved": bytes_step / (launch_ms * 1e-3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
                         "frac": bytes_step / (launch_ms * 1e-3) / 1e9 / hbm_peak, "peak_kind": peak_kind,
                         "launch_ms": launch_ms, "launches": kernel_launches,
                         "note": "instruction-issue bound (FP64 prefilter and taps), not HBM-bound",
                         "traffic": None},
            "mean_intensity": out.mean_intensity, "clipped_mean_intensity": out.clipped_mean_intensity,
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": 3 * args.steps, "clocks": clocks.summary()}),
            flush=True)


def run_positions(args, world, rank, local):
    """Position correction (PtychographyPositionCorrection) in the FP64 form on the precision workload's data: 65,536
    positions started up to 0.4 px off the data's raster (seeded), per-iteration limit 0.5 A at 0.4 A per pixel; one
    step = one full-batch GD iteration with the position update of every position, the scan tables rebuilt from the
    moved positions before the next one (host work included in the timed region)."""
    import torch
    import cubokit_b200 as cb
    from cubokit_b200 import synthetic
    ds = synthetic.dataset(args.scan, DET, dose=DOSE, step=STEP, pinned=True, device=local)
    P, n = len(ds.positions), DET * DET
    start = ds.positions + np.random.default_rng(5).uniform(-0.4, 0.4, ds.positions.shape)
    settings = dict(step_size=0.5, max_update_distance=0.5, row_sampling=0.4, column_sampling=0.4)
    ctx = cb.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))
    plan = cb.Plan(ds.amplitudes, start, ds.object_start.shape, ds.probe.shape, ctx=ctx, step_size=0.5,
                   precision="fp64", position_correction=cb.PtychographyPositionCorrection(**settings))
    plan.set_state(ds.object_start, ds.probe)
    plan.enqueue(args.warmup)
    ctx.synchronize()
    barrier(world)
    start_ev, stop_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = plan.launch_count
    with ClockSampler(local) as clocks:
        start_ev.record(stream)
        plan.enqueue(args.steps)
        stop_ev.record(stream)
        stop_ev.synchronize()
    ms = max_over_ranks(start_ev.elapsed_time(stop_ev), world)
    launches = plan.launch_count - launches0
    moved = float(np.max(np.abs(plan.positions() - start)))
    plan.set_timing(True)
    timed_iterations = max(2, min(args.steps, 4))
    plan.enqueue(timed_iterations)
    stats = plan.kernel_stats()
    plan.set_timing(False)
    plan.close()
    value = P * args.steps / (ms * 1e-3) * world
    hbm_peak, _, peak_kind = measured_peaks()
    corr_ms, corr_launches = stats["position_correction"]
    corr_ms /= timed_iterations
    # algorithmic bytes of the position update: amplitudes (4n) and the position's shifted probe (16n) read once; the
    # object patches come from L2 (the object is 21 MB)
    corr_bytes = P * 20 * n
    cpu = None
    if rank == 0 and not args.no_cpu:
        from oracle import numpy_oracle as no
        sample = 64
        idx = np.arange(sample)
        amps = ds.amplitudes.reshape(P, DET, DET)[idx].astype(np.float64)
        t0 = time.perf_counter()
        no.reconstruct(amps, start[idx], ds.object_start, ds.probe, iterations=1, step_size=0.5,
                       position_correction=no.PositionCorrection(**settings))
        cpu = {"value": sample / (time.perf_counter() - t0), "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"one iteration over {sample} of {P} positions, NumPy FP64 restatement"}
    if rank == 0:
        per_kind = {k: round(v[0] / timed_iterations, 3) for k, v in stats.items() if v[1]}
        print(json.dumps({
            "metric": "positions*iter/s, GD with position correction (FP64 form, 128^2 detector)", "value": value,
            "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"positions: {P} positions ({args.scan}^2 raster started <= 0.4 px off), "
                                   f"{DET}x{DET} detector, limit 0.5 A at 0.4 A/px",
                       "l2": "amplitudes 4.3 GB, residuals 17 GB: far larger than L2"},
            "roofline": {"kernel": "position update (exit waves, FP64 far fields, 2x2 solves)", "bound": "hbm",
                         "achieved": corr_bytes / (corr_ms * 1e-3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
                         "frac": corr_bytes / (corr_ms * 1e-3) / 1e9 / hbm_peak, "peak_kind": peak_kind,
                         "launch_ms": corr_ms, "note": "three forward plane launches write each position's far "
                                                       "fields, the 2x2 solves read them back; 20 bytes per pixel is "
                                                       "the algorithmic floor",
                         "traffic": None},
            "kernel_ms_per_iteration": per_kind, "moved_px_max": moved,
            "cpu_baseline": cpu, "e2e": None, "gpu_launches": launches, "clocks": clocks.summary()}), flush=True)


def run_mixed(args, world, rank, local):
    """The mixed-state engine (MixedstatePtychography, FP64) on the precision workload's data with 4 probe states from
    the seeded initial-state recipe (py4DSTEM's phase ramps, NumPy RandomState(11)), the centre of mass and the
    orthogonalisation on; one step = one full-batch iteration over all positions and states."""
    import torch
    import cubokit_b200 as cb
    from cubokit_b200 import synthetic
    states = 4
    ds = synthetic.dataset(args.scan, DET, dose=DOSE, step=STEP, pinned=True, device=local)
    P, n = len(ds.positions), DET * DET
    probes = cb.MixedstatePtychography.initial_probes(ds.probe / np.sqrt(states), states, seed=11)
    ctx = cb.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))
    plan = cb.Plan(ds.amplitudes, ds.positions, ds.object_start.shape, ds.probe.shape, ctx=ctx, step_size=0.5,
                   fix_probe_center_of_mass=True, mixed_states=states)
    plan.set_state(ds.object_start, probes)
    plan.enqueue(args.warmup)
    ctx.synchronize()
    barrier(world)
    start_ev, stop_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = plan.launch_count
    with ClockSampler(local) as clocks:
        start_ev.record(stream)
        plan.enqueue(args.steps)
        stop_ev.record(stream)
        stop_ev.synchronize()
    ms = max_over_ranks(start_ev.elapsed_time(stop_ev), world)
    launches = plan.launch_count - launches0
    errors = plan.errors(args.warmup + args.steps)
    plan.set_timing(True)
    timed_iterations = max(2, min(args.steps, 4))
    plan.enqueue(timed_iterations)
    stats = plan.kernel_stats()
    plan.set_timing(False)
    plan.close()
    value = P * args.steps / (ms * 1e-3) * world
    hbm_peak, _, peak_kind = measured_peaks()
    pass_ms = stats["position_pass"][0] / timed_iterations
    # algorithmic bytes of the position pass: amplitudes read once (4n), every state's residual written once (16n)
    pass_bytes = P * (4 + 16 * states) * n
    peaks = fma_peaks(ctx)
    pass_flops = states * P * 10 * n * math.log2(n)  # every state's FFT and inverse (FFT-equivalent)
    cpu = None
    if rank == 0 and not args.no_cpu:
        from oracle import numpy_oracle as no
        sample = 32
        amps = ds.amplitudes.reshape(P, DET, DET)[:sample].astype(np.float64)
        t0 = time.perf_counter()
        no.mixedstate_reconstruct(amps, ds.positions[:sample], ds.object_start, probes, iterations=1, step_size=0.5,
                                  fix_probe_center_of_mass=True)
        cpu = {"value": sample / (time.perf_counter() - t0), "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"one iteration over {sample} of {P} positions, {states} states, NumPy FP64 restatement"}
    if rank == 0:
        per_kind = {k: round(v[0] / timed_iterations, 3) for k, v in stats.items() if v[1]}
        print(json.dumps({
            "metric": f"positions*iter/s, mixed-state GD ({states} probe states, FP64, 128^2 detector)", "value": value,
            "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"mixed: {P} positions ({args.scan}^2 raster), {DET}x{DET} detector, "
                                   f"{states} states, centre of mass + orthogonalisation",
                       "l2": "amplitudes 4.3 GB, residuals 69 GB: far larger than L2"},
            "roofline": {"kernel": "mixed position pass (per state a forward plane launch, the summed-intensity "
                                   "projection, per state an inverse plane launch; FP64)",
                         "bound": "hbm", "achieved": pass_bytes / (pass_ms * 1e-3) / 1e9, "peak": hbm_peak,
                         "unit": "GB/s", "frac": pass_bytes / (pass_ms * 1e-3) / 1e9 / hbm_peak,
                         "peak_kind": peak_kind, "launch_ms": pass_ms,
                         "note": "every state's far field is written, projected in place and read back (the "
                                 "projection needs all states); the plane launches are latency-bound",
                         "traffic": None, "fft_equivalent_tflops": pass_flops / (pass_ms * 1e-3) / 1e12,
                         "frac_of_fp64_fma_peak": pass_flops / (pass_ms * 1e-3) / 1e12 / peaks["fp64_tflops"],
                         "cuda_core_peaks": peaks},
            "kernel_ms_per_iteration": per_kind, "errors_first_last": [errors[0], errors[-1]],
            "cpu_baseline": cpu, "e2e": None, "gpu_launches": launches, "clocks": clocks.summary()}), flush=True)


def run_multislice(args, world, rank, local):
    """The multislice engine (MultislicePtychography, FP64) on the precision workload's data: 4 slices of the start
    object 20 A apart at 300 kV and the data's object sampling; one step = one full-batch iteration (forward through
    every slice, projection, back-propagation with every slice's gradient, the updates)."""
    import torch
    import cubokit_b200 as cb
    from cubokit_b200 import synthetic
    slices, thickness = 4, 20.0
    ds = synthetic.dataset(args.scan, DET, dose=DOSE, step=STEP, pinned=True, device=local)
    P, n = len(ds.positions), DET * DET
    sampling = float(ds.config["sampling_A"])
    wavelength = cb.electron_wavelength(300e3)
    obj = np.stack([ds.object_start] * slices)
    multislice = dict(slices=slices, slice_thicknesses=[thickness] * (slices - 1), wavelength=wavelength,
                      row_sampling=sampling, column_sampling=sampling)
    ctx = cb.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))
    plan = cb.Plan(ds.amplitudes, ds.positions, ds.object_start.shape, ds.probe.shape, ctx=ctx, step_size=0.5,
                   fix_probe_center_of_mass=True, multislice=multislice)
    plan.set_state(obj, ds.probe)
    plan.enqueue(args.warmup)
    ctx.synchronize()
    barrier(world)
    start_ev, stop_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = plan.launch_count
    with ClockSampler(local) as clocks:
        start_ev.record(stream)
        plan.enqueue(args.steps)
        stop_ev.record(stream)
        stop_ev.synchronize()
    ms = max_over_ranks(start_ev.elapsed_time(stop_ev), world)
    launches = plan.launch_count - launches0
    errors = plan.errors(args.warmup + args.steps)
    plan.set_timing(True)
    timed_iterations = max(2, min(args.steps, 4))
    plan.enqueue(timed_iterations)
    stats = plan.kernel_stats()
    plan.set_timing(False)
    plan.close()
    value = P * args.steps / (ms * 1e-3) * world
    hbm_peak, _, peak_kind = measured_peaks()
    pass_ms = stats["position_pass"][0] / timed_iterations
    # algorithmic bytes of the forward pass per pixel: slice 0 writes the wave entering slice 1 (16; the shifted probe
    # and the object come from L2), slices 1 .. L-2 read their entering wave and write the next (32), the last slice
    # reads its entering wave and the amplitude and writes the residual (36): 32 L - 12
    pass_bytes = P * (32 * slices - 12) * n
    peaks = fma_peaks(ctx)
    pass_flops = slices * P * 10 * n * math.log2(n)  # one FFT and one inverse per slice (FFT-equivalent)
    cpu = None
    if rank == 0 and not args.no_cpu:
        from oracle import numpy_oracle as no
        sample = 32
        amps = ds.amplitudes.reshape(P, DET, DET)[:sample].astype(np.float64)
        t0 = time.perf_counter()
        no.multislice_reconstruct(amps, ds.positions[:sample], obj, ds.probe, multislice["slice_thicknesses"],
                                  wavelength, sampling, sampling, iterations=1, step_size=0.5,
                                  fix_probe_center_of_mass=True)
        cpu = {"value": sample / (time.perf_counter() - t0), "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"one iteration over {sample} of {P} positions, {slices} slices, NumPy FP64 restatement"}
    if rank == 0:
        per_kind = {k: round(v[0] / timed_iterations, 3) for k, v in stats.items() if v[1]}
        print(json.dumps({
            "metric": f"positions*iter/s, multislice GD ({slices} slices, FP64, 128^2 detector)", "value": value,
            "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"multislice: {P} positions ({args.scan}^2 raster), {DET}x{DET} detector, "
                                   f"{slices} slices {thickness:g} A apart, 300 kV, centre of mass",
                       "l2": f"amplitudes {P * n * 4 / 1e9:.1f} GB, entering waves and residuals "
                             f"{P * n * 16 * slices / 1e9:.0f} GB: far larger than L2"},
            "roofline": {"kernel": "multislice forward pass (one clustered plane launch per slice: patch product, "
                                   "FP64 FFT, propagator or projection, inverse FFT)",
                         "bound": "hbm", "achieved": pass_bytes / (pass_ms * 1e-3) / 1e9, "peak": hbm_peak,
                         "unit": "GB/s", "frac": pass_bytes / (pass_ms * 1e-3) / 1e9 / hbm_peak,
                         "peak_kind": peak_kind, "launch_ms": pass_ms,
                         "note": "latency-bound: one 512-thread CTA per SM holds half a plane in registers; its "
                                 "load, transform and store phases do not overlap", "traffic": None,
                         "fft_equivalent_tflops": pass_flops / (pass_ms * 1e-3) / 1e12,
                         "frac_of_fp64_fma_peak": pass_flops / (pass_ms * 1e-3) / 1e12 / peaks["fp64_tflops"],
                         "cuda_core_peaks": peaks},
            "kernel_ms_per_iteration": per_kind, "errors_first_last": [errors[0], errors[-1]],
            "cpu_baseline": cpu, "e2e": None, "gpu_launches": launches, "clocks": clocks.summary()}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="both", choices=["both", "all", "fp32", "split_bf16"],
                    help="both: split-BF16 (the headline) and FP32 measured on the same data; all: also the any-size "
                         "FP32 transform (fp32_generic) and the FP64 form")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--scan", type=int, default=SCAN, help="scan side (the benchmark workload is 256)")
    ap.add_argument("--workload", default="precision",
                    choices=["precision", "batched", "preprocess", "positions", "mixed", "multislice"],
                    help="precision: the 256^2-scan 128^2-detector GD (default); batched: 64 independent "
                         "reconstructions of uneven sizes in one graph; preprocess: amplitude preprocessing of the "
                         "precision workload's cube; positions: GD with position correction (FP64 form); mixed: the mixed-state "
                         "engine with 4 probe states (FP64); multislice: the multislice engine with 4 slices (FP64)")
    args = ap.parse_args()
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank)
        barrier(world)
        return

    import torch
    torch.cuda.set_device(local)
    import cubokit_b200 as cb
    from cubokit_b200 import synthetic

    if args.workload == "batched":
        run_batched(args, world, rank, local)
        return
    if args.workload == "preprocess":
        run_preprocess(args, world, rank, local)
        return
    if args.workload == "positions":
        run_positions(args, world, rank, local)
        return
    if args.workload == "mixed":
        run_mixed(args, world, rank, local)
        return
    if args.workload == "multislice":
        run_multislice(args, world, rank, local)
        return

    ds = synthetic.dataset(args.scan, DET, dose=DOSE, step=STEP, pinned=True, device=local)
    P, n = len(ds.positions), DET * DET
    objects = ds.object_start.size
    ctx = cb.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))
    forms = {"both": ["split_bf16", "fp32"], "all": ["split_bf16", "fp32", "fp32_generic", "fp64"]}.get(
        args.form, [args.form])
    results = {}
    for form in forms:
        # fp32_generic: the FP32 form through the any-size shared-memory transform instead of the 128 x 128 kernel
        plan = cb.Plan(ds.amplitudes, ds.positions, ds.object_start.shape, ds.probe.shape, ctx=ctx, step_size=0.5,
                       precision="fp32" if form == "fp32_generic" else form,
                       variant="generic" if form == "fp32_generic" else "auto")
        plan.set_state(ds.object_start, ds.probe)
        plan.enqueue(args.warmup)
        ctx.synchronize()
        barrier(world)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        launches0 = plan.launch_count
        with ClockSampler(local) as clocks:
            torch.cuda.synchronize()
            start.record(stream)
            plan.enqueue(args.steps)
            stop.record(stream)
            stop.synchronize()
        ms = max_over_ranks(start.elapsed_time(stop), world)
        launches = plan.launch_count - launches0
        errors = plan.errors(args.warmup + args.steps)
        obj, _ = plan.get_state()
        # per-kernel device time over separate iterations (events around every launch)
        plan.set_timing(True)
        plan.enqueue(max(3, min(args.steps, 10)))
        stats = plan.kernel_stats()
        plan.set_timing(False)
        plan.close()
        results[form] = dict(ms=ms, launches=launches, errors=errors, object=obj, stats=stats,
                             clocks=clocks.summary())

    head = forms[0]
    r = results[head]
    ms = r["ms"]
    stats = r["stats"]
    bytes_iter, flops_iter = algorithmic(P, n, objects)
    hbm_peak, bf16_peak, peak_kind = measured_peaks()
    value = P * args.steps / (ms * 1e-3) * world
    pass_ms, pass_launches = stats["position_pass"]
    pass_avg_s = pass_ms / max(pass_launches, 1) * 1e-3
    fft_flops = P * (10 * n * math.log2(n) + 40 * n)  # algorithmic: two 2-D FFTs + 40 flops per pixel per position
    if head == "split_bf16":
        # executed tensor work: 4 stages per position, each the real 128 x 128 x 128 product C B of the re and of the im
        # plane, 3 bf16 split products each: 48 x 2 x 128^3 = 100.7 MFLOP per position
        tensor_flops = P * 4 * 2 * 3 * 2 * 128 ** 3
        roofline = {"kernel": "position_pass (bf16_position_kernel)", "bound": "tensor",
                    "achieved": tensor_flops / pass_avg_s / 1e12, "peak": bf16_peak, "unit": "TFLOP/s",
                    "frac": tensor_flops / pass_avg_s / 1e12 / bf16_peak, "peak_kind": peak_kind + " (bf16 dense burst)",
                    # ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch at 4096 positions (748.3 MB,
                    # profiles/position_pass_bf16_scan64_det128.md), scaled to this launch by positions
                    "traffic": 748.3e6 / 4096 * P, "executed_tflop_per_launch": tensor_flops / 1e12,
                    "note": "executed split-BF16 DFT-GEMM flops (100.7 MFLOP per position); the FFT-equivalent "
                            "algorithmic rate is fft_equivalent_tflops",
                    "fft_equivalent_tflops": fft_flops / pass_avg_s / 1e12,
                    "amplitude_hbm_gbs": P * 4 * n / pass_avg_s / 1e9}
    else:
        roofline = {"kernel": "position_pass (fast128_kernel)", "bound": "hbm",
                    "achieved": P * 4 * n / pass_avg_s / 1e9, "peak": hbm_peak, "unit": "GB/s",
                    "frac": P * 4 * n / pass_avg_s / 1e9 / hbm_peak, "peak_kind": peak_kind, "traffic": None,
                    "note": "algorithmic bytes = amplitudes read (4n per position); the FP32 form is bound by FP32 "
                            "issue, reported as fft_equivalent_tflops",
                    "fft_equivalent_tflops": fft_flops / pass_avg_s / 1e12}
    roofline["iteration_hbm_gbs"] = bytes_iter / (ms / args.steps * 1e-3) / 1e9
    total_stat_ms = sum(v[0] for v in stats.values())

    peaks = fma_peaks(ctx)
    forms_out = {}
    for form, fr in results.items():
        pass_form_ms = fr["stats"]["position_pass"][0] / max(fr["stats"]["position_pass"][1], 1)
        forms_out[form] = {"value": P * args.steps / (fr["ms"] * 1e-3) * world, "ms_per_step": fr["ms"] / args.steps,
                           "position_pass_ms": pass_form_ms, "error_last": float(fr["errors"][-1]),
                           "fft_equivalent_tflops": fft_flops / (pass_form_ms * 1e-3) / 1e12}
        if form in ("fp32", "fp32_generic"):
            forms_out[form]["frac_of_fp32_fma_peak"] = forms_out[form]["fft_equivalent_tflops"] / peaks["fp32_tflops"]
        if form == "fp64":
            forms_out[form]["frac_of_fp64_fma_peak"] = forms_out[form]["fft_equivalent_tflops"] / peaks["fp64_tflops"]
    roofline["cuda_core_peaks"] = peaks
    comparison = None
    if "split_bf16" in results and "fp32" in results:
        a, b = results["split_bf16"]["object"], results["fp32"]["object"]
        comparison = {"ratio_split_bf16_over_fp32": forms_out["split_bf16"]["value"] / forms_out["fp32"]["value"],
                      "object_rel_l2_split_bf16_vs_fp32": float(np.linalg.norm(a - b) / np.linalg.norm(b)),
                      "iterations_compared": args.warmup + args.steps}
        for other in ("fp32_generic", "fp64"):
            if other in results:
                c = results[other]["object"]
                comparison[f"ratio_split_bf16_over_{other}"] = (forms_out["split_bf16"]["value"] /
                                                                forms_out[other]["value"])
                comparison[f"object_rel_l2_split_bf16_vs_{other}"] = float(np.linalg.norm(a - c) / np.linalg.norm(c))

    e2e = None
    if not args.no_e2e:
        t0 = time.perf_counter()
        rr = cb.SingleslicePtychography.reconstruct(ds.amplitudes, ds.positions, ds.object_start, ds.probe,
                                                    iterations=args.steps, step_size=0.5, precision=head,
                                                    device=local)
        e2e_s = max_over_ranks(time.perf_counter() - t0, world)
        h2d = ds.amplitudes.nbytes + ds.positions.nbytes + objects * 16 + n * 16
        d2h = objects * 16 + n * 16 + args.steps * 8
        e2e = {"value": P * args.steps / e2e_s * world, "unit": UNIT, "seconds": e2e_s, "form": head,
               "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
               "final_error": float(rr.errors[-1])}

    cpu = None
    if rank == 0 and not args.no_cpu:
        from oracle import c_oracle
        threads = c_oracle.host_cores()
        v, sample = cpu_oracle_sample(ds, threads)
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16x3/f32" if head == "split_bf16" else "f32", "data": "synthetic",
            "config": {"workload": f"{args.scan}x{args.scan} scan, step {STEP} px, {DET}x{DET} detector, object "
                                   f"{ds.object_start.shape[0]}x{ds.object_start.shape[1]}, dose 1e5, GD step 0.5",
                       "form": head, "positions": P, "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                       "l2": f"inputs larger than L2 ({P * n * 4 / 1e9:.2f} GB amplitudes, "
                             f"{P * n * 8 / 1e9:.2f} GB residuals; L2 126 MB)"},
            "forms": forms_out, "comparison": comparison, "roofline": roofline,
            "kernels": {k: {"ms_per_launch": v[0] / max(v[1], 1), "launches": v[1],
                            "share": v[0] / total_stat_ms if total_stat_ms else None} for k, v in stats.items() if v[1]},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": r["launches"], "clocks": r["clocks"],
            "errors_first_last": [float(r["errors"][0]), float(r["errors"][-1])],
        }
        print(json.dumps(line), flush=True)
    barrier(world)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
