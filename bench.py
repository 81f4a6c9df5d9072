"""Benchmark of the single-slice ptychography GD engine on B200.

Workload (the precision-form configuration): 256 x 256 raster scan, step 4 px, 128 x 128 detector, object 1152 x 1152,
Float32 amplitudes at 1e5 e/pattern, seeded synthetic data (cubokit_b200.synthetic).  One step = one full-batch GD
iteration over all 65,536 positions.  Metric: positions * iterations / s.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--form both|fp32|split_bf16] [--impl ours|reference]

The headline form is split-BF16 (the DFT-matrix products on the tensor cores); the FP32 form runs on the same data in
the same invocation and the line reports both and their ratio.  `parity` holds each form's relative L2 object error
against the FP64 device form after every one of 100 iterations on the same data (bounds: split-BF16 1e-4, FP32 1e-5);
`extras` adds the FP32 form at the 128^2-scan workload (50 iterations against the FP64 form, and the FP64 form against
the FP64 C restatement of the Double path after 2 iterations), the CPU-path workload run exactly (32^2 scan, 64^2
detector, 20 iterations, one core and all cores) and the 64-reconstruction batch.

`value` is device-timed (CUDA events on the engine's stream) with amplitudes resident in HBM; the 4.3 GB amplitude
stack and the 8.6 GB residual buffer are far larger than L2, so no flush is needed.  `e2e` is one
SingleslicePtychography.reconstruct call (the public API) of K iterations from pinned host buffers, host<->device
copies, validation and plan set-up included, timed by the wall clock around the blocking call.  With --gpus N > 1
(torchrun), the ranks share ONE reconstruction of the workload (cubokit_b200.sharded: contiguous position bands, the
bands' gradient sums added in rank order after an all-gather of each rank's touched object rows): value = all
positions * iterations / the slowest rank's device time, scaling "strong".  The other --workload choices run
independent replicas per rank.
`cpu_baseline` and `--impl reference` time the same code: the FP64 C restatement of CuboPtycho's Double CPU path
(oracle/) over the first 4,096 positions of the workload, one iteration per step, OpenMP over all host cores
(`cpu_baseline` also gives the single-core rate).
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
    """HBM copy GB/s and dense BF16 TFLOP/s (burst and sustained) measured on this pool's B200s, else the fallback."""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d["hbm_gbs"], "bf16_tflops": d.get("bf16_tflops"),
                "bf16_tflops_sustained": d.get("bf16_tflops_sustained"), "kind": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0, "kind": "fallback"}


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per position of one position-pass launch, from ncu on a
# 4,096-position launch (64^2 scan, 128^2 detector) of each kernel, divided by its positions: amplitudes read (64 KB)
# plus residuals written (128 KB) less what stays in L2.  The bench scales them to its launch by positions.
PASS_DRAM_BYTES_PER_POSITION = {"split_bf16": 748.1e6 / 4096, "fp32": None}


def position_pass_roofline(head, stats, P, n, objects, ms_iter, peaks, fma):
    """The dominant kernel (the position pass) against the roofline that binds its algorithmic work.

    Algorithmic work per position: the amplitudes read once (4n bytes) and two n-point 2-D FFTs plus 40 flops per
    pixel (10 n log2 n + 40 n flops).  At the measured peaks the bytes take longer than the flops on any pipe the pass
    could use, so HBM binds: achieved = 4 n P / launch time, frac = achieved / measured HBM copy rate.  The executed
    split-BF16 tensor work (100.7 MFLOP per position of real 128 x 128 x 128 products) is reported beside it as a
    utilisation figure, not as the roofline."""
    pass_ms, pass_launches = stats["position_pass"]
    pass_s = pass_ms / max(pass_launches, 1) * 1e-3
    pass_bytes = P * 4 * n
    achieved = pass_bytes / pass_s / 1e9
    per_position = PASS_DRAM_BYTES_PER_POSITION.get(head)
    traffic = per_position * P if per_position else None
    bytes_iter = P * 4 * n + 16 * objects + 16 * n
    fft_flops = P * (10 * n * math.log2(n) + 40 * n)
    out = {"kernel": "position_pass (bf16_position_kernel)" if head == "split_bf16" else "position_pass (fast128_kernel)",
           "bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
           "frac": achieved / peaks["hbm_gbs"], "peak_kind": f"{peaks['kind']} HBM copy",
           "algorithmic_bytes_per_launch": pass_bytes, "launch_ms": pass_s * 1e3,
           "traffic": traffic, "traffic_over_algorithmic": traffic / pass_bytes if traffic else None,
           "traffic_source": "ncu DRAM bytes per position of a 4,096-position launch, scaled to this launch"
           if traffic else None,
           "fft_equivalent_tflops": fft_flops / pass_s / 1e12,
           "iteration": {"algorithmic_bytes": bytes_iter, "ms": ms_iter,
                         "gbs": bytes_iter / (ms_iter * 1e-3) / 1e9,
                         "frac": bytes_iter / (ms_iter * 1e-3) / 1e9 / peaks["hbm_gbs"]},
           "cuda_core_peaks": fma}
    if head == "split_bf16":
        tensor_flops = P * 4 * 2 * 3 * 2 * 128 ** 3  # 4 stages x 2 planes x 3 split products x 2 * 128^3
        t = tensor_flops / pass_s / 1e12
        out.update({"tensor_exec_tflops": t, "tensor_exec_frac": t / peaks["bf16_tflops"],
                    "tensor_exec_frac_sustained": t / peaks["bf16_tflops_sustained"]
                    if peaks.get("bf16_tflops_sustained") else None,
                    "tensor_exec_note": "executed split-BF16 DFT products (100.7 MFLOP per position) against the "
                                        "dense BF16 peak: tensor-pipe utilisation, not the roofline fraction"})
    else:
        out["frac_of_fp32_fma_peak"] = out["fft_equivalent_tflops"] / fma["fp32_tflops"]
    return out


def error_curves(ds, ctx, iterations, forms):
    """Relative L2 error of the object and of the probe of each form against the FP64 device form after every
    iteration, all started from the same state on the same data, plus each form's normalised errors."""
    import cubokit_b200 as cb
    plans = {}
    try:
        for f in ("fp64",) + tuple(forms):
            plans[f] = cb.Plan(ds.amplitudes, ds.positions, ds.object_start.shape, ds.probe.shape, ctx=ctx,
                               step_size=0.5, precision=f)
            plans[f].set_state(ds.object_start, ds.probe)
        obj = {f: [] for f in forms}
        prb = {f: [] for f in forms}
        for _ in range(iterations):
            for p in plans.values():
                p.enqueue(1)
            ro, rp = plans["fp64"].get_state()
            no, npb = np.linalg.norm(ro), np.linalg.norm(rp)
            for f in forms:
                o, pr = plans[f].get_state()
                obj[f].append(float(np.linalg.norm(o - ro) / no))
                prb[f].append(float(np.linalg.norm(pr - rp) / npb))
        errors = {f: [float(e) for e in plans[f].errors(iterations)] for f in plans}
    finally:
        for p in plans.values():
            p.close()
    return {"object": obj, "probe": prb, "errors": errors}


def curve_summary(curves, bounds, what):
    out = {"what": what, "iterations": len(next(iter(curves["object"].values())))}
    for f, c in curves["object"].items():
        out[f] = {"object_rel_l2_max": max(c), "object_rel_l2_last": c[-1], "bound": bounds[f],
                  "within_bound_every_iteration": bool(max(c) <= bounds[f]),
                  "probe_rel_l2_max": max(curves["probe"][f]),
                  "object_rel_l2_per_iteration": [float(f"{v:.3g}") for v in c],
                  "error_last": curves["errors"][f][-1], "error_last_fp64": curves["errors"]["fp64"][-1]}
    return out


FP32_SCAN, FP32_ITERATIONS = 128, 50
CPU_SCAN, CPU_DET, CPU_DOSE, CPU_ITERATIONS = 32, 64, 1e4, 20
BATCH_STEPS = 5


def fp32_workload_parity(ctx, local):
    """The plain FP32 form at 128^2 scan, 128^2 detector, object 640^2: its object error against the FP64 device form
    after each of 50 iterations, and the FP64 device form against the FP64 C restatement of the Double path after 2
    iterations on the same data (all host cores)."""
    from cubokit_b200 import synthetic
    from oracle import c_oracle
    ds = synthetic.dataset(FP32_SCAN, DET, dose=DOSE, step=STEP, pinned=True, device=local)
    P = len(ds.positions)
    out = curve_summary(error_curves(ds, ctx, FP32_ITERATIONS, ("fp32",)), {"fp32": 1e-5},
                        f"{FP32_SCAN}^2 scan, 128^2 detector, object {ds.object_start.shape[0]}^2, "
                        f"{FP32_ITERATIONS} iterations, FP32 against the FP64 form")
    import cubokit_b200 as cb
    plan = cb.Plan(ds.amplitudes, ds.positions, ds.object_start.shape, ds.probe.shape, ctx=ctx, step_size=0.5,
                   precision="fp64")
    plan.set_state(ds.object_start, ds.probe)
    dev_err = plan.iterate(2)
    do, dp = plan.get_state()
    plan.close()
    threads = c_oracle.host_cores()
    t0 = time.perf_counter()
    oo, op, oe = c_oracle.reconstruct(ds.amplitudes.reshape(P, -1).astype(np.float64), ds.positions, ds.object_start,
                                      ds.probe, iterations=2, step_size=0.5, threads=threads,
                                      shift_every_position=False)
    t = time.perf_counter() - t0
    out["fp64_vs_c_oracle"] = {
        "iterations": 2, "object_rel_l2": float(np.linalg.norm(do - oo) / np.linalg.norm(oo)),
        "object_max_abs": float(np.max(np.abs(do - oo))),
        "probe_rel_l2": float(np.linalg.norm(dp - op) / np.linalg.norm(op)),
        "errors_rel": float(np.max(np.abs(np.asarray(dev_err) - oe) / np.abs(oe))),
        "c_oracle_seconds": t, "c_oracle_threads": threads}
    return out


def cpu_workload(ctx, local, with_cpu=True):
    """The CPU-path workload exactly (32^2 raster, step 4, 64^2 detector, object 192^2, 1e4 e/pattern, 20 iterations):
    the FP64 C restatement of the Double path on one core and on all host cores, and the FP32 GPU form on the same
    data with its object error against that restatement."""
    import torch
    import cubokit_b200 as cb
    from cubokit_b200 import synthetic
    from oracle import c_oracle
    ds = synthetic.dataset(CPU_SCAN, CPU_DET, dose=CPU_DOSE, step=STEP, pinned=True, device=local)
    P = len(ds.positions)
    amps = ds.amplitudes.reshape(P, -1).astype(np.float64)
    out = {"workload": f"{CPU_SCAN}^2 scan, step {STEP}, {CPU_DET}^2 detector, object "
                       f"{ds.object_start.shape[0]}^2, dose {CPU_DOSE:g}, {CPU_ITERATIONS} iterations",
           "positions": P}
    threads = c_oracle.host_cores()
    ref = None
    if with_cpu:
        for label, th in (("one_core", 1), ("all_cores", threads)):
            t0 = time.perf_counter()
            ref = c_oracle.reconstruct(amps, ds.positions, ds.object_start, ds.probe, iterations=CPU_ITERATIONS,
                                       step_size=0.5, threads=th)
            t = time.perf_counter() - t0
            out[label] = {"seconds": t, "value": P * CPU_ITERATIONS / t, "unit": UNIT, "cores": th,
                          "cpu_model": cpu_model()}
    plan = cb.Plan(ds.amplitudes, ds.positions, ds.object_start.shape, ds.probe.shape, ctx=ctx, step_size=0.5,
                   precision="fp32")
    plan.set_state(ds.object_start, ds.probe)
    plan.enqueue(3)
    ctx.synchronize()
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))
    plan.set_state(ds.object_start, ds.probe)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    plan.enqueue(CPU_ITERATIONS)
    stop.record(stream)
    stop.synchronize()
    ms = start.elapsed_time(stop)
    o, _ = plan.get_state()
    plan.close()
    out["gpu_fp32"] = {"value": P * CPU_ITERATIONS / (ms * 1e-3), "unit": UNIT, "ms": ms}
    if ref is not None:
        out["gpu_fp32"]["object_rel_l2_vs_c_oracle"] = float(np.linalg.norm(o - ref[0]) / np.linalg.norm(ref[0]))
    return out


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
        # CUBO_BENCH_BACKEND=gloo: the GPU arm's collectives through host memory, so that several ranks can share one
        # GPU in a test (their kernels never wait on one another); the benchmark itself uses NCCL
        backend = "gloo" if args.impl == "reference" else os.environ.get("CUBO_BENCH_BACKEND", "nccl")
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


CPU_SAMPLE_ALL = 4096  # positions per all-core step of the CPU restatement (its per-call set-up stays below 5 %)
CPU_SAMPLE_ONE = 512   # positions per single-core step


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_iteration(amps, positions, obj, probe, count, threads):
    """One GD iteration of the FP64 C restatement of the Double CPU path over positions [0, count) (whole detector,
    whole object); returns its wall time in seconds."""
    from oracle import c_oracle
    a = np.ascontiguousarray(amps[:count], np.float64)
    t0 = time.perf_counter()
    c_oracle.reconstruct(a, positions[:count], obj, probe, iterations=1, step_size=0.5, threads=threads)
    return time.perf_counter() - t0


def cpu_rates(amps, positions, obj, probe, repeats=3):
    """The CPU baseline both arms report: positions*iter/s of the C restatement on all host cores (median of
    `repeats` one-iteration calls over CPU_SAMPLE_ALL positions) and on one core (CPU_SAMPLE_ONE positions)."""
    from oracle import c_oracle
    threads = c_oracle.host_cores()
    P = len(positions)
    count_all, count_one = min(P, CPU_SAMPLE_ALL), min(P, CPU_SAMPLE_ONE)
    all_t = [cpu_iteration(amps, positions, obj, probe, count_all, threads) for _ in range(repeats)]
    one_t = [cpu_iteration(amps, positions, obj, probe, count_one, 1) for _ in range(max(1, repeats - 1))]
    return {"value": count_all / statistics.median(all_t), "unit": UNIT, "cores": threads, "kind": "port",
            "cpu_model": cpu_model(),
            "sample": f"one GD iteration over the first {count_all} of {P} positions (whole 128x128 detector and "
                      f"object), median of {repeats}, FP64 C restatement of the Double path, OpenMP over positions",
            "single_core": {"value": count_one / statistics.median(one_t), "unit": UNIT, "cores": 1,
                            "sample": f"one GD iteration over the first {count_one} positions, median of "
                                      f"{max(1, repeats - 1)}"}}


def run_reference(args, world, rank):
    if rank != 0:
        return
    from oracle import c_oracle
    threads = c_oracle.host_cores()
    ds = synthetic_dataset_cpu()
    P = len(ds.positions)
    amps = ds.amplitudes.reshape(P, -1)
    # one step = a bounded sample of the iteration: the first CPU_SAMPLE_ALL positions, scaled to positions*iter/s
    sample = min(P, CPU_SAMPLE_ALL)
    times = []
    for i in range(args.warmup + args.steps):
        dt = cpu_iteration(amps, ds.positions, ds.object_start, ds.probe, sample, threads)
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
                             "cpu_model": cpu_model(),
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
    count = CPU_SAMPLE_ALL
    idx = numpy_oracle.patch_indices(n, n, size, size, positions[:count, 0].astype(np.int64),
                                     positions[:count, 1].astype(np.int64))
    f = np.fft.fft2((p.reshape(1, -1) * truth.reshape(-1)[idx]).reshape(count, n, n))
    rng = np.random.default_rng(2)
    amps = np.sqrt(rng.poisson(np.abs(f) ** 2)).astype(np.float32)
    full = np.zeros((len(positions), n, n), np.float32)
    full[:count] = amps
    start = np.exp(1j * np.random.default_rng(3).normal(0, 0.02, (size, size)))
    return synthetic.Dataset(full, positions, start, p, truth, {})


BATCH_ITEMS = 64


def batched_items(local):
    """The batched workload's inputs: 64 independent reconstructions, scan sides uniform in 24..96 (step 4 px),
    detectors from {64, 96, 128}^2, each with its own seeded phase field (seed 1000 + i) and probe defocus uniform in
    50..200 A; FP32 form; gather tiles picked by the autotuner per detector size."""
    from cubokit_b200 import autotune, synthetic
    rng = np.random.default_rng(7)
    items, sizes = [], []
    for i in range(BATCH_ITEMS):
        scan = int(rng.integers(24, 97))
        det = int(rng.choice([64, 96, 128]))
        defocus = float(rng.uniform(50, 200))
        ds = synthetic.dataset(scan, det, dose=DOSE, step=STEP, seed_object=1000 + i, seed_noise=2000 + i,
                               seed_start=3000 + i, defocus=defocus, device=local)
        items.append(dict(amplitudes=ds.amplitudes, positions=ds.positions, object=ds.object_start, probe=ds.probe,
                          step_size=0.5, precision="fp32"))
        sizes.append((scan, det))
    tiles, shapes = {}, {}
    for it, (scan, det) in zip(items, sizes):
        if det not in tiles:
            tiles[det] = autotune.tune(it["amplitudes"], it["positions"], it["object"], it["probe"], device=local)[0]
            shapes[det] = autotune.tune_pass(it["amplitudes"], it["positions"], it["object"], it["probe"],
                                             device=local)[0]
        it["gather_tile"] = tiles[det]
        it["pass_shape"] = shapes[det]
    return items, sizes, (tiles, shapes)


def measure_batched(steps, warmup, world, local):
    """One graph replay per iteration of the 64-reconstruction batch; `steps` iterations timed on the device."""
    import torch
    import cubokit_b200 as cb
    from cubokit_b200 import autotune
    items, sizes, (tiles, shapes) = batched_items(local)
    ctx = cb.context(local)
    batch = cb.Batch(items, ctx=ctx)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))
    batch.run(warmup)
    barrier(world)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        start.record(stream)
        batch.run(steps, synchronize=False)
        stop.record(stream)
        stop.synchronize()
    ms = max_over_ranks(start.elapsed_time(stop), world)
    total_positions = sum(len(it["positions"]) for it in items)
    # one reconstruction of each detector size alone (a 60 x 60 scan, the batch's mean side), to set the batch's rate
    # against the single-reconstruction rate at equal detector sizes
    from cubokit_b200 import synthetic
    single = {}
    for det in (64, 96, 128):
        ds = synthetic.dataset(60, det, dose=DOSE, step=STEP, seed_object=77, seed_noise=78, seed_start=79,
                               device=local)
        plan = cb.Plan(ds.amplitudes, ds.positions, ds.object_start.shape, ds.probe.shape, ctx=ctx, step_size=0.5,
                       precision="fp32", gather_tile=tiles.get(det, 0), pass_shape=shapes.get(det, 0))
        plan.set_state(ds.object_start, ds.probe)
        plan.enqueue(warmup)
        ctx.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        plan.enqueue(steps)
        b.record(stream)
        b.synchronize()
        single[str(det)] = len(ds.positions) * steps / (a.elapsed_time(b) * 1e-3)
        plan.close()
    by_det = {d: sum(len(it["positions"]) for it, s in zip(items, sizes) if s[1] == d) for d in (64, 96, 128)}
    single_equivalent = total_positions / sum(by_det[d] / single[str(d)] for d in (64, 96, 128) if by_det[d])
    out = {"value": total_positions * steps / (ms * 1e-3) * world, "unit": UNIT, "ms_per_step": ms / steps,
           "single_reconstruction_by_detector": {"value": single, "unit": UNIT, "scan": "60x60, FP32 form"},
           "single_equivalent_value": single_equivalent,
           "batch_over_single_equivalent": total_positions * steps / (ms * 1e-3) * world / single_equivalent,
           "steps": steps, "warmup": warmup, "positions_total": total_positions,
           "positions_by_detector": {str(d): sum(len(it["positions"]) for it, s in zip(items, sizes) if s[1] == d)
                                     for d in (64, 96, 128)},
           "detectors": {str(d): sum(1 for s in sizes if s[1] == d) for d in (64, 96, 128)},
           "gather_tiles": {str(d): autotune.NAMES[t] for d, t in tiles.items()},
           "pass_shapes": {str(d): autotune.PASS_NAMES[t] for d, t in shapes.items()},
           "gpu_launches": batch.launches_per_iteration * steps, "graph_launches": steps, "clocks": clocks.summary()}
    batch.close()
    return out


def run_batched(args, world, rank, local):
    """The batched workload alone (`--workload batched`)."""
    r = measure_batched(args.steps, args.warmup, world, local)
    if rank == 0:
        print(json.dumps({
            "metric": "positions*iter/s, 64 independent reconstructions in one captured graph", "value": r["value"],
            "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": "batched: 64 reconstructions, scans 24..96 (step 4), detectors {64,96,128}^2, "
                                   "defocus 50..200 A, seeds 1000+i", "positions_total": r["positions_total"],
                       "detectors": r["detectors"], "gather_tiles": r["gather_tiles"],
                       "pass_shapes": r["pass_shapes"]},
            "gpu_launches": r["gpu_launches"], "graph_launches": r["graph_launches"], "clocks": r["clocks"]}),
            flush=True)


def sum_over_ranks(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t)
    return float(t.item())


def run_sharded(args, world, rank, local):
    """--gpus N > 1: ONE reconstruction of the workload sharded over the ranks (cubokit_b200.sharded: rank r takes
    the r-th contiguous band of the positions; every iteration each rank runs its band's position pass and gathers,
    the bands' gradient sums are added in rank order after an all-gather of each rank's touched object rows, and
    every rank applies the same update).  value = all positions * iterations / the slowest rank's device time
    (strong scaling: the total work is the workload's whatever N is)."""
    import torch
    from cubokit_b200 import sharded, synthetic
    # every rank builds the same inputs (the same seeds) and uploads its own band; pageable host memory, as N ranks
    # pinning the whole stack each would lock N x 4.3 GB of host memory
    ds = synthetic.dataset(args.scan, DET, dose=DOSE, step=STEP, pinned=False, device=local)
    P, n = len(ds.positions), DET * DET
    form = "fp32" if args.form == "fp32" else "split_bf16"
    run = sharded.ShardedRun(ds.amplitudes, ds.positions, ds.object_start, ds.probe, precision=form, device=local,
                             step_size=0.5)
    try:
        run.enqueue(args.warmup)
        run.ctx.synchronize()
        barrier(world)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        launches0 = run.plan.launch_count
        with ClockSampler(local) as clocks:
            start.record(run.stream)
            run.enqueue(args.steps)
            stop.record(run.stream)
            stop.synchronize()
        ms = max_over_ranks(start.elapsed_time(stop), world)
        launches = sum_over_ranks(run.plan.launch_count - launches0, world)
        errors = run.result().errors
    finally:
        run.close()
    value = P * args.steps / (ms * 1e-3)
    e2e = None
    if not args.no_e2e:
        barrier(world)
        t0 = time.perf_counter()
        r = sharded.reconstruct(ds.amplitudes, ds.positions, ds.object_start, ds.probe, iterations=args.steps,
                                precision=form, device=local, step_size=0.5)
        e2e_s = max_over_ranks(time.perf_counter() - t0, world)
        lo, hi = sharded.band_bounds(P, world, rank)
        h2d = sum_over_ranks((hi - lo) * n * 4 + (hi - lo) * 16 + ds.object_start.size * 16 + n * 16, world)
        d2h = sum_over_ranks(ds.object_start.size * 16 + n * 16 + args.steps * 8, world)
        e2e = {"value": P * args.steps / e2e_s, "unit": UNIT, "seconds": e2e_s, "form": form,
               "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
               "final_error": float(r.errors[-1])}
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "bf16x3/f32" if form == "split_bf16" else "f32", "data": "synthetic",
            "config": {"workload": f"{args.scan}x{args.scan} scan, step {STEP} px, {DET}x{DET} detector, object "
                                   f"{ds.object_start.shape[0]}x{ds.object_start.shape[1]}, dose 1e5, GD step 0.5",
                       "form": form, "positions": P,
                       "parallelism": f"one reconstruction in {world} position bands (ordered halo exchange)",
                       "l2": f"inputs larger than L2 ({P * n * 4 / 1e9:.2f} GB amplitudes in all)"},
            "roofline": None, "cpu_baseline": None, "e2e": e2e, "gpu_launches": launches, "clocks": clocks.summary(),
            "errors_first_last": [float(errors[0]), float(errors[-1])]}), flush=True)


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
    _pk = measured_peaks()
    hbm_peak, peak_kind = _pk["hbm_gbs"], _pk["kind"]
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
    _pk = measured_peaks()
    hbm_peak, peak_kind = _pk["hbm_gbs"], _pk["kind"]
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
    _pk = measured_peaks()
    hbm_peak, peak_kind = _pk["hbm_gbs"], _pk["kind"]
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


LARGE_DET, LARGE_SCAN = 256, 64


def run_large_detector(args, world, rank, local):
    """The FP32 form on a 256 x 256 detector (more pixels than one CTA's plane holds: the global-memory pass of
    global32.cu), a 64^2 raster scan (--scan other than 256 sets it), step 4; one step = one full-batch iteration."""
    import torch
    import cubokit_b200 as cb
    from cubokit_b200 import synthetic
    from oracle import c_oracle
    scan = LARGE_SCAN if args.scan == SCAN else args.scan
    ds = synthetic.dataset(scan, LARGE_DET, dose=DOSE, step=STEP, pinned=True, device=local)
    P, n = len(ds.positions), LARGE_DET * LARGE_DET
    ctx = cb.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))
    plan = cb.Plan(ds.amplitudes, ds.positions, ds.object_start.shape, ds.probe.shape, ctx=ctx, step_size=0.5,
                   precision="fp32")
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
    errors = plan.errors(args.warmup + args.steps)
    plan.set_timing(True)
    timed_iterations = max(2, min(args.steps, 4))
    plan.enqueue(timed_iterations)
    stats = plan.kernel_stats()
    plan.set_timing(False)
    plan.close()
    value = P * args.steps / (ms * 1e-3) * world
    _pk = measured_peaks()
    hbm_peak, peak_kind = _pk["hbm_gbs"], _pk["kind"]
    pass_ms = stats["position_pass"][0] / timed_iterations
    pass_bytes = P * 4 * n  # algorithmic: the amplitudes, once
    moved = P * 44 * n  # the three launches: 8n written, 8n + 4n read and 8n written, 8n read and 8n written
    cpu = None
    if rank == 0 and not args.no_cpu:
        threads = c_oracle.host_cores()
        sample = min(P, 256)
        t = cpu_iteration(ds.amplitudes.reshape(P, -1), ds.positions, ds.object_start, ds.probe, sample, threads)
        cpu = {"value": sample / t, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"one GD iteration over the first {sample} of {P} positions (whole detector and object), "
                         f"FP64 C restatement of the Double path, OpenMP over positions"}
    if rank == 0:
        per_kind = {k: round(v[0] / timed_iterations, 3) for k, v in stats.items() if v[1]}
        print(json.dumps({
            "metric": f"positions*iter/s, FP32 GD on a {LARGE_DET}^2 detector", "value": value, "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"large detector: {P} positions ({scan}^2 raster, step {STEP} px), "
                                   f"{LARGE_DET}x{LARGE_DET} detector, object {ds.object_start.shape[0]}^2",
                       "l2": f"amplitudes {P * n * 4 / 1e9:.2f} GB, residuals {P * n * 8 / 1e9:.2f} GB: larger "
                             f"than L2"},
            "roofline": {"kernel": "global-memory FP32 position pass (rows with the exit wave, columns around the "
                                   "projection, inverse rows)",
                         "bound": "hbm", "achieved": pass_bytes / (pass_ms * 1e-3) / 1e9, "peak": hbm_peak,
                         "unit": "GB/s", "frac": pass_bytes / (pass_ms * 1e-3) / 1e9 / hbm_peak,
                         "peak_kind": peak_kind, "launch_ms": pass_ms,
                         "moved_gbs": moved / (pass_ms * 1e-3) / 1e9,
                         "note": "algorithmic bytes 4n per position; the three launches move 44n",
                         "traffic": None},
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
    _pk = measured_peaks()
    hbm_peak, peak_kind = _pk["hbm_gbs"], _pk["kind"]
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
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the per-iteration error curves against the FP64 form and the smaller workloads")
    ap.add_argument("--parity-iterations", type=int, default=100)
    ap.add_argument("--no-batched", action="store_true", help="skip the 64-reconstruction batch in the extras")
    ap.add_argument("--scan", type=int, default=SCAN, help="scan side (the benchmark workload is 256)")
    ap.add_argument("--workload", default="precision",
                    choices=["precision", "batched", "preprocess", "positions", "mixed", "multislice",
                             "large_detector"],
                    help="precision: the 256^2-scan 128^2-detector GD (default); batched: 64 independent "
                         "reconstructions of uneven sizes in one graph; preprocess: amplitude preprocessing of the "
                         "precision workload's cube; positions: GD with position correction (FP64 form); mixed: "
                         "the mixed-state engine with 4 probe states (FP64); multislice: the multislice engine with 4 "
                         "slices (FP64); "
                         "large_detector: the FP32 form on a 256^2 detector (64^2 scan unless --scan is given)")
    args = ap.parse_args()
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank)
        barrier(world)
        return

    import torch
    if world > 1 and os.environ.get("CUBO_BENCH_BACKEND") == "gloo":
        local %= max(1, torch.cuda.device_count())  # ranks sharing the GPUs there are
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
    if args.workload == "large_detector":
        run_large_detector(args, world, rank, local)
        return

    if world > 1:
        run_sharded(args, world, rank, local)
        barrier(world)
        import torch.distributed as dist
        dist.destroy_process_group()
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
        # per-kernel device time over separate iterations (events around every launch)
        plan.set_timing(True)
        plan.enqueue(max(3, min(args.steps, 10)))
        stats = plan.kernel_stats()
        plan.set_timing(False)
        plan.close()
        results[form] = dict(ms=ms, launches=launches, errors=errors, stats=stats, clocks=clocks.summary())

    head = forms[0]
    r = results[head]
    ms = r["ms"]
    stats = r["stats"]
    value = P * args.steps / (ms * 1e-3) * world
    peaks = measured_peaks()
    fma = fma_peaks(ctx)
    roofline = position_pass_roofline(head, stats, P, n, objects, ms / args.steps, peaks, fma)
    total_stat_ms = sum(v[0] for v in stats.values())

    fft_flops = P * (10 * n * math.log2(n) + 40 * n)
    forms_out = {}
    for form, fr in results.items():
        pass_form_ms = fr["stats"]["position_pass"][0] / max(fr["stats"]["position_pass"][1], 1)
        forms_out[form] = {"value": P * args.steps / (fr["ms"] * 1e-3) * world, "ms_per_step": fr["ms"] / args.steps,
                           "position_pass_ms": pass_form_ms, "error_last": float(fr["errors"][-1]),
                           "fft_equivalent_tflops": fft_flops / (pass_form_ms * 1e-3) / 1e12}
        if form in ("fp32", "fp32_generic"):
            forms_out[form]["frac_of_fp32_fma_peak"] = forms_out[form]["fft_equivalent_tflops"] / fma["fp32_tflops"]
        if form == "fp64":
            forms_out[form]["frac_of_fp64_fma_peak"] = forms_out[form]["fft_equivalent_tflops"] / fma["fp64_tflops"]
    comparison = None
    if "split_bf16" in results and "fp32" in results:
        ratio = forms_out["split_bf16"]["value"] / forms_out["fp32"]["value"]
        comparison = {"ratio_split_bf16_over_fp32": ratio, "target_ratio": 3.0, "target_met": ratio >= 3.0}
        for other in ("fp32_generic", "fp64"):
            if other in results:
                comparison[f"ratio_split_bf16_over_{other}"] = (forms_out["split_bf16"]["value"] /
                                                                forms_out[other]["value"])

    # accuracy of the measured forms against the FP64 device form, after every iteration, on this data
    parity = None
    if rank == 0 and not args.no_parity and {"split_bf16", "fp32"} <= set(results):
        parity = {"precision_workload": curve_summary(
            error_curves(ds, ctx, args.parity_iterations, ("split_bf16", "fp32")),
            {"split_bf16": 1e-4, "fp32": 1e-5}, f"{args.scan}^2 scan, 128^2 detector, {args.parity_iterations} "
                                                f"iterations from the same start, each form against the FP64 form")}

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
        cpu = cpu_rates(ds.amplitudes.reshape(P, -1), ds.positions, ds.object_start, ds.probe)
    del ds

    extras = {}
    if rank == 0 and not args.no_parity:
        extras["fp32_workload"] = fp32_workload_parity(ctx, local)
        extras["cpu_workload"] = cpu_workload(ctx, local, with_cpu=not args.no_cpu)
    if rank == 0 and not args.no_batched:
        extras["batched"] = measure_batched(BATCH_STEPS, 3, 1, local)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16x3/f32" if head == "split_bf16" else "f32", "data": "synthetic",
            "config": {"workload": f"{args.scan}x{args.scan} scan, step {STEP} px, {DET}x{DET} detector, object "
                                   f"{int(math.isqrt(objects))}x{int(math.isqrt(objects))}, dose 1e5, GD step 0.5",
                       "form": head, "positions": P, "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                       "l2": f"inputs larger than L2 ({P * n * 4 / 1e9:.2f} GB amplitudes, "
                             f"{P * n * 8 / 1e9:.2f} GB residuals; L2 126 MB)"},
            "forms": forms_out, "comparison": comparison, "parity": parity, "roofline": roofline,
            "kernels": {k: {"ms_per_launch": v[0] / max(v[1], 1), "launches": v[1],
                            "share": v[0] / total_stat_ms if total_stat_ms else None} for k, v in stats.items() if v[1]},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": r["launches"], "clocks": r["clocks"],
            "errors_first_last": [float(r["errors"][0]), float(r["errors"][-1])], "extras": extras,
        }
        print(json.dumps(line), flush=True)
    barrier(world)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()

if __name__ == "__main__":
    main()
