"""The FP32 and split-BF16 forms against the FP64 C oracle after every iteration, at the headline workload's shape.

The benchmark's workload is a 256^2 raster (step 4 px) over a 1152^2 object with a 128^2 detector; this test keeps the
detector, the step, the dose and the synthetic recipe and shrinks the raster to 32^2 (1,024 positions, object 256^2)
so that the C restatement of CuboPtycho's Double path (Ptychography.swift:280-402) runs all 30 iterations in seconds.
The bounds are the ones stated for the two forms: relative L2 object error at most 1e-5 for FP32 and 1e-4 for
split-BF16 against the FP64 oracle, held after every iteration, not only the last.  The probe is held to the same
bounds.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ITERATIONS = 30
BOUNDS = {"fp32": 1e-5, "split_bf16": 1e-4}


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_fp32_and_split_bf16_track_the_fp64_oracle_every_iteration():
    import cubokit_b200 as cb
    from cubokit_b200 import synthetic
    from oracle import c_oracle

    ds = synthetic.dataset(32, 128, dose=1e5, step=4, device=0)
    P = len(ds.positions)
    amps = ds.amplitudes.reshape(P, -1).astype(np.float64)
    threads = c_oracle.host_cores()
    ctx = cb.context(0)
    plans = {}
    for form in BOUNDS:
        plans[form] = cb.Plan(ds.amplitudes, ds.positions, ds.object_start.shape, ds.probe.shape, ctx=ctx,
                              step_size=0.5, precision=form)
        plans[form].set_state(ds.object_start, ds.probe)
    obj, probe = ds.object_start, ds.probe
    worst = {form: 0.0 for form in BOUNDS}
    try:
        for it in range(ITERATIONS):
            obj, probe, err = c_oracle.reconstruct(amps, ds.positions, obj, probe, iterations=1, step_size=0.5,
                                                   threads=threads, shift_every_position=False)
            for form, plan in plans.items():
                plan.enqueue(1)
                o, p = plan.get_state()
                ro, rp = _rel(o, obj), _rel(p, probe)
                worst[form] = max(worst[form], ro)
                assert ro <= BOUNDS[form], (form, it, ro)
                assert rp <= BOUNDS[form], (form, it, rp)
        for form, plan in plans.items():
            got = plan.errors(ITERATIONS)[-1]
            assert abs(got - err[0]) <= 1e-5 * abs(err[0]), (form, got, err[0])
    finally:
        for plan in plans.values():
            plan.close()
    # the split products keep the tensor-core form well inside its bound; FP32 likewise
    assert worst["split_bf16"] < 1e-4 and worst["fp32"] < 1e-5, worst
