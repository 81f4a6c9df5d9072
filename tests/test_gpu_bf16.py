"""The split-BF16 tensor-core form (128 x 128 detector) against the FP64 oracle and the FP32 form.

Bound: relative L2 error of the reconstructed object against the FP64 oracle <= 1e-4 (the precision form's target), and
per-iteration errors within 1e-4 relative.
"""
import numpy as np
import pytest

from oracle import c_oracle
from tests import scenes

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("fractional", [False, True])
def test_split_bf16_against_fp64_oracle(fractional):
    import cubokit_b200 as cb
    if fractional:
        s = scenes.nonsquare_scene(128, 128, 300)
    else:
        s = scenes.raster_scene(scan=4, det=128, step=4, seed=13)
    ref = c_oracle.reconstruct(s["amplitudes"].astype(np.float32), s["positions"], s["object"], s["probe"],
                               iterations=3)
    r = cb.SingleslicePtychography.reconstruct(s["amplitudes"], s["positions"], s["object"], s["probe"], iterations=3,
                                               precision="split_bf16")
    assert rel_l2(r.object, ref[0]) <= 1e-4, rel_l2(r.object, ref[0])
    assert rel_l2(r.probe, ref[1]) <= 1e-4, rel_l2(r.probe, ref[1])
    assert np.all(np.abs(r.errors - ref[2]) <= 1e-4 * ref[2]), (r.errors, ref[2])


@pytest.mark.parametrize("shift,odd_width", [(-40, False), (0, True)])
def test_split_bf16_patches_across_the_object_edge(shift, odd_width):
    """Windows that wrap around the periodic object's edge, and an object of odd width, take the kernel's
    complex-by-complex exit-wave gather instead of its aligned row loads; both must match the FP64 oracle."""
    import cubokit_b200 as cb
    s = scenes.raster_scene(scan=4, det=128, step=4, seed=17)
    positions = s["positions"].copy()
    positions[:, 1] += shift
    obj = np.ascontiguousarray(s["object"][:, :-1]) if odd_width else s["object"]
    ref = c_oracle.reconstruct(s["amplitudes"].astype(np.float32), positions, obj, s["probe"], iterations=3)
    r = cb.SingleslicePtychography.reconstruct(s["amplitudes"], positions, obj, s["probe"], iterations=3,
                                               precision="split_bf16")
    assert rel_l2(r.object, ref[0]) <= 1e-4, rel_l2(r.object, ref[0])
    assert rel_l2(r.probe, ref[1]) <= 1e-4, rel_l2(r.probe, ref[1])
    assert np.all(np.abs(r.errors - ref[2]) <= 1e-4 * ref[2]), (r.errors, ref[2])


def test_split_bf16_is_deterministic_and_close_to_fp32():
    import cubokit_b200 as cb
    s = scenes.raster_scene(scan=4, det=128, step=4, seed=17)
    a = cb.SingleslicePtychography.reconstruct(s["amplitudes"], s["positions"], s["object"], s["probe"], iterations=2,
                                               precision="split_bf16")
    b = cb.SingleslicePtychography.reconstruct(s["amplitudes"], s["positions"], s["object"], s["probe"], iterations=2,
                                               precision="split_bf16")
    assert np.array_equal(a.object, b.object) and np.array_equal(a.probe, b.probe)
    f = cb.SingleslicePtychography.reconstruct(s["amplitudes"], s["positions"], s["object"], s["probe"], iterations=2)
    assert rel_l2(a.object, f.object) <= 1e-4


def test_split_bf16_refuses_other_detector_sizes():
    import cubokit_b200 as cb
    s = scenes.raster_scene(scan=3, det=64, step=4, seed=1)
    with pytest.raises(cb.UnsupportedError):
        cb.SingleslicePtychography.reconstruct(s["amplitudes"], s["positions"], s["object"], s["probe"], iterations=1,
                                               precision="split_bf16")


def test_split_bf16_adjoint_against_fp64():
    import cubokit_b200 as cb
    s = scenes.raster_scene(scan=4, det=128, step=4, seed=19)
    amps = (s["amplitudes"] * 1.05).astype(np.float32)
    out = {}
    for precision in ("split_bf16", "fp32"):
        plan = cb.Plan(amps, s["positions"], s["object"].shape, s["probe"].shape, precision=precision)
        plan.set_state(s["object"], s["probe"])
        out[precision] = plan.backward(recompute_exit_waves=True)
    (l1, go1, gp1), (l2, go2, gp2) = out["split_bf16"], out["fp32"]
    assert abs(l1 - l2) <= 1e-4 * l2
    assert np.max(np.abs(go1 - go2)) <= 1e-3 * np.max(np.abs(go2))
    assert np.max(np.abs(gp1 - gp2)) <= 1e-3 * np.max(np.abs(gp2))


def _bf16_run(s, iterations, band_positions, monkeypatch, precision="split_bf16"):
    import cubokit_b200 as cb
    monkeypatch.setenv("CUBO_PTYCHO_BAND_POSITIONS", str(band_positions))
    plan = cb.Plan(s["amplitudes"], s["positions"], s["object"].shape, s["probe"].shape, step_size=0.5,
                   precision=precision)
    try:
        plan.set_state(s["object"], s["probe"])
        errors = plan.iterate(iterations)
        o, p = plan.get_state()
    finally:
        plan.close()
    return o, p, errors


def test_banded_iteration_equals_one_band(monkeypatch):
    """With CUBO_PTYCHO_BAND_POSITIONS the iteration runs in bands of positions whose residuals stay in L2 (each band's
    pass, then its object and probe gathers).  The object gather continues every pixel's sum from memory in the same candidate order, so after one
    iteration the object equals the one-band run bit for bit; the probe partials are grouped per band, so the probe
    (and every later iteration) agrees to FP32 round-off.  Band sizes that do not divide the scan, and one position per
    band, included."""
    s = scenes.raster_scene(scan=9, det=128, step=4, seed=29)  # 81 positions
    o1, p1, e1 = _bf16_run(s, 1, 0, monkeypatch)
    for band in (1, 16, 37):
        ob, pb, eb = _bf16_run(s, 1, band, monkeypatch)
        assert np.array_equal(ob, o1), band
        assert rel_l2(pb, p1) <= 1e-6, (band, rel_l2(pb, p1))
        assert np.array_equal(eb, e1), band  # per-position error partials: the same kernel, the same sums
    o4, _, _ = _bf16_run(s, 4, 0, monkeypatch)
    ob4, _, _ = _bf16_run(s, 4, 16, monkeypatch)
    assert rel_l2(ob4, o4) <= 1e-6, rel_l2(ob4, o4)


def test_banded_fp32_iteration_equals_one_pass(monkeypatch):
    """The FP32 128 x 128 pass keeps one probe-gradient partial per CTA (148 of them) across the bands: with bands of
    whole multiples of 148 positions every CTA still sums its positions in the same order, so object, probe and errors
    equal one pass bit for bit, iteration after iteration (169 positions: a full band and a partial one)."""
    s = scenes.raster_scene(scan=13, det=128, step=4, seed=31)
    o1, p1, e1 = _bf16_run(s, 3, 0, monkeypatch, precision="fp32")
    ob, pb, eb = _bf16_run(s, 3, 148, monkeypatch, precision="fp32")
    assert np.array_equal(ob, o1) and np.array_equal(pb, p1) and np.array_equal(eb, e1)
