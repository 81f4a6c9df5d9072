"""Amplitude preprocessing on the device (``cubo_ptycho_prepare_amplitudes``) against the reference's pins and the
NumPy restatement of ``PtychographyPreparation.amplitudes(from:origins:shift:)``.

Bounds: the reference's own, 2e-6 of max(1, max|a|) for amplitudes and 2e-6 relative for the mean intensities
(``PreparationTests.swift:39-53``, ``PtychographyTests.swift:184-193``).  The device computes in FP64 and returns
Float32 amplitudes (the engine's input), so against the FP64 oracle the difference is the Float32 rounding.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle import numpy_oracle as no

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"


def gap(a, b):
    a, b = np.asarray(a, np.float64).ravel(), np.asarray(b, np.float64).ravel()
    return float(np.max(np.abs(a - b)) / max(1.0, np.max(np.abs(b))))


def _pre():
    d = np.load(GOLDEN / "preprocess.npz")
    count = int(d["scanRows"]) * int(d["scanColumns"])
    return d, d["cube"].reshape(count, int(d["detectorRows"]), int(d["detectorColumns"]))


@pytest.mark.parametrize("order,shift", [("1", "bilinear"), ("3", "cubicSpline")])
def test_preprocessing_pins(order, shift):
    import cubokit_b200 as cb
    d, cube = _pre()
    a = cb.PtychographyPreparation.amplitudes(cube, (d["originRows"], d["originColumns"]), shift=shift)
    assert a.values.dtype == np.float32 and a.values.shape == cube.shape
    assert gap(a.values, d[f"order{order}_amplitudes"]) < 2e-6
    assert abs(a.mean_intensity / float(d[f"order{order}_meanIntensity"]) - 1) < 2e-6
    assert abs(a.clipped_mean_intensity / float(d[f"order{order}_clippedMeanIntensity"]) - 1) < 2e-6
    assert a.error_normalization == ("meanIntensity", a.mean_intensity)


def test_preprocessing_feeds_the_engine_pin():
    """The raw 64-pattern cube through device preprocessing (uniform origin, bilinear) meets the engine's amplitude pin;
    reconstructing from the device-resident result with the mean-intensity normalisation equals reconstructing from
    the same amplitudes on the host, bit for bit."""
    import cubokit_b200 as cb
    p = np.load(GOLDEN / "ptycho.npz")
    rows, columns = int(p["rows"]), int(p["columns"])
    raw = p["preprocessing_raw"].reshape(-1, rows, columns)
    o = p["preprocessing_origin"]
    a = cb.PtychographyPreparation.amplitudes(raw, (o[0], o[1]), shift="bilinear")
    assert gap(a.values, p["amplitudes"]) < 2e-6
    assert abs(a.mean_intensity / float(p["meanIntensity"]) - 1) < 2e-6
    d = cb.PtychographyPreparation.amplitudes(raw, (o[0], o[1]), shift="bilinear", keep_on_device=True)
    assert np.array_equal(d.values.cpu().numpy(), a.values) and d.mean_intensity == a.mean_intensity
    obj = p["initialObject_re"] + 1j * p["initialObject_im"]
    probe = p["initialProbe_re"] + 1j * p["initialProbe_im"]
    obj = obj.reshape(int(p["objectRows"]), int(p["objectColumns"]))
    probe = probe.reshape(rows, columns)
    kw = dict(iterations=3, step_size=0.35, normalization_minimum=0.7, error_normalization=a.error_normalization)
    host = cb.SingleslicePtychography.reconstruct(a.values, p["positions"], obj, probe, **kw)
    dev = cb.SingleslicePtychography.reconstruct(d.values, p["positions"], obj, probe, **kw)
    assert np.array_equal(host.object, dev.object) and np.array_equal(host.errors, dev.errors)


@pytest.mark.parametrize("shift", ["bilinear", "cubicSpline"])
@pytest.mark.parametrize("shape", [(32, 48), (21, 17), (128, 128)])
def test_against_the_oracle_on_random_cubes(shift, shape):
    """Per-position fractional origins (including negative and beyond one period), non-square and odd detectors,
    negative raw values (clipped) — against the FP64 NumPy restatement."""
    import cubokit_b200 as cb
    rng = np.random.default_rng(sum(shape) + len(shift))
    count = 12
    cube = (rng.standard_normal((count,) + shape) + 0.3).astype(np.float32)
    o_rows = rng.uniform(-2.5 * shape[0], 2.5 * shape[0], count)
    o_cols = rng.uniform(-2.5 * shape[1], 2.5 * shape[1], count)
    ref = no.prepare_amplitudes(cube, o_rows, o_cols, shift)
    a = cb.PtychographyPreparation.amplitudes(cube, (o_rows, o_cols), shift=shift)
    assert gap(a.values, ref.values) < 2e-6
    assert abs(a.mean_intensity - ref.mean_intensity) <= 1e-10 * max(1.0, abs(ref.mean_intensity))
    assert abs(a.clipped_mean_intensity - ref.clipped_mean_intensity) <= 1e-10 * ref.clipped_mean_intensity


def test_zero_origin_and_integer_roll_are_exact():
    """``PreparationTests.swift:63-81``: a zero origin reproduces sqrt(max(data, 0)) (bilinear: bit for bit after the
    Float32 rounding; spline: to roundoff of the exact prefilter), and an integer origin is a roll."""
    import cubokit_b200 as cb
    d, cube = _pre()
    count = len(cube)
    data = cube.astype(np.float32)
    expect = np.sqrt(np.maximum(data.astype(np.float64), 0)).astype(np.float32)
    a = cb.PtychographyPreparation.amplitudes(data, (0.0, 0.0), shift="bilinear")
    assert np.array_equal(a.values, expect)
    s = cb.PtychographyPreparation.amplitudes(data, (0.0, 0.0), shift="cubicSpline")
    assert gap(s.values.astype(np.float64) ** 2, np.maximum(data.astype(np.float64), 0)) < 1e-6
    r = cb.PtychographyPreparation.amplitudes(data, (2.0, -3.0), shift="bilinear")
    rolled = np.roll(np.roll(data.astype(np.float64), -2, axis=1), 3, axis=2)
    assert np.array_equal(r.values, np.sqrt(np.maximum(rolled, 0)).astype(np.float32))
    assert r.position_count == count


def test_host_chunks_and_device_path_agree_bit_for_bit():
    """5000 patterns of 128 x 128 (the host path moves them in two chunks of at most 256 MB) against one device-resident
    call: the same amplitudes and the same mean intensities, bit for bit."""
    import cubokit_b200 as cb
    import torch
    rng = np.random.default_rng(3)
    count = 5000
    cube = rng.gamma(2.0, 1.0, (count, 128, 128)).astype(np.float32)
    o_rows, o_cols = rng.uniform(-3, 3, count), rng.uniform(-3, 3, count)
    a = cb.PtychographyPreparation.amplitudes(cube, (o_rows, o_cols), shift="cubicSpline")
    d = cb.PtychographyPreparation.amplitudes(torch.from_numpy(cube).cuda(), (o_rows, o_cols), shift="cubicSpline",
                                              keep_on_device=True)
    assert np.array_equal(a.values, d.values.cpu().numpy())
    assert a.mean_intensity == d.mean_intensity and a.clipped_mean_intensity == d.clipped_mean_intensity


def test_preprocessing_refusals():
    import cubokit_b200 as cb
    d, cube = _pre()
    count = len(cube)
    z = np.zeros(count)
    bad = cube.astype(np.float32).copy()
    bad[3, 2, 1] = np.nan
    cases = [(bad, (0.0, 0.0), "bilinear"), (cube, (np.nan, 0.0), "bilinear"), (cube, (0.0, 2e9), "cubicSpline"),
             (cube, (z[:-1], z), "bilinear"), (cube[:, :1, :], (0.0, 0.0), "bilinear"), (cube, (0.0, 0.0), "nearest")]
    for c, o, shift in cases:
        with pytest.raises(cb.PtychographyError):
            cb.PtychographyPreparation.amplitudes(c, o, shift=shift)


@pytest.mark.parametrize("shift", ["bilinear", "cubicSpline"])
def test_every_staging_form_against_the_oracle(shift):
    """The kernel's three ways to reach a pattern: staged in shared memory with 16-byte row taps (columns a multiple
    of 4, aligned output), staged with single taps (odd columns, or an output 4 bytes off alignment), and read straight
    from global memory (an input 4 bytes off alignment) — each against the FP64 restatement.  Also `out=`: the result
    lands in the caller's tensor."""
    import cubokit_b200 as cb
    import torch
    rng = np.random.default_rng(11 + len(shift))
    for shape in [(20, 17), (24, 32)]:
        count = 9
        n = shape[0] * shape[1]
        cube = (rng.standard_normal((count,) + shape) + 0.5).astype(np.float32)
        o_rows, o_cols = rng.uniform(-40, 40, count), rng.uniform(-40, 40, count)
        ref = no.prepare_amplitudes(cube, o_rows, o_cols, shift)
        flat = torch.from_numpy(cube).cuda().reshape(-1)
        shifted_in = torch.empty(count * n + 1, device="cuda")
        shifted_in[1:] = flat
        shifted_out = torch.empty(count * n + 1, device="cuda")
        for src, out in [(flat, None), (flat, shifted_out[1:]), (shifted_in[1:], None)]:
            a = cb.PtychographyPreparation.amplitudes(src.view((count,) + shape), (o_rows, o_cols), shift=shift, out=out)
            if out is not None:
                assert a.values.data_ptr() == out.data_ptr()
            got = a.values.cpu().numpy() if hasattr(a.values, "cpu") else a.values
            assert gap(got.reshape(cube.shape), ref.values) < 2e-6
            assert abs(a.mean_intensity - ref.mean_intensity) <= 1e-10 * max(1.0, abs(ref.mean_intensity))
            assert abs(a.clipped_mean_intensity - ref.clipped_mean_intensity) <= 1e-10 * ref.clipped_mean_intensity
    with pytest.raises(cb.PtychographyError):
        cb.PtychographyPreparation.amplitudes(cube, (0.0, 0.0), shift=shift, out=torch.empty(5, device="cuda"))
