"""The CUDA path (through the C ABI) against the FP64 oracle and CuboKit's py4DSTEM pins.

Bounds:
  * FP64 form vs the pins: the reference Double engine's own bound, ``max|a - b| / max(1, max|b|) < 2e-6``
    (``PtychographyTests.swift:28-31,60``).
  * FP32 form vs the FP64 oracle: the reference's Float-vs-Double bounds (``SinglePrecisionTests.swift:5-8,64-69``):
    object 1e-4 and probe 1e-5 absolute, errors 1e-5 relative (1e-4 for the fractional non-square scenes,
    ``SinglePrecisionTests.swift:204-208``).
"""
import numpy as np
import pytest

from oracle import c_oracle
from tests import golden_cases as gc
from tests import scenes

pytestmark = pytest.mark.gpu

ENGINE_CASES = gc.engine_cases()
PROBE_CASES = gc.probe_cases()


@pytest.fixture(scope="module")
def cb():
    import cubokit_b200
    return cubokit_b200


def _gpu(cb, case, precision, **extra):
    kw = dict(case.kwargs)
    kw.update(extra)
    if kw.get("error_normalization") == "meanIntensity":
        kw["error_normalization"] = ("meanIntensity", kw.pop("mean_intensity"))
    else:
        kw.pop("mean_intensity", None)
    return cb.SingleslicePtychography.reconstruct(case.amplitudes, case.positions, case.object, case.probe,
                                                  precision=precision, **kw)


def _oracle(case, **extra):
    kw = dict(case.kwargs)
    kw.update(extra)
    return c_oracle.reconstruct(case.amplitudes.astype(np.float32).astype(np.float64), case.positions, case.object,
                                case.probe, **kw)


@pytest.mark.parametrize("case", ENGINE_CASES, ids=[c.name for c in ENGINE_CASES])
def test_fp64_form_meets_the_pins(cb, case):
    r = _gpu(cb, case, "fp64")
    g = case.result_gap(r.object, r.probe, r.errors)
    assert g < 2e-6, (case.name, case.source, g)


@pytest.mark.parametrize("case", ENGINE_CASES, ids=[c.name for c in ENGINE_CASES])
def test_fp32_form_against_fp64_oracle(cb, case):
    r = _gpu(cb, case, "fp32")
    o, p, e = _oracle(case)
    assert np.max(np.abs(r.object - o)) <= 1e-4, case.name
    assert np.max(np.abs(r.probe - p)) <= 1e-5 * max(1.0, np.max(np.abs(p))), case.name
    assert np.all(np.abs(r.errors - e) <= 1e-5 * np.abs(e)), (case.name, r.errors, e)


@pytest.mark.parametrize("name,kw,expect", PROBE_CASES, ids=[c[0] for c in PROBE_CASES])
def test_probe_build_on_device_meets_the_pins(cb, name, kw, expect):
    kw = dict(kw)
    terms = kw.pop("terms", None)
    got = cb.PtychographyProbe.build(**kw, higher_order=() if terms is None else terms)
    bound = 1e-8 if name.startswith("options.app.") else 2e-6
    assert gc.complex_gap(got, expect) < bound, name


def test_gaussian_scene_fp32_against_fp64(cb):
    """``SinglePrecisionTests.swift:58-72`` with the GPU FP32 form in place of the Float engine."""
    s = scenes.gaussian_scene()
    ref = c_oracle.reconstruct(s["amplitudes"].astype(np.float32), s["positions"], s["object"], s["probe"], iterations=3)
    r = cb.SingleslicePtychography.reconstruct(s["amplitudes"], s["positions"], s["object"], s["probe"], iterations=3)
    assert np.max(np.abs(ref[0].real - r.object.real)) <= 1e-4 and np.max(np.abs(ref[0].imag - r.object.imag)) <= 1e-4
    assert np.max(np.abs(ref[1].real - r.probe.real)) <= 1e-5 and np.max(np.abs(ref[1].imag - r.probe.imag)) <= 1e-5
    assert np.all(np.abs(ref[2] - r.errors) <= 1e-5 * np.abs(ref[2]))
    assert r.errors[2] < r.errors[0]
    assert len(r.positions) == len(s["positions"])


@pytest.mark.parametrize("shape", [(32, 48), (22, 21), (14, 14), (13, 26), (165, 40), (32, 21)])
def test_fractional_nonsquare_scenes_fp32_against_fp64(cb, shape):
    """``SinglePrecisionTests.swift:148-210``: every detector size the reference pins, fractional positions."""
    size = 96 if shape == (32, 48) else 2 * max(shape) + 40
    s = scenes.nonsquare_scene(shape[0], shape[1], size)
    ref = c_oracle.reconstruct(s["amplitudes"].astype(np.float32), s["positions"], s["object"], s["probe"], iterations=3)
    r = cb.SingleslicePtychography.reconstruct(s["amplitudes"], s["positions"], s["object"], s["probe"], iterations=3)
    assert np.max(np.abs(ref[0] - r.object)) <= 1e-4
    assert np.max(np.abs(ref[1] - r.probe)) <= 1e-5
    assert np.all(np.abs(ref[2] - r.errors) <= 1e-4 * np.abs(ref[2]))
    assert r.errors[2] < r.errors[0]


def test_options_in_fp32(cb):
    """``SinglePrecisionTests.swift:74-87``: pure phase + centre of mass + amplitude constraint."""
    s = scenes.gaussian_scene()
    kw = dict(iterations=2, pure_phase_object=True, fix_probe_center_of_mass=True, constrain_probe_amplitude=True)
    a = c_oracle.reconstruct(s["amplitudes"], s["positions"], s["object"], s["probe"], **kw)
    b = cb.SingleslicePtychography.reconstruct(s["amplitudes"], s["positions"], s["object"], s["probe"], **kw)
    assert np.max(np.abs(a[0].real - b.object.real)) <= 1e-4
    assert np.max(np.abs(a[1].imag - b.probe.imag)) <= 1e-4
    assert np.all(np.abs(np.abs(b.object) - 1) < 1e-5)


@pytest.mark.parametrize("det", [64, 96])
def test_raster_scene_64_and_96_fp32_and_fp64(cb, det):
    """64 x 64 and 96 x 96 detectors take the shared-memory pass with a compile-time radix plan (8 * 8, 8 * 4 * 3)."""
    s = scenes.raster_scene(scan=6, det=det, step=4, seed=7)
    ref = c_oracle.reconstruct(s["amplitudes"], s["positions"], s["object"], s["probe"], iterations=4)
    for precision, obj_tol in (("fp32", 1e-4), ("fp64", 1e-10)):
        r = cb.SingleslicePtychography.reconstruct(s["amplitudes"], s["positions"], s["object"], s["probe"],
                                                   iterations=4, precision=precision)
        assert np.max(np.abs(ref[0] - r.object)) <= obj_tol, precision
        assert np.all(np.abs(ref[2] - r.errors) <= (1e-5 if precision == "fp32" else 1e-12) * ref[2]), precision


def test_deterministic_and_resumable(cb):
    """Two runs are bitwise identical; 2 + 3 iterations on a plan equal 5 in one call, bitwise."""
    case = ENGINE_CASES[0]
    a = _gpu(cb, case, "fp32")
    b = _gpu(cb, case, "fp32")
    assert np.array_equal(a.object, b.object) and np.array_equal(a.probe, b.probe) and np.array_equal(a.errors, b.errors)
    kw = dict(case.kwargs)
    kw["error_normalization"] = ("meanIntensity", kw.pop("mean_intensity"))
    kw.pop("iterations")
    plan = cb.Plan(case.amplitudes, case.positions, case.object.shape, case.probe.shape, **kw)
    plan.set_state(case.object, case.probe)
    e1 = plan.iterate(2)
    e2 = plan.iterate(3)
    o, p = plan.get_state()
    plan.close()
    full = _gpu(cb, case, "fp32", iterations=5)
    assert np.array_equal(o, full.object) and np.array_equal(p, full.probe)
    assert np.array_equal(np.concatenate([e1, e2]), full.errors)


def test_refusals_through_the_c_abi(cb):
    """``PtychographyTests.swift:73-85,172-180``; ``SinglePrecisionTests.swift:102-116``."""
    case = ENGINE_CASES[0]
    with pytest.raises(cb.PtychographyError):
        cb.SingleslicePtychography.reconstruct([], [], case.probe, case.probe)
    for radius, width in [(-0.1, 0.05), (0.51, 0.05), (np.nan, 0.05), (0.5, 0.0), (0.5, 0.51), (0.5, np.inf)]:
        with pytest.raises(cb.PtychographyError):
            _gpu(cb, case, "fp32", iterations=1, constrain_probe_amplitude=True, probe_amplitude_relative_radius=radius,
                 probe_amplitude_relative_width=width)
    for precision in ("fp32", "split_bf16"):  # the reference's Float path refuses position correction
        with pytest.raises((cb.PtychographyError, cb.UnsupportedError)):
            _gpu(cb, case, precision, iterations=1, position_correction=cb.PtychographyPositionCorrection())
    for value in (-1.0, np.nan, np.inf):  # checked on the device after the upload
        bad = case.amplitudes.copy()
        bad.flat[5] = value
        with pytest.raises(cb.PtychographyError):
            cb.SingleslicePtychography.reconstruct(bad, case.positions, case.object, case.probe, iterations=1)
    with pytest.raises(cb.PtychographyError):  # no supplied energy to normalise the errors by
        cb.SingleslicePtychography.reconstruct(np.zeros_like(case.amplitudes), case.positions, case.object, case.probe,
                                               iterations=1)
    with pytest.raises(cb.PtychographyError):
        cb.SingleslicePtychography.reconstruct(case.amplitudes, case.positions, case.object, case.probe, iterations=1,
                                               step_size=0.0)
    wide = np.full((16, 96), 0.1 + 0j)
    with pytest.raises(cb.PtychographyError):
        cb.SingleslicePtychography.reconstruct(np.ones(16 * 96), [[4, 4]], np.ones((80, 80), complex), wide, iterations=1)
    with pytest.raises(cb.PtychographyError):
        cb.PtychographyProbe.build(2, 2, 0, 1, 0.02, 0.01)
    small = np.full((14, 14), 0.1 + 0j)  # a Bluestein-length detector runs (SinglePrecisionTests.swift:106-110)
    r = cb.SingleslicePtychography.reconstruct(np.ones(196), [[4, 4]], np.ones((80, 80), complex), small, iterations=1)
    assert len(r.errors) == 1 and np.isfinite(r.errors[0])


def test_progress_and_cancellation(cb):
    """``SinglePrecisionTests.swift:89-101``."""
    s = scenes.gaussian_scene()
    seen = []
    cb.SingleslicePtychography.reconstruct(s["amplitudes"], s["positions"], s["object"], s["probe"], iterations=2,
                                           progress=lambda done, total: seen.append((done, total)))
    assert seen == [(1, 2), (2, 2)]
    polls = [0]

    def cancelled():
        polls[0] += 1
        return polls[0] > 2

    with pytest.raises(cb.CancellationError):
        cb.SingleslicePtychography.reconstruct(s["amplitudes"], s["positions"], s["object"], s["probe"], iterations=5,
                                               is_cancelled=cancelled)


def test_fixed_probe_is_returned_unchanged(cb):
    """``PtychographyTests.swift:128-132``: with the probe fixed no probe constraint applies."""
    case = [c for c in ENGINE_CASES if c.name == "ptycho.constraint.com"][0]
    r = _gpu(cb, case, "fp32", fix_probe=True, fix_probe_center_of_mass=True, constrain_probe_amplitude=True,
             probe_amplitude_relative_radius=0.3, probe_amplitude_relative_width=0.1)
    assert np.array_equal(r.probe, case.probe)


@pytest.mark.parametrize("fractional", [False, True])
def test_fast128_against_generic_and_oracle(cb, fractional):
    """The 128 x 128 register-resident kernel against the any-size kernel and the FP64 oracle."""
    if fractional:
        s = scenes.nonsquare_scene(128, 128, 300)
    else:
        s = scenes.raster_scene(scan=3, det=128, step=4, seed=9)
    ref = c_oracle.reconstruct(s["amplitudes"].astype(np.float32), s["positions"], s["object"], s["probe"],
                               iterations=3)
    fast = cb.SingleslicePtychography.reconstruct(s["amplitudes"], s["positions"], s["object"], s["probe"],
                                                  iterations=3)
    gen = cb.SingleslicePtychography.reconstruct(s["amplitudes"], s["positions"], s["object"], s["probe"],
                                                 iterations=3, variant="generic")
    for r in (fast, gen):
        assert np.max(np.abs(r.object - ref[0])) <= 1e-4
        assert np.max(np.abs(r.probe - ref[1])) <= 1e-5 * max(1.0, np.max(np.abs(ref[1])))
        assert np.all(np.abs(r.errors - ref[2]) <= 1e-5 * ref[2])
    assert np.max(np.abs(fast.object - gen.object)) <= 2e-5


def test_measured_fma_peaks_are_plausible():
    """``cubo_ptycho_measure_peaks``: the FP32 and FP64 FMA rates the compute fractions divide by, within what a B200
    can do (FP32 at most ~90 TFLOP/s, FP64 at most ~45) and well above a broken measurement."""
    import cubokit_b200 as cb
    f32, f64 = cb.context(0).measure_peaks()
    assert 20.0 < f32 < 120.0
    assert 5.0 < f64 < 60.0
