"""The oracles (C and NumPy FP64 restatements of CuboPtycho's Double path) against CuboKit's own py4DSTEM pins.

Bound and metric are the reference's: ``max|a - b| / max(1, max|b|) < 2e-6`` (``PtychographyTests.swift:28-31,60``).
"""
from pathlib import Path

import numpy as np
import pytest

from oracle import c_oracle, numpy_oracle
from tests import golden_cases as gc
from tests import scenes

ENGINE_CASES = gc.engine_cases()
PROBE_CASES = gc.probe_cases()


def _numpy_call(case):
    kw = dict(case.kwargs)
    return numpy_oracle.reconstruct(case.amplitudes, case.positions, case.object, case.probe, **kw)


def _c_call(case, **extra):
    kw = dict(case.kwargs)
    kw.update(extra)
    return c_oracle.reconstruct(case.amplitudes, case.positions, case.object, case.probe, **kw)


@pytest.mark.parametrize("case", ENGINE_CASES, ids=[c.name for c in ENGINE_CASES])
def test_c_oracle_against_pins(case):
    o, p, e = _c_call(case)
    g = case.result_gap(o, p, e)
    assert g < 2e-6, (case.name, case.source, g)


@pytest.mark.parametrize("case", ENGINE_CASES, ids=[c.name for c in ENGINE_CASES])
def test_numpy_oracle_against_pins(case):
    o, p, e = _numpy_call(case)
    g = case.result_gap(o, p, e)
    assert g < 2e-6, (case.name, case.source, g)


def test_c_and_numpy_oracles_agree_to_roundoff():
    for case in ENGINE_CASES[:4]:
        a = _c_call(case)
        b = _numpy_call(case)
        for x, y in zip(a, b):
            assert gc.complex_gap(x, y) < 1e-11, case.name


def test_uncapped_object_really_exceeds_one():
    """``OptionsTests.swift:71-78``: the pinned uncapped runs leave |object| > 1, and the cap changes the result."""
    for case in [c for c in ENGINE_CASES if c.name.startswith("options.") and not c.kwargs["pure_phase_object"]]:
        o, _, _ = _c_call(case)
        amp = np.abs(o).max()
        assert amp > 1.002 and abs(amp - case.extra["maxAmplitude"]) < 1e-5
        capped, _, _ = _c_call(case, constrain_object_amplitude=True)
        assert np.abs(capped).max() <= 1 + 1e-12
        assert gc.gap(capped.real, o.real) > 1e-3


@pytest.mark.parametrize("name,kw,expect", PROBE_CASES, ids=[c[0] for c in PROBE_CASES])
def test_probe_build_against_pins(name, kw, expect):
    kw = dict(kw)
    terms = kw.pop("terms", None)
    got = c_oracle.probe_build(**kw, terms=terms)
    bound = 1e-8 if name.startswith("options.app.") else 2e-6  # OptionsTests.swift:143 vs :107
    assert gc.complex_gap(got, expect) < bound, name
    ho = [] if terms is None else [numpy_oracle.AberrationTerm(int(t[0]), int(t[1]), bool(t[2]), float(t[3])) for t in terms]
    got_np = numpy_oracle.probe_build(kw["rows"], kw["columns"], kw["row_sampling"], kw["column_sampling"],
                                      kw["wavelength"], kw["cutoff"], kw.get("rolloff", 0.002), kw.get("defocus", 0.0),
                                      kw.get("astigmatism", 0.0), kw.get("astigmatism_angle", 0.0),
                                      kw.get("spherical_aberration", 0.0), ho)
    assert gc.complex_gap(got_np, expect) < bound, name


def test_initial_probe_energy_scaling():
    """``OptionsTests.swift:115-123``: ``PtychographyPreparation.initialProbe`` (probe build + energy scaling)."""
    o = gc.load("options")
    g = lambda k: o["initial_" + k]
    terms = []
    for n, m, mag, az in g("terms"):
        terms += numpy_oracle.AberrationTerm.polar(int(n), int(m), float(mag), float(az))
    p = numpy_oracle.initial_probe(int(g("rows")), int(g("columns")), float(g("samplingRow")),
                                   float(g("samplingColumn")), float(g("wavelength")), float(g("semiangle")),
                                   float(g("rolloff")), float(g("defocus")), float(g("astigmatism")),
                                   float(g("astigmatismAngle")), float(g("sphericalAberration")), terms,
                                   float(g("meanIntensity")))
    expect = (o["initial_probe_re"] + 1j * o["initial_probe_im"]).reshape(p.shape)
    assert gc.complex_gap(p, expect) < 2e-6


def test_invalid_inputs_are_refused():
    """``PtychographyTests.swift:73-85,172-180``, ``SinglePrecisionTests.swift:111-116``."""
    case = ENGINE_CASES[0]
    with pytest.raises(ValueError):
        c_oracle.reconstruct(np.zeros(0), np.zeros((0, 2)), case.object, case.probe)
    for radius, width in [(-0.1, 0.05), (0.51, 0.05), (np.nan, 0.05), (0.5, 0.0), (0.5, 0.51), (0.5, np.inf)]:
        with pytest.raises(ValueError):
            _c_call(case, iterations=1, constrain_probe_amplitude=True, probe_amplitude_relative_radius=radius,
                    probe_amplitude_relative_width=width)
    with pytest.raises(ValueError):
        c_oracle.probe_build(2, 2, 0, 1, 0.02, 0.01)
    wide = np.full((16, 96), 0.1 + 0j)
    with pytest.raises(ValueError):
        c_oracle.reconstruct(np.ones(16 * 96), [[4, 4]], np.ones((80, 80), complex), wide, iterations=1)


def test_threaded_oracle_is_deterministic_and_agrees():
    case = ENGINE_CASES[0]
    a = _c_call(case, threads=3)
    b = _c_call(case, threads=3)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    c = _c_call(case)
    for x, y in zip(a, c):
        assert gc.complex_gap(x, y) < 1e-12


def test_float_path_agrees_with_double_on_the_gaussian_scene():
    """``SinglePrecisionTests.swift:58-72``: object 1e-4, probe 1e-5 absolute, errors 1e-5 relative, convergence."""
    s = scenes.gaussian_scene()
    ref = c_oracle.reconstruct(s["amplitudes"], s["positions"], s["object"], s["probe"], iterations=3)
    sgl = c_oracle.reconstruct(s["amplitudes"], s["positions"], s["object"], s["probe"], iterations=3, single=True)
    assert np.max(np.abs(ref[0].real - sgl[0].real)) <= 1e-4 and np.max(np.abs(ref[0].imag - sgl[0].imag)) <= 1e-4
    assert np.max(np.abs(ref[1].real - sgl[1].real)) <= 1e-5 and np.max(np.abs(ref[1].imag - sgl[1].imag)) <= 1e-5
    assert np.all(np.abs(ref[2] - sgl[2]) <= 1e-5 * np.abs(ref[2]))
    assert sgl[2][2] < sgl[2][0]


@pytest.mark.parametrize("shape", [(32, 48), (22, 21), (13, 26)])
def test_float_path_agrees_with_double_on_fractional_nonsquare_scenes(shape):
    """``SinglePrecisionTests.swift:148-210`` (a subset of its sizes)."""
    s = scenes.nonsquare_scene(shape[0], shape[1], 96 if shape == (32, 48) else 2 * max(shape) + 40)
    ref = c_oracle.reconstruct(s["amplitudes"], s["positions"], s["object"], s["probe"], iterations=3)
    sgl = c_oracle.reconstruct(s["amplitudes"], s["positions"], s["object"], s["probe"], iterations=3, single=True)
    assert np.max(np.abs(ref[0] - sgl[0])) <= 1.5e-4
    assert np.max(np.abs(ref[1] - sgl[1])) <= 1.5e-5
    assert np.all(np.abs(ref[2] - sgl[2]) <= 1e-4 * np.abs(ref[2]))
    assert ref[2][2] < ref[2][0]


def test_adjoint_matches_central_differences_in_fp64():
    """The loss gradient ``-2 n sum conj(S) dpsi`` (object) and ``-2 n sum conj(O) dpsi`` (probe) of the reference's
    accumulations, against central differences, integer positions."""
    s = scenes.raster_scene(scan=4, det=16, step=4, seed=3)
    amps = s["amplitudes"] * 1.05  # off the solution, so the gradient is not ~0
    loss, go, gp = numpy_oracle.loss_and_gradients(amps, s["positions"], s["object"], s["probe"])
    rng = np.random.default_rng(5)
    h = 1e-6
    for _ in range(8):
        j = tuple(rng.integers(0, n) for n in s["object"].shape)
        for unit, part in ((1.0, "re"), (1j, "im")):
            o1 = s["object"].copy(); o1[j] += unit * h
            o2 = s["object"].copy(); o2[j] -= unit * h
            fd = (numpy_oracle.loss_and_gradients(amps, s["positions"], o1, s["probe"])[0] -
                  numpy_oracle.loss_and_gradients(amps, s["positions"], o2, s["probe"])[0]) / (2 * h)
            an = go[j].real if part == "re" else go[j].imag
            assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)) + 1e-5 * abs(loss) * h, (j, part, fd, an)


# ---------------------------------------------------------------------------------------------------- preprocessing

PRE = np.load(Path(__file__).resolve().parent / "golden" / "preprocess.npz")
PTYCHO = np.load(Path(__file__).resolve().parent / "golden" / "ptycho.npz")
no = numpy_oracle
gap = gc.gap


def _pre_cube():
    rows, columns = int(PRE["detectorRows"]), int(PRE["detectorColumns"])
    count = int(PRE["scanRows"]) * int(PRE["scanColumns"])
    return PRE["cube"].reshape(count, rows, columns)


@pytest.mark.parametrize("order,shift", [("1", "bilinear"), ("3", "cubicSpline")])
def test_prepared_amplitudes_meet_the_preprocessing_pins(order, shift):
    """``PreparationTests.swift:39-53``: both interpolation orders, per-position origins, at the reference's bounds
    (2e-6 of max(1, max|a|); mean intensities 2e-6 relative)."""
    r = no.prepare_amplitudes(_pre_cube(), PRE["originRows"], PRE["originColumns"], shift)
    assert gap(r.values.ravel(), PRE[f"order{order}_amplitudes"]) < 2e-6
    assert abs(r.mean_intensity / float(PRE[f"order{order}_meanIntensity"]) - 1) < 2e-6
    assert abs(r.clipped_mean_intensity / float(PRE[f"order{order}_clippedMeanIntensity"]) - 1) < 2e-6


def test_prepared_amplitudes_meet_the_engine_pin():
    """``PtychographyTests.swift:184-193``: the raw 64-pattern cube with a uniform origin, bilinear, through to the
    engine's amplitude pin and py4DSTEM's mean intensity."""
    rows, columns = int(PTYCHO["rows"]), int(PTYCHO["columns"])
    raw = PTYCHO["preprocessing_raw"].reshape(-1, rows, columns)
    o = PTYCHO["preprocessing_origin"]
    r = no.prepare_amplitudes(raw, np.full(len(raw), o[0]), np.full(len(raw), o[1]), "bilinear")
    assert gap(r.values.ravel(), PTYCHO["amplitudes"]) < 2e-6
    assert abs(r.mean_intensity / float(PTYCHO["meanIntensity"]) - 1) < 2e-6


def test_zero_origin_and_integer_roll():
    """``PreparationTests.swift:63-81``: a zero origin reproduces the clipped data (exact for bilinear, FFT roundoff for
    the spline, compared as intensities), and an integer origin is a roll of the pattern."""
    cube = _pre_cube()
    count = len(cube)
    for shift, bound in (("bilinear", 1e-15), ("cubicSpline", 1e-13)):
        r = no.prepare_amplitudes(cube, np.zeros(count), np.zeros(count), shift)
        expected = np.maximum(cube.astype(np.float32).astype(np.float64), 0)
        assert gap((r.values ** 2).ravel(), expected.ravel()) < bound
    r = no.prepare_amplitudes(cube, np.full(count, 2.0), np.full(count, -3.0), "bilinear")
    rolled = np.roll(np.roll(cube.astype(np.float32).astype(np.float64), -2, axis=1), 3, axis=2)
    assert np.array_equal(r.values, np.sqrt(np.maximum(rolled, 0)))


def test_preprocessing_refusals():
    """``PreparationTests.swift:170-186`` (the amplitude part): empty cubes, a one-pixel axis, non-finite or huge
    origins, origins of the wrong count and non-finite values are invalid input."""
    cube = _pre_cube()
    count = len(cube)
    z = np.zeros(count)
    bad = [(cube[:0], z[:0], z[:0]), (cube[:, :1, :], z, z), (cube, np.full(count, np.nan), z),
           (cube, z, np.full(count, 1e9)), (cube, z[:-1], z)]
    c2 = cube.copy()
    c2[0, 0, 0] = np.inf
    bad.append((c2, z, z))
    for c, r, k in bad:
        with pytest.raises(no.PtychographyError):
            no.prepare_amplitudes(c, r, k, "bilinear")


# ---------------------------------------------------------------------------------------------- position correction

@pytest.mark.parametrize("case", gc.position_cases(), ids=lambda c: c[0])
def test_position_correction_meets_the_pins(case):
    """``PositionCorrectionTests.swift:43-62``: object, probe and errors within 2e-6 of max(1, max|b|), positions within
    2e-6 px, and the positions did move (more than 0.05 px)."""
    name, inputs, settings, (obj, probe, errors, positions) = case
    o, p, e, pos = no.reconstruct(**inputs, position_correction=no.PositionCorrection(**settings))
    assert max(gap(pos[:, 0], positions[:, 0]), gap(pos[:, 1], positions[:, 1])) < 2e-6
    assert max(gc.complex_gap(o, obj), gc.complex_gap(p, probe), gap(e, errors)) < 2e-6
    assert np.max(np.abs(pos - inputs["positions"])) > 0.05


def test_position_correction_moves_toward_the_data_positions():
    """``PositionCorrectionTests.swift:83-101``: exact object and probe, object frozen; the corrected positions meet
    py4DSTEM's at 2e-6 and their mean distance to the data's positions drops below 0.7 of the start's."""
    inputs, settings, expected, truth, _ = gc.position_exact_case()
    _, _, _, pos = no.reconstruct(**inputs, position_correction=no.PositionCorrection(**settings))
    assert max(gap(pos[:, 0], expected[:, 0]), gap(pos[:, 1], expected[:, 1])) < 2e-6
    before = np.mean(np.hypot(*(inputs["positions"] - truth).T))
    after = np.mean(np.hypot(*(pos - truth).T))
    assert after < 0.7 * before


def test_position_correction_limits_zero_step_and_refusals():
    """``PositionCorrectionTests.swift:64-81,103-141``: a zero step leaves everything as without the option; the update
    limit clips moves (some to the limit); a total limit smaller than any move keeps every position; invalid settings
    are refused."""
    name, inputs, settings, _ = gc.position_cases()[0]
    short = dict(inputs, iterations=2)
    o0, p0, e0 = no.reconstruct(**short)
    o1, p1, e1, pos = no.reconstruct(**short, position_correction=no.PositionCorrection(step_size=0.0))
    assert np.array_equal(pos, inputs["positions"]) and np.array_equal(o0, o1) and np.array_equal(e0, e1)
    one = dict(inputs, iterations=1)
    rs, cs = settings["row_sampling"], settings["column_sampling"]
    _, _, _, pos = no.reconstruct(**one, position_correction=no.PositionCorrection(
        step_size=0.5, max_update_distance=0.2, row_sampling=rs, column_sampling=cs))
    limit = 0.2 / np.hypot(rs, cs)
    moves = np.hypot(*(pos - inputs["positions"]).T)
    assert moves.max() <= limit * (1 + 1e-12) and moves.max() > 0.5 * limit
    _, _, _, pos = no.reconstruct(**one, position_correction=no.PositionCorrection(
        step_size=0.5, max_total_distance=1e-6, row_sampling=rs, column_sampling=cs))
    assert np.array_equal(pos, inputs["positions"])
    for bad in (no.PositionCorrection(step_size=np.nan), no.PositionCorrection(step_size=np.inf),
                no.PositionCorrection(max_update_distance=1.0),
                no.PositionCorrection(max_update_distance=-1.0, row_sampling=rs, column_sampling=cs),
                no.PositionCorrection(max_total_distance=0.0, row_sampling=rs, column_sampling=cs),
                no.PositionCorrection(max_update_distance=1.0, row_sampling=0.0, column_sampling=cs)):
        with pytest.raises(no.PtychographyError):
            no.reconstruct(**one, position_correction=bad)


# ---------------------------------------------------------------------------------------------------- mixed state

@pytest.mark.parametrize("case", gc.mixed_cases(), ids=lambda c: c[0])
def test_mixedstate_meets_the_pins(case):
    """``EngineTests.swift:86-110,262-305``: object, errors and phase-aligned probes within 2e-6; without the
    orthogonalisation the probes themselves (no free phase)."""
    name, inputs, (obj, probes, errors), orthogonalized = case
    o, p, e = no.mixedstate_reconstruct(**inputs)
    assert max(gc.complex_gap(o, obj), gap(e, errors), gc.complex_gap(gc.align_phases(p, probes), probes)) < 2e-6
    if not orthogonalized:
        assert gc.complex_gap(p, probes) < 2e-6


def test_mixedstate_orthogonalization_and_initial_states():
    """``EngineTests.swift:111-149``: the orthogonalisation pin (phase-aligned), mutually orthogonal states of the same
    total intensity in decreasing order; py4DSTEM's initial states from NumPy's RandomState draws."""
    x, expected = gc.mixed_orthogonalization_case()
    q = no.orthogonalize(x)
    assert gc.complex_gap(gc.align_phases(q, expected), expected) < 2e-6
    flat = q.reshape(len(q), -1)
    g = np.conj(flat) @ flat.T
    assert np.max(np.abs(g - np.diag(np.diag(g)))) < 1e-13 * np.max(np.abs(np.diag(g)))
    assert abs(np.sum(np.abs(q) ** 2) - np.sum(np.abs(x) ** 2)) < 1e-12 * np.sum(np.abs(x) ** 2)
    energy = np.real(np.diag(g))
    assert np.all(energy[:-1] >= energy[1:])
    for first, count, seed, states, draws in gc.mixed_init_cases():
        assert gc.complex_gap(no.initial_probes(first, count, seed), states) < 2e-6
        assert np.array_equal(np.random.RandomState(seed).rand(len(draws)), draws)


def test_mixedstate_initial_probes_of_the_package():
    """``EngineTests.swift:131-149``: the package's host-side ``initial_probes`` (NumPy's RandomState draws) against
    py4DSTEM's initial states."""
    import cubokit_b200 as cb
    for first, count, seed, states, draws in gc.mixed_init_cases():
        assert gc.complex_gap(cb.MixedstatePtychography.initial_probes(first, count, seed), states) < 2e-6


# ---------------------------------------------------------------------------------------------------- multislice

@pytest.mark.parametrize("case", gc.multislice_cases(), ids=lambda c: c[0])
def test_multislice_meets_the_pins(case):
    """``EngineTests.swift:205-228,262-305``: slices, probe and errors within 2e-6."""
    name, inputs, (obj, probe, errors) = case
    o, p, e = no.multislice_reconstruct(**inputs)
    assert max(gc.complex_gap(o, obj), gc.complex_gap(p, probe), gap(e, errors)) < 2e-6


def test_multislice_propagators_one_slice_and_refusals():
    """``EngineTests.swift:192-203,230-255``: the propagator pin (unit modulus), one slice equals the single-slice engine
    (1e-12), a thickness count other than slices - 1 and non-positive samplings are refused."""
    args, expected = gc.multislice_propagator_case()
    props = no.propagators(**args)
    assert gc.complex_gap(props, expected) < 2e-6
    assert np.max(np.abs(np.abs(props) - 1)) < 1e-14
    name, inputs, _ = gc.multislice_cases()[0]
    one = dict(inputs, obj=inputs["obj"][:1], slice_thicknesses=[], error_normalization="suppliedAmplitudeEnergy")
    one.pop("mean_intensity")
    o1, p1, e1 = no.multislice_reconstruct(**one)
    o2, p2, e2 = no.reconstruct(one["amplitudes"], one["positions"], one["obj"][0], one["probe"], iterations=3,
                                step_size=0.35, normalization_minimum=0.7)
    assert max(gc.complex_gap(o1[0], o2), gc.complex_gap(p1, p2), gap(e1, e2)) < 1e-12
    with pytest.raises(no.PtychographyError):
        no.multislice_reconstruct(**dict(inputs, slice_thicknesses=[10.0]))
    with pytest.raises(no.PtychographyError):
        no.propagators(**dict(args, row_sampling=0.0))


@pytest.mark.parametrize("shape,step", [((256, 256), 8), ((160, 200), 8), ((512, 64), 8)])
def test_c_and_numpy_oracles_agree_on_large_detectors(shape, step):
    """The C oracle the large-detector GPU tests check against, against the NumPy restatement on the same scenes:
    detectors above one CTA's plane, square and not, power-of-two and mixed-radix lengths."""
    s = scenes.raster_scene(scan=3, det=shape[0], step=step, seed=31, shape=shape)
    amps = s["amplitudes"].astype(np.float32).astype(np.float64)
    a = c_oracle.reconstruct(amps, s["positions"], s["object"], s["probe"], iterations=2)
    b = numpy_oracle.reconstruct(amps, s["positions"], s["object"], s["probe"], iterations=2)
    for x, y in zip(a, b):
        assert gc.complex_gap(np.asarray(x), np.asarray(y)) < 1e-11, shape
