"""The mixed-state engine on the device (FP64, through the C ABI) against CuboKit's py4DSTEM pins and the FP64 NumPy
restatement of ``MixedstatePtychography`` (``PtychographyEngines.swift:121-330``).

Bounds: the reference's (``EngineTests.swift:87-88``): 2e-6 of max(1, max|b|) on the object, the errors and the
probes, the probes after per-state phase alignment when they were orthogonalised (the eigenvector phase is free).
"""
import numpy as np
import pytest

from oracle import numpy_oracle as no
from tests import golden_cases as gc
from tests import scenes

pytestmark = pytest.mark.gpu

gap = gc.gap


@pytest.fixture(scope="module")
def cb():
    import cubokit_b200
    return cubokit_b200


def _gpu(cb, inputs, **extra):
    kw = dict(inputs)
    kw.update(extra)
    amplitudes, positions, obj, probes = kw.pop("amplitudes"), kw.pop("positions"), kw.pop("obj"), kw.pop("probes")
    if kw.get("error_normalization") == "meanIntensity":
        kw["error_normalization"] = ("meanIntensity", kw.pop("mean_intensity"))
    else:
        kw.pop("mean_intensity", None)
    return cb.MixedstatePtychography.reconstruct(amplitudes, positions, obj, probes, **kw)


@pytest.mark.parametrize("case", gc.mixed_cases(), ids=lambda c: c[0])
def test_mixedstate_meets_the_pins(cb, case):
    """``EngineTests.swift:86-110`` (two and three states; centre of mass, amplitude constraint, no orthogonalisation,
    fixed probe, pure phase) and ``:262-305`` (the mixed engine's aperture / support extras)."""
    name, inputs, (obj, probes, errors), orthogonalized = case
    r = _gpu(cb, inputs)
    assert r.probes.shape == probes.shape
    g = max(gc.complex_gap(r.object, obj), gap(r.errors, errors),
            gc.complex_gap(gc.align_phases(r.probes, probes), probes))
    assert g < 2e-6, (name, g)
    if not orthogonalized:
        assert gc.complex_gap(r.probes, probes) < 2e-6


def test_orthogonalization_on_the_device(cb):
    """``EngineTests.swift:111-128``: the pin (phase-aligned), orthogonal states, the same total intensity, intensities
    in decreasing order."""
    x, expected = gc.mixed_orthogonalization_case()
    q = cb.MixedstatePtychography.orthogonalize(x)
    assert gc.complex_gap(gc.align_phases(q, expected), expected) < 2e-6
    flat = q.reshape(len(q), -1)
    g = np.conj(flat) @ flat.T
    assert np.max(np.abs(g - np.diag(np.diag(g)))) < 1e-13 * np.max(np.abs(np.diag(g)))
    assert abs(np.sum(np.abs(q) ** 2) - np.sum(np.abs(x) ** 2)) < 1e-12 * np.sum(np.abs(x) ** 2)
    energy = np.real(np.diag(g))
    assert np.all(energy[:-1] >= energy[1:])


def test_fixed_probe_leaves_the_states_alone_and_refusals(cb):
    """``EngineTests.swift:158-186``: a fixed probe without orthogonalisation returns the states bit for bit (centre of
    mass and amplitude constraint are gated on it); invalid input is refused."""
    name, inputs, _, _ = gc.mixed_cases()[1]
    r = _gpu(cb, inputs, iterations=2, fix_probe=True, fix_probe_center_of_mass=True, constrain_probe_amplitude=True,
             orthogonalize_probes=False)
    assert np.array_equal(r.probes, inputs["probes"])
    with pytest.raises(cb.PtychographyError):
        _gpu(cb, inputs, constrain_probe_amplitude=True, probe_amplitude_relative_radius=0.9)
    with pytest.raises(cb.PtychographyError):
        cb.MixedstatePtychography.reconstruct([], [], inputs["obj"], inputs["probes"])
    with pytest.raises(cb.PtychographyError):
        _gpu(cb, inputs, probes=np.repeat(inputs["probes"][:1], 17, axis=0))


def test_zero_far_field_pixels(cb):
    """``PtychographyEngines.swift:188-195``: with zero probes every far-field pixel is exactly zero: an infinite
    error (py4DSTEM) or, in the finite mode, sum A^2 over the divisor; nothing moves."""
    name, inputs, _, _ = gc.mixed_cases()[0]
    zero = np.zeros_like(inputs["probes"])
    r = _gpu(cb, inputs, probes=zero, iterations=1)
    assert np.isinf(r.errors[0])
    f = _gpu(cb, inputs, probes=zero, iterations=1, zero_far_field_pixel_error="finite")
    expected = np.sum(np.asarray(inputs["amplitudes"], np.float32).astype(np.float64) ** 2) / (
        inputs["mean_intensity"] * len(inputs["positions"]))
    assert abs(f.errors[0] / expected - 1) < 1e-12
    assert np.array_equal(f.probes, zero)


@pytest.mark.parametrize("shape,states", [((40, 48), 3), ((128, 128), 2)])
def test_against_the_oracle_on_raster_scenes(cb, shape, states):
    """Fractional raster scenes (non-square, and 128 x 128) with seeded initial states, three iterations with the
    centre of mass, the amplitude constraint and the orthogonalisation, against the FP64 restatement."""
    s = scenes.raster_scene(scan=3, det=shape[0], step=6, seed=sum(shape) + states, shape=shape)
    start = cb.MixedstatePtychography.initial_probes(s["probe"], states, seed=11)
    positions = s["positions"] + np.array([0.25, -0.35])
    kw = dict(iterations=3, step_size=0.5, normalization_minimum=0.8, fix_probe_center_of_mass=True,
              constrain_probe_amplitude=True, probe_amplitude_relative_radius=0.45,
              probe_amplitude_relative_width=0.08)
    o, p, e = no.mixedstate_reconstruct(s["amplitudes"], positions, s["object"], start, **kw)
    r = cb.MixedstatePtychography.reconstruct(s["amplitudes"], positions, s["object"], start, **kw)
    assert max(gc.complex_gap(r.object, o), gap(r.errors, e), gc.complex_gap(gc.align_phases(r.probes, p), p)) < 1e-9
