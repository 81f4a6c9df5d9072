"""The multislice engine on the device (FP64, through the C ABI) against CuboKit's py4DSTEM pins and the FP64 NumPy
restatement of ``MultislicePtychography.reconstruct`` (``PtychographyEngines.swift:458-588``).

Bounds: the reference's own (``EngineTests.swift:5-8``): slices, probe and errors 2e-6 of max(1, max|b|); against the
restatement on the same inputs 1e-9 (the same FP64 arithmetic in another summation order).
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
    amplitudes, positions, obj, probe = kw.pop("amplitudes"), kw.pop("positions"), kw.pop("obj"), kw.pop("probe")
    if kw.get("error_normalization") == "meanIntensity":
        kw["error_normalization"] = ("meanIntensity", kw.pop("mean_intensity"))
    else:
        kw.pop("mean_intensity", None)
    return cb.MultislicePtychography.reconstruct(amplitudes, positions, obj, probe, **kw)


@pytest.mark.parametrize("case", gc.multislice_cases(), ids=lambda c: c[0])
def test_multislice_meets_the_pins(cb, case):
    """``EngineTests.swift:205-228`` (one to three slices, pure phase, identical slices, fixed probe, centre of mass,
    amplitude constraint) and ``:262-305`` (aperture and support)."""
    name, inputs, (obj, probe, errors) = case
    r = _gpu(cb, inputs)
    assert max(gc.complex_gap(r.object, obj), gc.complex_gap(r.probe, probe), gap(r.errors, errors)) < 2e-6, name


def test_one_slice_equals_the_single_slice_engine(cb):
    """``EngineTests.swift:230-245``: one slice (no propagation) is the single-slice engine; here against the FP64
    single-slice engine on the device, to FP64 roundoff."""
    name, inputs, _ = gc.multislice_cases()[0]
    one = dict(inputs, obj=inputs["obj"][:1], slice_thicknesses=[], error_normalization="suppliedAmplitudeEnergy")
    one.pop("mean_intensity")
    r1 = _gpu(cb, one)
    r2 = cb.SingleslicePtychography.reconstruct(one["amplitudes"], one["positions"], one["obj"][0], one["probe"],
                                                iterations=3, step_size=0.35, normalization_minimum=0.7,
                                                precision="fp64")
    assert max(gc.complex_gap(r1.object[0], r2.object), gc.complex_gap(r1.probe, r2.probe),
               gap(r1.errors, r2.errors)) < 1e-12


@pytest.mark.parametrize("shape,slices", [((40, 48), 3), ((128, 128), 2)])
def test_against_the_oracle_on_raster_scenes(cb, shape, slices):
    """Raster scenes at fractional positions (a non-square detector; the 128 x 128 detector of the benchmark), slices
    from a seeded perturbation of the start, centre of mass and amplitude constraint on, against the restatement."""
    s = scenes.raster_scene(scan=3, det=shape[0], step=6, seed=sum(shape) + slices, shape=shape)
    rng = np.random.default_rng(slices)
    start = s["positions"] + np.array([0.3, -0.2])
    obj = np.stack([s["object"] * np.exp(0.05j * rng.standard_normal(s["object"].shape)) for _ in range(slices)])
    kw = dict(slice_thicknesses=[40.0 + 15.0 * i for i in range(slices - 1)], wavelength=0.0197, row_sampling=0.45,
              column_sampling=0.5, iterations=3, step_size=0.5, normalization_minimum=0.8,
              fix_probe_center_of_mass=True, constrain_probe_amplitude=True, identical_slices=slices == 2)
    o, p, e = no.multislice_reconstruct(s["amplitudes"], start, obj, s["probe"], **kw)
    r = cb.MultislicePtychography.reconstruct(s["amplitudes"], start, obj, s["probe"], **kw)
    assert max(gc.complex_gap(r.object, o), gc.complex_gap(r.probe, p), gap(r.errors, e)) < 1e-9
    if slices == 2:
        assert np.array_equal(r.object[0], r.object[1])


def test_plan_resume_and_refusals(cb):
    """Two plus one iterations on a device-resident multislice plan equal three in one call, bit for bit; a thickness
    count other than slices - 1 and a non-positive sampling are refused (``EngineTests.swift:247-255``)."""
    name, inputs, _ = gc.multislice_cases()[1]
    full = _gpu(cb, inputs)
    kw = dict(inputs)
    amplitudes, positions, obj, probe = kw.pop("amplitudes"), kw.pop("positions"), kw.pop("obj"), kw.pop("probe")
    kw.pop("iterations")
    kw["error_normalization"] = ("meanIntensity", kw.pop("mean_intensity"))
    multislice = dict(slices=obj.shape[0], slice_thicknesses=kw.pop("slice_thicknesses"),
                      wavelength=kw.pop("wavelength"), row_sampling=kw.pop("row_sampling"),
                      column_sampling=kw.pop("column_sampling"), identical_slices=kw.pop("identical_slices"))
    kw["constrain_object_amplitude"] = True
    plan = cb.Plan(amplitudes, positions, obj.shape[1:], probe.shape, multislice=multislice, **kw)
    plan.set_state(obj, probe)
    e = np.concatenate([plan.iterate(2), plan.iterate(1)])
    o, p = plan.get_state()
    assert np.array_equal(e, full.errors) and np.array_equal(o, full.object) and np.array_equal(p, full.probe)
    with pytest.raises(cb.UnsupportedError):
        plan.forward()
    plan.close()
    with pytest.raises(cb.PtychographyError):
        _gpu(cb, dict(inputs, slice_thicknesses=[10.0] * obj.shape[0]))
    with pytest.raises(cb.PtychographyError):
        _gpu(cb, dict(inputs, row_sampling=0.0))



def test_edge_cases(cb):
    """Zero iterations return the inputs bit for bit with no errors; one position, and six slices on a non-square
    detector, agree with the restatement."""
    name, inputs, _ = gc.multislice_cases()[0]
    r0 = _gpu(cb, dict(inputs, iterations=0))
    assert np.array_equal(r0.object, inputs["obj"]) and np.array_equal(r0.probe, inputs["probe"])
    assert len(r0.errors) == 0
    one = dict(inputs, amplitudes=inputs["amplitudes"][:1], positions=inputs["positions"][:1],
               error_normalization="suppliedAmplitudeEnergy")
    one.pop("mean_intensity")
    r1 = _gpu(cb, one)
    kw = {k: v for k, v in one.items() if k not in ("amplitudes", "positions", "obj", "probe")}
    o, p, e = no.multislice_reconstruct(one["amplitudes"], one["positions"], one["obj"], one["probe"], **kw)
    assert max(gc.complex_gap(r1.object, o), gc.complex_gap(r1.probe, p), gap(r1.errors, e)) < 1e-9
    s = scenes.raster_scene(scan=2, det=24, step=5, seed=3, shape=(24, 20))
    obj = np.stack([s["object"]] * 6)
    kw6 = dict(slice_thicknesses=[12.0] * 5, wavelength=0.0197, row_sampling=0.5, column_sampling=0.45, iterations=2,
               step_size=0.5)
    o, p, e = no.multislice_reconstruct(s["amplitudes"], s["positions"] + 0.3, obj, s["probe"], **kw6)
    r6 = cb.MultislicePtychography.reconstruct(s["amplitudes"], s["positions"] + 0.3, obj, s["probe"], **kw6)
    assert max(gc.complex_gap(r6.object, o), gc.complex_gap(r6.probe, p), gap(r6.errors, e)) < 1e-9
