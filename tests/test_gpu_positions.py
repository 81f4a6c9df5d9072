"""Position correction on the device (FP64 form, through the C ABI) against CuboKit's py4DSTEM pins and the FP64
NumPy restatement of ``Ptychography.swift:371-377,398-401,411-472``.

Bounds: the reference's own (``PositionCorrectionTests.swift:5-8``): object, probe and errors 2e-6 of max(1, max|b|),
positions 2e-6 px (absolute, over max(1, max)).
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


def _gpu(cb, inputs, settings=None, **extra):
    kw = dict(inputs)
    kw.update(extra)
    amplitudes, positions, obj, probe = kw.pop("amplitudes"), kw.pop("positions"), kw.pop("obj"), kw.pop("probe")
    if kw.get("error_normalization") == "meanIntensity":
        kw["error_normalization"] = ("meanIntensity", kw.pop("mean_intensity"))
    else:
        kw.pop("mean_intensity", None)
    pc = None if settings is None else cb.PtychographyPositionCorrection(**settings)
    return cb.SingleslicePtychography.reconstruct(amplitudes, positions, obj, probe, precision="fp64",
                                                  position_correction=pc, **kw)


def _position_gap(a, b):
    return max(gap(a[:, 0], b[:, 0]), gap(a[:, 1], b[:, 1]))


@pytest.mark.parametrize("case", gc.position_cases(), ids=lambda c: c[0])
def test_position_correction_meets_the_pins(cb, case):
    """``PositionCorrectionTests.swift:43-62``: the five settings (default, small step, both limits, centre of mass,
    fixed probe), four iterations."""
    name, inputs, settings, (obj, probe, errors, positions) = case
    r = _gpu(cb, inputs, settings)
    assert _position_gap(r.positions, positions) < 2e-6, name
    assert max(gc.complex_gap(r.object, obj), gc.complex_gap(r.probe, probe), gap(r.errors, errors)) < 2e-6, name
    assert np.max(np.abs(r.positions - inputs["positions"])) > 0.05  # the option did something


def test_positions_move_toward_the_data_positions(cb):
    """``PositionCorrectionTests.swift:83-101``: exact object and probe, object frozen: the correction alone moves the
    positions, to py4DSTEM's at 2e-6 and closer to the data's positions."""
    inputs, settings, expected, truth, _ = gc.position_exact_case()
    r = _gpu(cb, inputs, settings)
    assert _position_gap(r.positions, expected) < 2e-6
    before = np.mean(np.hypot(*(inputs["positions"] - truth).T))
    after = np.mean(np.hypot(*(r.positions - truth).T))
    assert after < 0.7 * before


def test_off_by_default_and_a_zero_step_changes_nothing(cb):
    """``PositionCorrectionTests.swift:64-81``: without the option the positions come back as given; a zero step moves
    nothing and leaves object, probe and errors bit for bit as without the option."""
    name, inputs, settings, _ = gc.position_cases()[0]
    short = dict(inputs, iterations=2)
    plain = _gpu(cb, short)
    assert np.array_equal(plain.positions, inputs["positions"])
    zero = _gpu(cb, short, dict(settings, step_size=0.0))
    assert np.array_equal(zero.positions, inputs["positions"])
    assert np.array_equal(zero.object, plain.object) and np.array_equal(zero.probe, plain.probe)
    assert np.array_equal(zero.errors, plain.errors)


def test_limits_are_honoured(cb):
    """``PositionCorrectionTests.swift:103-118``: the update limit clips every move (some to the limit); a total limit
    smaller than any move keeps every position."""
    name, inputs, settings, _ = gc.position_cases()[0]
    one = dict(inputs, iterations=1)
    rs, cs = settings["row_sampling"], settings["column_sampling"]
    r = _gpu(cb, one, dict(step_size=0.5, max_update_distance=0.2, row_sampling=rs, column_sampling=cs))
    limit = 0.2 / np.hypot(rs, cs)
    moves = np.hypot(*(r.positions - inputs["positions"]).T)
    assert moves.max() <= limit * (1 + 1e-12) and moves.max() > 0.5 * limit
    held = _gpu(cb, one, dict(step_size=0.5, max_total_distance=1e-6, row_sampling=rs, column_sampling=cs))
    assert np.array_equal(held.positions, inputs["positions"])


def test_invalid_settings_and_forms_are_refused(cb):
    """``PositionCorrectionTests.swift:120-141`` (invalid settings) and ``Ptychography.swift:236`` (the Float path
    refuses the option: here the FP32 and split-BF16 forms), and graph-replayed batches."""
    name, inputs, settings, _ = gc.position_cases()[0]
    one = dict(inputs, iterations=1)
    bad = [dict(step_size=np.nan), dict(step_size=np.inf), dict(step_size=0.5, max_update_distance=1.0),
           dict(step_size=0.5, max_total_distance=1.0, row_sampling=1.0),
           dict(step_size=0.5, max_update_distance=-1.0, row_sampling=1.0, column_sampling=1.0),
           dict(step_size=0.5, max_total_distance=0.0, row_sampling=1.0, column_sampling=1.0),
           dict(step_size=0.5, max_update_distance=1.0, row_sampling=0.0, column_sampling=1.0),
           dict(step_size=0.5, max_update_distance=np.nan, row_sampling=1.0, column_sampling=1.0)]
    for b in bad:
        with pytest.raises(cb.PtychographyError):
            _gpu(cb, one, b)
    kw = dict(one)
    amplitudes, positions, obj, probe = kw.pop("amplitudes"), kw.pop("positions"), kw.pop("obj"), kw.pop("probe")
    kw["error_normalization"] = ("meanIntensity", kw.pop("mean_intensity"))
    with pytest.raises(cb.PtychographyError):
        cb.SingleslicePtychography.reconstruct(amplitudes, positions, obj, probe, precision="fp32",
                                               position_correction=cb.PtychographyPositionCorrection(), **kw)
    with pytest.raises(cb.PtychographyError):
        cb.Batch([dict(amplitudes=amplitudes, positions=positions, object=obj, probe=probe, precision="fp64",
                       position_correction=cb.PtychographyPositionCorrection())])


def test_plan_resume_and_positions(cb):
    """Two plus two iterations on a device-resident plan equal four in one call, bit for bit, positions included."""
    name, inputs, settings, _ = gc.position_cases()[0]
    full = _gpu(cb, inputs, settings)
    kw = dict(inputs)
    amplitudes, positions, obj, probe = kw.pop("amplitudes"), kw.pop("positions"), kw.pop("obj"), kw.pop("probe")
    kw.pop("iterations")
    kw["error_normalization"] = ("meanIntensity", kw.pop("mean_intensity"))
    plan = cb.Plan(amplitudes, positions, obj.shape, probe.shape, precision="fp64",
                   position_correction=cb.PtychographyPositionCorrection(**settings), **kw)
    plan.set_state(obj, probe)
    e = np.concatenate([plan.iterate(2), plan.iterate(2)])
    o, p = plan.get_state()
    assert np.array_equal(e, full.errors) and np.array_equal(o, full.object) and np.array_equal(p, full.probe)
    assert np.array_equal(plan.positions(), full.positions)
    plan.close()


@pytest.mark.parametrize("shape", [(24, 24), (20, 28)])
def test_against_the_oracle_on_a_raster_started_off_its_positions(cb, shape):
    """A raster scene whose positions start up to 0.45 px off (non-square detector too), three iterations with a
    per-iteration limit and the centre-of-mass constraint, against the FP64 restatement (same Float32 amplitudes)."""
    s = scenes.raster_scene(scan=5, det=shape[0], step=5, seed=sum(shape), shape=shape)
    rng = np.random.default_rng(7)
    start = s["positions"] + rng.uniform(-0.45, 0.45, s["positions"].shape)
    settings = dict(step_size=0.5, max_update_distance=0.3, max_total_distance=None, row_sampling=0.5,
                    column_sampling=0.7, constrain_center_of_mass=True)
    kw = dict(iterations=3, step_size=0.5, normalization_minimum=0.8)
    o, p, e, pos = no.reconstruct(s["amplitudes"], start, s["object"], s["probe"], **kw,
                                  position_correction=no.PositionCorrection(**settings))
    r = cb.SingleslicePtychography.reconstruct(s["amplitudes"], start, s["object"], s["probe"], precision="fp64",
                                               position_correction=cb.PtychographyPositionCorrection(**settings), **kw)
    assert _position_gap(r.positions, pos) < 2e-6
    assert max(gc.complex_gap(r.object, o), gc.complex_gap(r.probe, p), gap(r.errors, e)) < 2e-6
    assert np.max(np.abs(r.positions - start)) > 0.01


# ------------------------------------------------------------------ FP64 planes larger than one CTA (global memory)

def test_fp64_global_pass_equals_the_shared_memory_pass(cb):
    """The FP64 position pass through global memory (forced on a 48 x 40 detector) against the shared-memory pass:
    the same line transforms in the same order, so the same results to FP64 roundoff."""
    s = scenes.raster_scene(scan=4, det=48, step=6, seed=21, shape=(48, 40))
    kw = dict(iterations=3, step_size=0.5, precision="fp64")
    a = cb.SingleslicePtychography.reconstruct(s["amplitudes"], s["positions"] + 0.25, s["object"], s["probe"], **kw)
    b = cb.SingleslicePtychography.reconstruct(s["amplitudes"], s["positions"] + 0.25, s["object"], s["probe"],
                                               variant="global", **kw)
    assert gc.complex_gap(a.object, b.object) < 1e-12 and gc.complex_gap(a.probe, b.probe) < 1e-12
    assert gap(a.errors, b.errors) < 1e-12


def test_fp64_form_at_128x128_against_the_oracle(cb):
    """128 x 128 detectors in the FP64 form (the reference's default precision): against the FP64 restatement, with
    fractional positions and with position correction."""
    s = scenes.raster_scene(scan=3, det=128, step=8, seed=5)
    start = s["positions"] + np.array([0.3, -0.2])
    kw = dict(iterations=2, step_size=0.5, normalization_minimum=0.8)
    o, p, e = no.reconstruct(s["amplitudes"], start, s["object"], s["probe"], **kw)
    r = cb.SingleslicePtychography.reconstruct(s["amplitudes"], start, s["object"], s["probe"], precision="fp64", **kw)
    assert max(gc.complex_gap(r.object, o), gc.complex_gap(r.probe, p), gap(r.errors, e)) < 1e-9
    settings = dict(step_size=0.5, max_update_distance=None, max_total_distance=None, row_sampling=None,
                    column_sampling=None, constrain_center_of_mass=False)
    o, p, e, pos = no.reconstruct(s["amplitudes"], start, s["object"], s["probe"], **kw,
                                  position_correction=no.PositionCorrection(**settings))
    r = cb.SingleslicePtychography.reconstruct(s["amplitudes"], start, s["object"], s["probe"], precision="fp64",
                                               position_correction=cb.PtychographyPositionCorrection(**settings), **kw)
    assert _position_gap(r.positions, pos) < 2e-6
    assert max(gc.complex_gap(r.object, o), gc.complex_gap(r.probe, p), gap(r.errors, e)) < 2e-6
