"""The FP32 position pass through global memory (``global32.cu``) against the FP64 C oracle.

It serves FP32 detectors above one CTA's shared memory (more than 16,384 pixels: 256 x 256, 160 x 200 ...) and any
detector with ``variant="global"``.  Bounds are the reference's Float-vs-Double ones, as for every FP32 test
(``SinglePrecisionTests.swift:5-8,64-69``): object 1e-4 and probe 1e-5 absolute, errors 1e-5 relative (1e-4 for the
fractional non-square scenes, ``SinglePrecisionTests.swift:204-208``).
"""
import numpy as np
import pytest

from oracle import c_oracle
from tests import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cb():
    import cubokit_b200
    return cubokit_b200


def _check(ref, r, err_rel=1e-5):
    assert np.max(np.abs(ref[0] - r.object)) <= 1e-4
    assert np.max(np.abs(ref[1] - r.probe)) <= 1e-5 * max(1.0, float(np.max(np.abs(ref[1]))))
    assert np.all(np.abs(ref[2] - r.errors) <= err_rel * np.abs(ref[2])), (r.errors, ref[2])
    assert r.errors[-1] < r.errors[0]


@pytest.mark.parametrize("shape,step", [((256, 256), 8), ((160, 200), 8), ((192, 192), 6), ((512, 64), 8)])
def test_large_fp32_detectors_against_fp64_oracle(cb, shape, step):
    """Detectors whose FP32 plane exceeds one CTA: compile-time radix plans (256 = 8*8*4, 192 = 8*8*3, 512 = 8*8*8)
    and run-time ones (160 = 8*4*5, 200 = 8*5*5, 64 = 8*8), square and not."""
    s = scenes.raster_scene(scan=3, det=shape[0], step=step, seed=31, shape=shape)
    ref = c_oracle.reconstruct(s["amplitudes"].astype(np.float32), s["positions"], s["object"], s["probe"],
                               iterations=3)
    r = cb.SingleslicePtychography.reconstruct(s["amplitudes"], s["positions"], s["object"], s["probe"], iterations=3,
                                               precision="fp32")
    _check(ref, r)


@pytest.mark.parametrize("shape", [(32, 48), (22, 21), (13, 26), (128, 128)])
def test_global_variant_at_small_detectors_against_fp64_oracle(cb, shape):
    """``variant="global"`` takes the same pass at sizes the shared-memory kernels also serve: fractional positions,
    a prime-length axis (direct DFT), and 128 x 128 (8*8*2)."""
    size = 96 if shape == (32, 48) else 2 * max(shape) + 40
    s = scenes.nonsquare_scene(shape[0], shape[1], size)
    ref = c_oracle.reconstruct(s["amplitudes"].astype(np.float32), s["positions"], s["object"], s["probe"],
                               iterations=3)
    r = cb.SingleslicePtychography.reconstruct(s["amplitudes"], s["positions"], s["object"], s["probe"], iterations=3,
                                               precision="fp32", variant="global")
    _check(ref, r, err_rel=1e-4)


def test_global_variant_agrees_with_the_shared_memory_pass(cb):
    """The same reconstruction through global memory and through the any-size shared-memory kernel: FP32 round-off
    apart (the 2-D transform's 1-D passes run in a different order), the same result."""
    s = scenes.raster_scene(scan=5, det=48, step=4, seed=17)
    kw = dict(iterations=4, precision="fp32")
    a = cb.SingleslicePtychography.reconstruct(s["amplitudes"], s["positions"], s["object"], s["probe"],
                                               variant="global", **kw)
    b = cb.SingleslicePtychography.reconstruct(s["amplitudes"], s["positions"], s["object"], s["probe"],
                                               variant="generic", **kw)
    assert np.max(np.abs(a.object - b.object)) <= 2e-5
    assert np.all(np.abs(a.errors - b.errors) <= 1e-5 * np.abs(b.errors))


def test_large_detector_is_deterministic(cb):
    """Fixed-order sums everywhere: two runs give the same bits."""
    s = scenes.raster_scene(scan=3, det=256, step=8, seed=32)
    runs = [cb.SingleslicePtychography.reconstruct(s["amplitudes"], s["positions"], s["object"], s["probe"],
                                                   iterations=2, precision="fp32") for _ in range(2)]
    assert np.array_equal(runs[0].object, runs[1].object)
    assert np.array_equal(runs[0].probe, runs[1].probe)
    assert np.array_equal(runs[0].errors, runs[1].errors)


def test_large_detector_in_a_batch_matches_its_own_reconstruction(cb):
    """A 256 x 256 FP32 item (its own pass launches) beside a 64 x 64 one (grouped) in one captured batch."""
    items = []
    for scan, det, step, seed in [(3, 256, 8, 41), (4, 64, 4, 42)]:
        s = scenes.raster_scene(scan=scan, det=det, step=step, seed=seed)
        items.append(dict(amplitudes=s["amplitudes"], positions=s["positions"], object=s["object"], probe=s["probe"],
                          step_size=0.5, precision="fp32"))
    batch = cb.Batch(items)
    batch.run(2)
    for i, it in enumerate(items):
        r = cb.SingleslicePtychography.reconstruct(it["amplitudes"], it["positions"], it["object"], it["probe"],
                                                   iterations=2, step_size=0.5, precision="fp32")
        o, p = batch.get_state(i)
        assert np.array_equal(o, r.object), i
        assert np.array_equal(p, r.probe), i
