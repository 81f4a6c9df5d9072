"""Batches: independent reconstructions of different scan, detector and object sizes, replayed from one captured CUDA
graph (the passes of items with a compile-time-plan detector and every item's gathers in grouped persistent launches),
give bitwise the results of running each reconstruction alone."""
import numpy as np
import pytest

from tests import scenes

pytestmark = pytest.mark.gpu


def _items():
    items = []
    # several items per grouped launch: two 64 x 64 FP32 passes, every item's gathers of a form
    for scan, det, seed, prec in [(4, 32, 1, "fp32"), (6, 64, 2, "fp32"), (3, 128, 3, "fp32"), (3, 128, 4, "split_bf16"),
                                  (5, 48, 5, "fp32"), (4, 64, 6, "fp64"), (5, 64, 8, "fp32"), (3, 96, 7, "fp32")]:
        s = scenes.raster_scene(scan=scan, det=det, step=4, seed=seed)
        items.append(dict(amplitudes=s["amplitudes"], positions=s["positions"], object=s["object"], probe=s["probe"],
                          step_size=0.5, precision=prec))
    s = scenes.nonsquare_scene(22, 21, 84)  # fractional positions, a Bluestein-length detector
    items.append(dict(amplitudes=s["amplitudes"], positions=s["positions"], object=s["object"], probe=s["probe"],
                      step_size=0.5, fix_probe_center_of_mass=True))
    return items


@pytest.mark.parametrize("grouped", ["1", "0"])
def test_batch_matches_individual_reconstructions_bitwise(monkeypatch, grouped):
    """Grouped launches (the default) and every item's own launches (CUBO_PTYCHO_BATCH_GROUPED=0) alike."""
    import cubokit_b200 as cb
    monkeypatch.setenv("CUBO_PTYCHO_BATCH_GROUPED", grouped)
    items = _items()
    batch = cb.Batch(items)
    batch.run(2)
    batch.run(1)  # a second run replays the same graph
    assert batch.launches_per_iteration > len(items)
    for i, it in enumerate(items):
        kw = {k: v for k, v in it.items() if k not in ("amplitudes", "positions", "object", "probe")}
        r = cb.SingleslicePtychography.reconstruct(it["amplitudes"], it["positions"], it["object"], it["probe"],
                                                   iterations=3, **kw)
        o, p = batch.get_state(i)
        assert np.array_equal(o, r.object) and np.array_equal(p, r.probe), i
        assert np.array_equal(batch.errors(i, 3), r.errors), i
    batch.close()


def test_gather_tiles_agree_bitwise_and_autotune_picks_one(tmp_path, monkeypatch):
    import cubokit_b200 as cb
    from cubokit_b200 import autotune
    monkeypatch.setenv("CUBOKIT_B200_CACHE", str(tmp_path))
    for precision, det in (("fp32", 64), ("split_bf16", 128)):
        s = scenes.raster_scene(scan=5, det=det, step=4, seed=8)
        ref = None
        for tile in (0, 1, 2, 3):
            r = cb.SingleslicePtychography.reconstruct(s["amplitudes"], s["positions"], s["object"], s["probe"],
                                                       iterations=2, precision=precision, gather_tile=tile)
            if ref is None:
                ref = r
            assert np.array_equal(r.object, ref.object) and np.array_equal(r.errors, ref.errors), (precision, tile)
        best, ms = autotune.tune(s["amplitudes"], s["positions"], s["object"], s["probe"], precision=precision)
        assert best in autotune.CANDIDATES and set(ms) == {"32x8", "16x16", "64x4"}
        assert autotune.tune(s["amplitudes"], s["positions"], s["object"], s["probe"], precision=precision)[0] == best


def test_pass_shapes_agree_bitwise_and_autotune_picks_one(tmp_path, monkeypatch):
    """The position pass at 64 x 64 and 96 x 96 runs as the shared-memory pass in several CTA shapes (128, 256, 512
    threads) or, in FP32 by default, as the register-line kernel.  The shared-memory shapes give the same object and
    probe bit for bit (the reported error is summed over the CTA's threads, so it agrees to round-off); the register-line
    kernel factors the transforms differently and agrees with them to FP32 round-off.  The autotuner times the
    candidates and caches its choice."""
    import cubokit_b200 as cb
    from cubokit_b200 import autotune
    monkeypatch.setenv("CUBOKIT_B200_CACHE", str(tmp_path))
    for precision in ("fp32", "fp64"):
        for det in (64, 96):
            s = scenes.raster_scene(scan=4, det=det, step=4, seed=9)
            results = {}
            for shape in (0, 1, 2, 3):
                plan = cb.Plan(s["amplitudes"], s["positions"], s["object"].shape, s["probe"].shape, step_size=0.5,
                               precision=precision, pass_shape=shape)
                plan.set_state(s["object"], s["probe"])
                errors = plan.iterate(2)
                o, p = plan.get_state()
                plan.close()
                results[shape] = (o, p, errors)
            ref = results[3]
            shared = (1, 2, 3) if precision == "fp32" else (0, 1, 2, 3)
            for shape in shared:
                o, p, errors = results[shape]
                assert np.array_equal(o, ref[0]) and np.array_equal(p, ref[1]), (precision, det, shape)
                assert np.allclose(errors, ref[2], rtol=1e-12 if precision == "fp64" else 1e-6, atol=0), (precision, det)
            if precision == "fp32":
                o, p, errors = results[0]
                assert np.max(np.abs(o - ref[0])) <= 1e-5 and np.max(np.abs(p - ref[1])) <= 1e-5 * np.max(np.abs(ref[1]))
                assert np.allclose(errors, ref[2], rtol=1e-5, atol=0)
            best, ms = autotune.tune_pass(s["amplitudes"], s["positions"], s["object"], s["probe"], precision=precision)
            cands = autotune.PASS_CANDIDATES[(precision, det)]
            assert best in cands and len(ms) == len(cands)
            assert autotune.tune_pass(s["amplitudes"], s["positions"], s["object"], s["probe"],
                                      precision=precision)[0] == best
