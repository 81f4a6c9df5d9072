"""The clustered 128 x 128 FP64 plane launches (``plane128.cu``: full, forward-only and inverse-only) against the
batched line transforms of the generic variant, engine by engine: the same arithmetic in another order, so the same
results to FP64 roundoff (1e-12 of max(1, max|b|)).  Every cluster size (2, 4 and 8 CTAs per plane); the size is
read once per process, so the other sizes run in child processes."""
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from tests import golden_cases as gc
from tests import scenes

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
gap = gc.gap
TOL = 1e-12


@pytest.fixture(scope="module")
def cb():
    import cubokit_b200
    return cubokit_b200


@pytest.fixture(scope="module")
def scene():
    s = scenes.raster_scene(scan=3, det=128, step=8, seed=9)
    s["start"] = s["positions"] + np.array([0.25, -0.4])
    return s


def _both(run):
    return run("auto"), run("generic")


def test_single_slice(cb, scene):
    """The FP64 single-slice pass (exit wave, FFT, projection, inverse FFT in one launch) and its shift table (one
    inverse launch over the fractional classes)."""
    a, b = _both(lambda v: cb.SingleslicePtychography.reconstruct(
        scene["amplitudes"], scene["start"], scene["object"], scene["probe"], iterations=3, step_size=0.5,
        precision="fp64", fix_probe_center_of_mass=True, variant=v))
    assert max(gc.complex_gap(a.object, b.object), gc.complex_gap(a.probe, b.probe), gap(a.errors, b.errors)) < TOL


def test_position_correction(cb, scene):
    """The three far fields of the position update (forward launches with the object patch one row / one column
    further), the shift table of one class per position."""
    pc = cb.PtychographyPositionCorrection(step_size=0.5, max_update_distance=0.3, row_sampling=0.5,
                                           column_sampling=0.5)
    a, b = _both(lambda v: cb.SingleslicePtychography.reconstruct(
        scene["amplitudes"], scene["start"], scene["object"], scene["probe"], iterations=3, step_size=0.5,
        precision="fp64", position_correction=pc, variant=v))
    assert np.max(np.abs(a.positions - b.positions)) < TOL
    assert max(gc.complex_gap(a.object, b.object), gc.complex_gap(a.probe, b.probe), gap(a.errors, b.errors)) < TOL
    assert np.max(np.abs(a.positions - scene["start"])) > 0.01


def test_mixed_state(cb, scene):
    """Every state's far field (forward launches), the summed projection, the inverses (inverse launches)."""
    probes = cb.MixedstatePtychography.initial_probes(scene["probe"] / np.sqrt(3), 3, seed=4)
    out = []
    for variant in ("auto", "generic"):
        plan = cb.Plan(scene["amplitudes"], scene["start"], scene["object"].shape, scene["probe"].shape,
                       mixed_states=3, variant=variant, step_size=0.5, fix_probe_center_of_mass=True)
        plan.set_state(scene["object"], probes)
        e = plan.iterate(3)
        o, p = plan.get_state()
        plan.close()
        out.append((o, p, e))
    (o1, p1, e1), (o2, p2, e2) = out
    assert max(gc.complex_gap(o1, o2), gc.complex_gap(p1, p2), gap(e1, e2)) < TOL


def test_multislice(cb, scene):
    """Forward slices, detector and back-propagation, one full launch each."""
    obj = np.stack([scene["object"] * np.exp(0.03j * i) for i in range(3)])
    ms = dict(slices=3, slice_thicknesses=[30.0, 50.0], wavelength=0.0197, row_sampling=0.45, column_sampling=0.5)
    out = []
    for variant in ("auto", "generic"):
        plan = cb.Plan(scene["amplitudes"], scene["start"], scene["object"].shape, scene["probe"].shape,
                       multislice=ms, variant=variant, step_size=0.5, fix_probe_center_of_mass=True)
        plan.set_state(obj, scene["probe"])
        e = plan.iterate(3)
        o, p = plan.get_state()
        plan.close()
        out.append((o, p, e))
    (o1, p1, e1), (o2, p2, e2) = out
    assert max(gc.complex_gap(o1, o2), gc.complex_gap(p1, p2), gap(e1, e2)) < TOL


@pytest.mark.parametrize("cluster", ["4", "8"])
def test_other_cluster_sizes(cluster):
    """The same four checks with four or eight CTAs per plane (CUBO_PTYCHO_PLANE_CLUSTER), in a child process."""
    if os.environ.get("CUBO_PTYCHO_PLANE_CLUSTER"):
        pytest.skip("this process already runs another cluster size")
    env = dict(os.environ, CUBO_PTYCHO_PLANE_CLUSTER=cluster)
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-x", "-p", "no:cacheprovider",
                        "tests/test_gpu_plane128.py", "-k", "not other_cluster_sizes"],
                       env=env, cwd=str(ROOT), capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
