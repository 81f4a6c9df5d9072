"""The adjoint pair (cubo_ptycho_plan_forward / _backward) against central finite differences and the CPU gradient.

Geometry of the differentiation check: 16 x 16 raster, step 4 px, 64 x 64 detector, 128 x 128 object, integer positions
(the reference's probe accumulation does not undo fractional shifts, so it is the exact probe gradient only for integer
positions).  Loss L = sum_p sum_k (|F_k| - A_k)^2 with the unnormalised forward FFT.
"""
import numpy as np
import pytest

from oracle import numpy_oracle
from tests import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def problem():
    s = scenes.raster_scene(scan=16, det=64, step=4, seed=4)
    amps = (s["amplitudes"] * 1.05).astype(np.float32)  # off the solution so the gradient is not ~0
    return s, amps


def _plan(cb, s, amps, precision):
    plan = cb.Plan(amps, s["positions"], s["object"].shape, s["probe"].shape, precision=precision)
    plan.set_state(s["object"], s["probe"])
    return plan


def test_fp64_adjoint_matches_the_cpu_gradient(problem):
    import cubokit_b200 as cb
    s, amps = problem
    plan = _plan(cb, s, amps, "fp64")
    loss, go, gp = plan.backward(recompute_exit_waves=True)
    l_ref, go_ref, gp_ref = numpy_oracle.loss_and_gradients(amps.astype(np.float64), s["positions"], s["object"],
                                                            s["probe"])
    assert abs(loss - l_ref) <= 1e-11 * l_ref
    assert np.max(np.abs(go - go_ref)) <= 1e-10 * np.max(np.abs(go_ref))
    assert np.max(np.abs(gp - gp_ref)) <= 1e-10 * np.max(np.abs(gp_ref))


def test_fp64_adjoint_matches_central_differences(problem):
    """64 seeded object pixels and 64 probe pixels, real and imaginary parts, h = 1e-6: max |fd - adjoint| over the
    largest sampled gradient component <= 1e-6."""
    import cubokit_b200 as cb
    s, amps = problem
    obj, probe = s["object"], s["probe"]
    plan = _plan(cb, s, amps, "fp64")
    _, go, gp = plan.backward(recompute_exit_waves=True)
    rng = np.random.default_rng(64)
    h = 1e-6

    def loss_at(o, p):
        plan.set_state(o, p)
        return plan.forward()

    for field, grad, which in ((obj, go, "object"), (probe, gp, "probe")):
        idx = [tuple(rng.integers(0, n) for n in field.shape) for _ in range(64)]
        fd, an = [], []
        for j in idx:
            for unit in (1.0, 1j):
                plus, minus = field.copy(), field.copy()
                plus[j] += unit * h
                minus[j] -= unit * h
                if which == "object":
                    d = (loss_at(plus, probe) - loss_at(minus, probe)) / (2 * h)
                else:
                    d = (loss_at(obj, plus) - loss_at(obj, minus)) / (2 * h)
                fd.append(d)
                an.append(grad[j].real if unit == 1.0 else grad[j].imag)
        fd, an = np.array(fd), np.array(an)
        gap = np.max(np.abs(fd - an)) / np.max(np.abs(an))
        assert gap <= 1e-6, (which, gap)


def test_fp32_adjoint_against_fp64(problem):
    import cubokit_b200 as cb
    s, amps = problem
    l64, go64, gp64 = _plan(cb, s, amps, "fp64").backward(recompute_exit_waves=True)
    l32, go32, gp32 = _plan(cb, s, amps, "fp32").backward(recompute_exit_waves=True)
    assert abs(l32 - l64) <= 1e-5 * l64
    assert np.max(np.abs(go32 - go64)) <= 1e-4 * np.max(np.abs(go64))
    assert np.max(np.abs(gp32 - gp64)) <= 1e-4 * np.max(np.abs(gp64))


def test_tape_and_recompute_agree_bitwise(problem):
    import cubokit_b200 as cb
    s, amps = problem
    plan = _plan(cb, s, amps, "fp32")
    loss = plan.forward()
    a = plan.backward(recompute_exit_waves=False)
    b = plan.backward(recompute_exit_waves=True)
    assert a[0] == b[0] == loss
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
