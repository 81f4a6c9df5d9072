"""Runs the C++ mirror's parity programs on CuboKit's pins: tests/cpp/test_reconstruct.cpp on the main single-slice
pin, tests/cpp/run_engines.cpp on a mixed-state and a multislice pin."""
import subprocess

import numpy as np
import pytest

from tests import golden_cases as gc
from tests.test_cpp_api import build, build_engines

pytestmark = pytest.mark.gpu


def test_cpp_mirror_meets_the_main_pin(tmp_path):
    case = gc.engine_cases()[0]  # PtychographyTests.swift:48-60
    kw = case.kwargs
    R, C = case.probe.shape
    OR, OC = case.object.shape
    path = tmp_path / "case.bin"
    with open(path, "wb") as f:
        np.asarray([R, C, OR, OC, len(case.positions), kw["iterations"]], np.int32).tofile(f)
        np.asarray([kw["step_size"], kw["normalization_minimum"], kw["mean_intensity"]], np.float64).tofile(f)
        for a in (case.amplitudes.ravel(), case.positions.ravel(), case.object.real.ravel(), case.object.imag.ravel(),
                  case.probe.real.ravel(), case.probe.imag.ravel(), case.expect_object.real.ravel(),
                  case.expect_object.imag.ravel(), case.expect_probe.real.ravel(), case.expect_probe.imag.ravel(),
                  case.expect_errors.ravel()):
            np.asarray(a, np.float64).tofile(f)
    exe = build()
    res = subprocess.run([str(exe), str(path)], capture_output=True, text=True, timeout=300)
    print(res.stdout, res.stderr)
    assert res.returncode == 0, res.stdout + res.stderr


def _ints(f, values):
    np.asarray(values, np.int32).tofile(f)


def _doubles(f, *arrays):
    for a in arrays:
        np.asarray(a, np.float64).ravel().tofile(f)


def _run(which, write, tmp_path):
    src, dst = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(src, "wb") as f:
        write(f)
    res = subprocess.run([str(build_engines()), which, str(src), str(dst)], capture_output=True, text=True,
                         timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    return np.fromfile(dst, np.float64)


def test_cpp_mixedstate_meets_the_pin(tmp_path):
    """``EngineTests.swift:86-110``, case "two" (two states, orthogonalised), through MixedstatePtychography."""
    name, kw, (obj, probes, errors), _ = gc.mixed_cases()[0]
    S, R, C = kw["probes"].shape
    OR, OC = kw["obj"].shape
    P = len(kw["positions"])

    def write(f):
        _ints(f, [R, C, OR, OC, P, S, kw["iterations"], kw["fix_probe"], kw["pure_phase_object"],
                  kw["fix_probe_center_of_mass"], kw["constrain_probe_amplitude"], kw["orthogonalize_probes"]])
        _doubles(f, [kw["step_size"], kw["normalization_minimum"], kw["mean_intensity"],
                     kw["probe_amplitude_relative_radius"], kw["probe_amplitude_relative_width"]],
                 kw["amplitudes"], kw["positions"], kw["obj"].real, kw["obj"].imag, kw["probes"].real,
                 kw["probes"].imag)

    out = _run("mixed", write, tmp_path)
    o, n = OR * OC, S * R * C
    got_obj = (out[:o] + 1j * out[o:2 * o]).reshape(OR, OC)
    got_probes = (out[2 * o:2 * o + n] + 1j * out[2 * o + n:2 * o + 2 * n]).reshape(S, R, C)
    got_errors = out[2 * o + 2 * n:]
    assert max(gc.complex_gap(got_obj, obj), gc.gap(got_errors, errors),
               gc.complex_gap(gc.align_phases(got_probes, probes), probes)) < 2e-6, name


def test_cpp_multislice_meets_the_pin(tmp_path):
    """``EngineTests.swift:205-228``, case "threeConstraints" (three slices, centre of mass and amplitude
    constraint), through MultislicePtychography."""
    name, kw, (obj, probe, errors) = gc.multislice_cases()[1]
    L, OR, OC = kw["obj"].shape
    R, C = kw["probe"].shape
    P = len(kw["positions"])

    def write(f):
        _ints(f, [R, C, OR, OC, P, L, kw["iterations"], kw["fix_probe"], kw["pure_phase_object"],
                  kw["identical_slices"], kw["fix_probe_center_of_mass"], kw["constrain_probe_amplitude"]])
        _doubles(f, [kw["step_size"], kw["normalization_minimum"], kw["mean_intensity"],
                     kw["probe_amplitude_relative_radius"], kw["probe_amplitude_relative_width"], kw["wavelength"],
                     kw["row_sampling"], kw["column_sampling"]],
                 kw["slice_thicknesses"], kw["amplitudes"], kw["positions"], kw["obj"].real, kw["obj"].imag,
                 kw["probe"].real, kw["probe"].imag)

    out = _run("multislice", write, tmp_path)
    o, n = L * OR * OC, R * C
    got_obj = (out[:o] + 1j * out[o:2 * o]).reshape(L, OR, OC)
    got_probe = (out[2 * o:2 * o + n] + 1j * out[2 * o + n:2 * o + 2 * n]).reshape(R, C)
    got_errors = out[2 * o + 2 * n:]
    assert max(gc.complex_gap(got_obj, obj), gc.complex_gap(got_probe, probe), gc.gap(got_errors, errors)) < 2e-6, name
