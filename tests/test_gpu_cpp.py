"""Runs the C++ parity program (tests/cpp/test_reconstruct.cpp) on CuboKit's main single-slice pin."""
import subprocess

import numpy as np
import pytest

from tests import golden_cases as gc
from tests.test_cpp_api import build

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
