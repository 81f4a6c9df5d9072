"""CPU-side checks of the C ABI: the library builds for sm_100a, loads, and exports every symbol the header declares.

No compute call is made here (there is no GPU in this environment); the one device query checks that a context refuses
cleanly when no device is present.
"""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "cubo_ptycho.h").read_text()
    return sorted(set(re.findall(r"CUBO_PTYCHO_API\s+[\w\s\*]+?\b(cubo_ptycho_\w+)\s*\(", text)))


def test_header_declares_the_entry_points():
    names = declared_symbols()
    for expected in ("cubo_ptycho_create", "cubo_ptycho_reconstruct", "cubo_ptycho_plan_create",
                     "cubo_ptycho_plan_iterate", "cubo_ptycho_probe_build"):
        assert expected in names


def test_library_exports_every_declared_symbol():
    from cubokit_b200 import _lib
    lib = _lib.load()
    for name in declared_symbols():
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"
    assert set(_lib.SIGNATURES) == set(declared_symbols())


def test_struct_layouts_match_the_header():
    """The ctypes mirrors must have the header's field order; a C compiler gives the reference layout."""
    import subprocess
    import tempfile
    from cubokit_b200 import _lib
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "cubo_ptycho.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(cubo_ptycho_problem), sizeof(cubo_ptycho_params),
         offsetof(cubo_ptycho_params, form), offsetof(cubo_ptycho_params, progress_user),
         offsetof(cubo_ptycho_params, max_position_total_distance),
         offsetof(cubo_ptycho_params, position_columns_out), sizeof(cubo_ptycho_mixed_params),
         sizeof(cubo_ptycho_multislice_params), offsetof(cubo_ptycho_multislice_params, identical_slices),
         offsetof(cubo_ptycho_params, pass_shape));
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        (Path(d) / "t.c").write_text(src)
        gcc = "/usr/bin/gcc" if Path("/usr/bin/gcc").exists() else "gcc"
        subprocess.run([gcc, "-I", str(ROOT / "include"), str(Path(d) / "t.c"), "-o", str(Path(d) / "t")], check=True)
        out = subprocess.run([str(Path(d) / "t")], capture_output=True, text=True, check=True).stdout.split()
    assert int(out[0]) == C.sizeof(_lib.Problem)
    assert int(out[1]) == C.sizeof(_lib.Params)
    assert int(out[2]) == _lib.Params.form.offset
    assert int(out[3]) == _lib.Params.progress_user.offset
    assert int(out[4]) == _lib.Params.max_position_total_distance.offset
    assert int(out[5]) == _lib.Params.position_columns_out.offset
    assert int(out[9]) == _lib.Params.pass_shape.offset
    assert int(out[6]) == C.sizeof(_lib.MixedParams)
    assert int(out[7]) == C.sizeof(_lib.MultisliceParams)
    assert int(out[8]) == _lib.MultisliceParams.identical_slices.offset


def test_propagators_on_the_host():
    """``MultislicePtychography.propagators`` (host arithmetic, no device): the Fresnel kernels equal the oracle's
    restatement, and invalid samplings, wavelengths and thicknesses are refused (``PtychographyEngines.swift:427-433``)."""
    import cubokit_b200
    from oracle import numpy_oracle as no
    args = (12, 10, 0.45, 0.5, 0.0197, [40.0, 55.0, 0.0])
    got = cubokit_b200.MultislicePtychography.propagators(*args)
    want = no.propagators(*args)
    assert got.shape == (3, 12, 10)
    assert np.max(np.abs(got - want)) < 1e-12
    bad = [(1, 10, 0.45, 0.5, 0.0197, [1.0]), (12, 10, 0.0, 0.5, 0.0197, [1.0]),
           (12, 10, 0.45, np.inf, 0.0197, [1.0]), (12, 10, 0.45, 0.5, -1.0, [1.0]),
           (12, 10, 0.45, 0.5, 0.0197, []), (12, 10, 0.45, 0.5, 0.0197, [np.nan])]
    for b in bad:
        with pytest.raises(cubokit_b200.PtychographyError):
            cubokit_b200.MultislicePtychography.propagators(*b)


def test_context_without_a_device_is_refused_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    import cubokit_b200
    with pytest.raises(cubokit_b200.DeviceError) as e:
        cubokit_b200.Context(0)
    assert e.value.status == -4  # CUBO_PTYCHO_NO_DEVICE


def test_params_default_is_the_reference_default():
    """``Ptychography.swift:220-232``."""
    from cubokit_b200 import _lib
    lib = _lib.load()
    p = _lib.Params()
    lib.cubo_ptycho_params_default(C.byref(p))
    assert (p.iterations, p.step_size, p.normalization_minimum) == (8, 0.5, 1.0)
    assert (p.fix_probe, p.pure_phase_object, p.constrain_object_amplitude) == (0, 0, 1)
    assert (p.probe_amplitude_relative_radius, p.probe_amplitude_relative_width) == (0.5, 0.05)
    assert p.form == _lib.FORM_FP32 and p.error_normalization == _lib.ERRORS_SUPPLIED_AMPLITUDE_ENERGY
