"""ctypes binding of the C oracle (``oracle/libptycho_oracle.so``) — TEST INFRASTRUCTURE ONLY.

Only tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU legs load this.  See ``ptycho_oracle.h``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "libptycho_oracle.so"


class OracleParams(C.Structure):
    _fields_ = [
        ("iterations", C.c_int),
        ("step_size", C.c_double),
        ("normalization_minimum", C.c_double),
        ("fix_probe", C.c_int),
        ("pure_phase_object", C.c_int),
        ("constrain_object_amplitude", C.c_int),
        ("fix_probe_center_of_mass", C.c_int),
        ("constrain_probe_amplitude", C.c_int),
        ("probe_amplitude_relative_radius", C.c_double),
        ("probe_amplitude_relative_width", C.c_double),
        ("fix_probe_aperture", C.c_int),
        ("probe_support_mask", C.POINTER(C.c_ubyte)),
        ("error_normalization", C.c_int),
        ("mean_intensity", C.c_double),
        ("threads", C.c_int),
        ("single_shift_fft", C.c_int),
    ]


def build():
    """Compile the oracle library with its Makefile (gcc)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        _lib = C.CDLL(str(LIB))
        d = C.POINTER(C.c_double)
        _lib.oracle_reconstruct.argtypes = [C.POINTER(OracleParams), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                            d, d, d, d, d, d, d, d]
        _lib.oracle_reconstruct_single.argtypes = [C.POINTER(OracleParams), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                                   C.POINTER(C.c_float), d, d, d, d, d, d, d]
        _lib.oracle_probe_build.argtypes = [C.c_int, C.c_int] + [C.c_double] * 9 + [C.c_int, d, d, d]
        _lib.oracle_fft2.argtypes = [C.c_int, C.c_int, d, d, C.c_int]
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def probe_build(rows, columns, row_sampling, column_sampling, wavelength, cutoff, rolloff=0.002, defocus=0.0,
                astigmatism=0.0, astigmatism_angle=0.0, spherical_aberration=0.0, terms=None):
    """``PtychographyProbe.build``; ``terms`` rows are ``(radialOrder, angularOrder, sine, coefficient)``."""
    t = np.ascontiguousarray(np.zeros((0, 4)) if terms is None else np.asarray(terms, np.float64).reshape(-1, 4))
    re = np.zeros(rows * columns)
    im = np.zeros(rows * columns)
    rc = lib().oracle_probe_build(rows, columns, row_sampling, column_sampling, wavelength, cutoff, rolloff, defocus,
                                  astigmatism, astigmatism_angle, spherical_aberration, len(t), _dp(t), _dp(re), _dp(im))
    if rc != 0:
        raise ValueError("invalid probe parameters")
    return (re + 1j * im).reshape(rows, columns)


def fft2(z, inverse=False):
    z = np.asarray(z, np.complex128)
    re = np.ascontiguousarray(z.real)
    im = np.ascontiguousarray(z.imag)
    lib().oracle_fft2(z.shape[0], z.shape[1], _dp(re), _dp(im), 1 if inverse else 0)
    return re + 1j * im


def reconstruct(amplitudes, positions, obj, probe, iterations=8, step_size=0.5, normalization_minimum=1.0,
                fix_probe=False, pure_phase_object=False, constrain_object_amplitude=True,
                fix_probe_center_of_mass=False, constrain_probe_amplitude=False,
                probe_amplitude_relative_radius=0.5, probe_amplitude_relative_width=0.05, fix_probe_aperture=False,
                probe_support_mask=None, error_normalization="suppliedAmplitudeEnergy", mean_intensity=0.0,
                threads=1, single=False, shift_every_position=True):
    """The C oracle's Double path (``single=False``) or Float32 path (``single=True``).  Returns (object, probe, errors).

    Raises ``ValueError`` on the reference's refusals.
    """
    obj = np.asarray(obj, np.complex128)
    probe = np.asarray(probe, np.complex128)
    rows, columns = probe.shape
    object_rows, object_columns = obj.shape
    positions = np.asarray(positions, np.float64).reshape(-1, 2)
    count = len(positions)
    mask = None
    if probe_support_mask is not None:
        mask = np.ascontiguousarray(np.asarray(probe_support_mask, bool).reshape(-1).astype(np.uint8))
    p = OracleParams(iterations, step_size, normalization_minimum, int(fix_probe), int(pure_phase_object),
                     int(constrain_object_amplitude), int(fix_probe_center_of_mass), int(constrain_probe_amplitude),
                     probe_amplitude_relative_radius, probe_amplitude_relative_width, int(fix_probe_aperture),
                     mask.ctypes.data_as(C.POINTER(C.c_ubyte)) if mask is not None else None,
                     1 if error_normalization == "meanIntensity" else 0, float(mean_intensity or 0.0), int(threads),
                     1 if shift_every_position else 0)
    ore = np.ascontiguousarray(obj.real.ravel())
    oim = np.ascontiguousarray(obj.imag.ravel())
    pre = np.ascontiguousarray(probe.real.ravel())
    pim = np.ascontiguousarray(probe.imag.ravel())
    pr = np.ascontiguousarray(positions[:, 0])
    pc = np.ascontiguousarray(positions[:, 1])
    errors = np.zeros(max(iterations, 1))
    if np.asarray(amplitudes).size != count * rows * columns:
        raise ValueError("invalid input")
    if single:
        a = np.ascontiguousarray(np.asarray(amplitudes, np.float32).ravel())
        rc = lib().oracle_reconstruct_single(C.byref(p), rows, columns, object_rows, object_columns, count,
                                             a.ctypes.data_as(C.POINTER(C.c_float)), _dp(pr), _dp(pc), _dp(ore),
                                             _dp(oim), _dp(pre), _dp(pim), _dp(errors))
    else:
        a = np.ascontiguousarray(np.asarray(amplitudes, np.float64).ravel())
        rc = lib().oracle_reconstruct(C.byref(p), rows, columns, object_rows, object_columns, count, _dp(a), _dp(pr),
                                      _dp(pc), _dp(ore), _dp(oim), _dp(pre), _dp(pim), _dp(errors))
    if rc != 0:
        raise ValueError("invalid input")
    return ((ore + 1j * oim).reshape(object_rows, object_columns), (pre + 1j * pim).reshape(rows, columns),
            errors[:iterations])


def host_cores():
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
