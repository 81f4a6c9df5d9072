"""ctypes binding of ``libcuboptycho.so`` (the C ABI in ``include/cubo_ptycho.h``).

Loading fails loudly: there is no CPU fallback.  If the library is missing it is built in-tree with nvcc first.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libcuboptycho.so"

OK, INVALID_INPUT, CANCELLED = 0, 1, 2
CUDA_ERROR, OUT_OF_MEMORY, DEVICE_TIMEOUT, NO_DEVICE, UNSUPPORTED = -1, -2, -3, -4, -5
FORM_FP32, FORM_SPLIT_BF16, FORM_FP64 = 0, 1, 2
ERRORS_SUPPLIED_AMPLITUDE_ENERGY, ERRORS_MEAN_INTENSITY = 0, 1
VARIANT_AUTO, VARIANT_GENERIC, VARIANT_GLOBAL = 0, 1, 2

PROGRESS_FN = C.CFUNCTYPE(None, C.c_int, C.c_int, C.c_void_p)


SHIFT_BILINEAR, SHIFT_CUBIC_SPLINE = 0, 1


class Problem(C.Structure):
    _fields_ = [
        ("rows", C.c_int), ("columns", C.c_int), ("object_rows", C.c_int), ("object_columns", C.c_int),
        ("count", C.c_int), ("amplitudes", C.POINTER(C.c_float)), ("position_rows", C.POINTER(C.c_double)),
        ("position_columns", C.POINTER(C.c_double)), ("amplitudes_on_device", C.c_int),
    ]


class Params(C.Structure):
    _fields_ = [
        ("iterations", C.c_int), ("step_size", C.c_double), ("normalization_minimum", C.c_double),
        ("fix_probe", C.c_int), ("pure_phase_object", C.c_int), ("constrain_object_amplitude", C.c_int),
        ("fix_probe_center_of_mass", C.c_int), ("constrain_probe_amplitude", C.c_int),
        ("probe_amplitude_relative_radius", C.c_double), ("probe_amplitude_relative_width", C.c_double),
        ("fix_probe_aperture", C.c_int), ("probe_support_mask", C.POINTER(C.c_ubyte)),
        ("error_normalization", C.c_int), ("mean_intensity", C.c_double), ("has_position_correction", C.c_int),
        ("form", C.c_int), ("cancel", C.POINTER(C.c_int)), ("progress", PROGRESS_FN), ("progress_user", C.c_void_p),
        ("variant", C.c_int), ("gather_tile", C.c_int),
        ("position_step_size", C.c_double), ("has_max_position_update_distance", C.c_int),
        ("max_position_update_distance", C.c_double), ("has_max_position_total_distance", C.c_int),
        ("max_position_total_distance", C.c_double), ("position_row_sampling", C.c_double),
        ("position_column_sampling", C.c_double), ("constrain_positions_center_of_mass", C.c_int),
        ("position_rows_out", C.POINTER(C.c_double)), ("position_columns_out", C.POINTER(C.c_double)),
        ("pass_shape", C.c_int),
    ]


class MixedParams(C.Structure):
    _fields_ = [("states", C.c_int), ("orthogonalize_probes", C.c_int), ("zero_pixel_error", C.c_int)]


ZERO_PIXEL_REFERENCE, ZERO_PIXEL_FINITE = 0, 1


class MultisliceParams(C.Structure):
    _fields_ = [("slices", C.c_int), ("slice_thicknesses", C.POINTER(C.c_double)), ("wavelength", C.c_double),
                ("row_sampling", C.c_double), ("column_sampling", C.c_double), ("identical_slices", C.c_int)]


# Every symbol the header declares, with its ctypes signature (restype, argtypes).
_dp = C.POINTER(C.c_double)
SIGNATURES = {
    "cubo_ptycho_params_default": (None, [C.POINTER(Params)]),
    "cubo_ptycho_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "cubo_ptycho_destroy": (C.c_int, [C.c_void_p]),
    "cubo_ptycho_last_error": (C.c_char_p, [C.c_void_p]),
    "cubo_ptycho_reconstruct": (C.c_int, [C.c_void_p, C.POINTER(Problem), C.POINTER(Params), _dp, _dp, _dp, _dp, _dp]),
    "cubo_ptycho_plan_create": (C.c_int, [C.c_void_p, C.POINTER(Problem), C.POINTER(Params), C.POINTER(C.c_void_p)]),
    "cubo_ptycho_plan_destroy": (C.c_int, [C.c_void_p]),
    "cubo_ptycho_plan_set_state": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp]),
    "cubo_ptycho_plan_get_state": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp]),
    "cubo_ptycho_plan_get_positions": (C.c_int, [C.c_void_p, _dp, _dp]),
    "cubo_ptycho_mixed_params_default": (None, [C.POINTER(MixedParams)]),
    "cubo_ptycho_mixed_reconstruct": (C.c_int, [C.c_void_p, C.POINTER(Problem), C.POINTER(Params),
                                                C.POINTER(MixedParams), _dp, _dp, _dp, _dp, _dp]),
    "cubo_ptycho_mixed_plan_create": (C.c_int, [C.c_void_p, C.POINTER(Problem), C.POINTER(Params),
                                                C.POINTER(MixedParams), C.POINTER(C.c_void_p)]),
    "cubo_ptycho_orthogonalize": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, _dp, _dp]),
    "cubo_ptycho_propagators": (C.c_int, [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, _dp, _dp,
                                          _dp]),
    "cubo_ptycho_multislice_reconstruct": (C.c_int, [C.c_void_p, C.POINTER(Problem), C.POINTER(Params),
                                                     C.POINTER(MultisliceParams), _dp, _dp, _dp, _dp, _dp]),
    "cubo_ptycho_multislice_plan_create": (C.c_int, [C.c_void_p, C.POINTER(Problem), C.POINTER(Params),
                                                     C.POINTER(MultisliceParams), C.POINTER(C.c_void_p)]),
    "cubo_ptycho_plan_iterate": (C.c_int, [C.c_void_p, C.c_int, _dp]),
    "cubo_ptycho_plan_enqueue": (C.c_int, [C.c_void_p, C.c_int]),
    "cubo_ptycho_plan_errors": (C.c_int, [C.c_void_p, C.c_int, _dp]),
    "cubo_ptycho_stream": (C.c_void_p, [C.c_void_p]),
    "cubo_ptycho_synchronize": (C.c_int, [C.c_void_p]),
    "cubo_ptycho_plan_set_timing": (C.c_int, [C.c_void_p, C.c_int]),
    "cubo_ptycho_plan_kernel_stats": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_char_p), _dp,
                                                C.POINTER(C.c_longlong), C.POINTER(C.c_int)]),
    "cubo_ptycho_plan_launch_count": (C.c_longlong, [C.c_void_p]),
    "cubo_ptycho_probe_build": (C.c_int, [C.c_void_p, C.c_int, C.c_int] + [C.c_double] * 9 + [C.c_int, _dp, _dp, _dp]),
    "cubo_ptycho_prepare_amplitudes": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, _dp, _dp, C.c_int,
                                                 C.c_void_p, _dp, _dp]),
    "cubo_ptycho_set_timing": (C.c_int, [C.c_void_p, C.c_int]),
    "cubo_ptycho_prepare_kernel_stats": (C.c_int, [C.c_void_p, _dp, C.POINTER(C.c_longlong)]),
    "cubo_ptycho_prepare_amplitudes_device": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, _dp, _dp,
                                                        C.c_int, C.c_void_p, _dp, _dp]),
    "cubo_ptycho_plan_forward": (C.c_int, [C.c_void_p, _dp]),
    "cubo_ptycho_plan_backward": (C.c_int, [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp, _dp]),
    "cubo_ptycho_batch_create": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(Problem), C.POINTER(Params),
                                           C.POINTER(C.c_void_p)]),
    "cubo_ptycho_batch_destroy": (C.c_int, [C.c_void_p]),
    "cubo_ptycho_batch_set_state": (C.c_int, [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp]),
    "cubo_ptycho_batch_get_state": (C.c_int, [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp]),
    "cubo_ptycho_batch_run": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "cubo_ptycho_batch_errors": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _dp]),
    "cubo_ptycho_batch_launches_per_iteration": (C.c_longlong, [C.c_void_p]),
    "cubo_ptycho_loss_fp32_noalloc": (C.c_int, [C.c_int] * 5 + [C.c_void_p] * 7),
    "cubo_ptycho_measure_peaks": (C.c_int, [C.c_void_p, _dp, _dp]),
    "cubo_ptycho_plan_enqueue_gradients": (C.c_int, [C.c_void_p]),
    "cubo_ptycho_plan_gradient_buffers": (C.c_int, [C.c_void_p] + [C.POINTER(C.c_void_p)] * 5 + [C.POINTER(C.c_int)]),
    "cubo_ptycho_plan_apply_gradients": (C.c_int, [C.c_void_p]),
}

_lib = None


def load(build_if_missing: bool = True):
    """The loaded library with every signature set.  Raises if it cannot be built or loaded."""
    global _lib
    if _lib is not None:
        return _lib
    if build_if_missing:
        from . import build as _build
        _build.build(quiet=True)
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing and could not be built; the CUDA path has no fallback")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
