"""Python mirror of CuboPtycho's single-slice API over the B200 engine.

``SingleslicePtychography.reconstruct`` here takes the parameters of the Swift call of the same name
(``Sources/CuboPtycho/Ptychography.swift:218-234``) in snake case, with the same defaults, refusals
(``PtychographyError`` for ``invalidInput``) and ``CancellationError``; ``precision`` picks the GPU form.  Every
call goes through the C ABI of ``include/cubo_ptycho.h``; nothing here computes on the CPU.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Callable, Optional, Sequence

import numpy as np

from . import _lib as L


class PtychographyError(ValueError):
    """``PtychographyError.invalidInput`` (``Ptychography.swift:24-27``)."""


class CancellationError(Exception):
    """Swift's ``CancellationError`` (``PtychographySingle.swift:222-224``)."""


class DeviceError(RuntimeError):
    """A device failure the CPU path cannot have (CUDA error, out of memory, device wait timed out, no device)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"status {status}: {message}")
        self.status = status


class UnsupportedError(DeviceError):
    pass


FORMS = {"fp32": L.FORM_FP32, "split_bf16": L.FORM_SPLIT_BF16, "fp64": L.FORM_FP64}


def _raise(status: int, message: str):
    if status == L.INVALID_INPUT:
        raise PtychographyError(message)
    if status == L.CANCELLED:
        raise CancellationError(message)
    if status == L.UNSUPPORTED:
        raise UnsupportedError(status, message)
    raise DeviceError(status, message)


class Context:
    """A device context (``cubo_ptycho_create``): a CUDA stream and the engine's scratch on one GPU."""

    def __init__(self, device: int = 0):
        self.lib = L.load()
        h = C.c_void_p()
        st = self.lib.cubo_ptycho_create(device, C.byref(h))
        if st != L.OK:
            _raise(st, "cubo_ptycho_create failed")
        self.handle = h
        self.device = device

    def check(self, status: int):
        if status != L.OK:
            _raise(status, self.lib.cubo_ptycho_last_error(self.handle).decode())

    @property
    def stream(self) -> int:
        return self.lib.cubo_ptycho_stream(self.handle)

    def synchronize(self):
        self.check(self.lib.cubo_ptycho_synchronize(self.handle))

    def set_timing(self, enabled: bool):
        """CUDA events around each preprocessing kernel launch (clears the totals)."""
        self.check(self.lib.cubo_ptycho_set_timing(self.handle, 1 if enabled else 0))

    def prepare_kernel_stats(self) -> tuple[float, int]:
        """(device milliseconds, launches) of the preprocessing kernel since timing was switched on."""
        ms, launches = C.c_double(), C.c_longlong()
        self.check(self.lib.cubo_ptycho_prepare_kernel_stats(self.handle, C.byref(ms), C.byref(launches)))
        return ms.value, launches.value

    def measure_peaks(self):
        """``(fp32_tflops, fp64_tflops)``: this device's CUDA-core FMA rates (``cubo_ptycho_measure_peaks``)."""
        f32, f64 = C.c_double(0), C.c_double(0)
        self.check(self.lib.cubo_ptycho_measure_peaks(self.handle, C.byref(f32), C.byref(f64)))
        return f32.value, f64.value

    def close(self):
        if getattr(self, "handle", None):
            self.lib.cubo_ptycho_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_contexts: dict[int, Context] = {}


def context(device: int = 0) -> Context:
    if device not in _default_contexts:
        _default_contexts[device] = Context(device)
    return _default_contexts[device]


@dataclass
class PtychographyPositionCorrection:
    """``PtychographyPositionCorrection`` (``Ptychography.swift:53-85``): the step, the two distance limits in Å
    (``None`` = unlimited; they need both samplings, Å per pixel) and the centre-of-mass constraint.  Runs with
    ``precision="fp64"`` (the reference's Double path; its Float path refuses it)."""
    step_size: float = 0.5
    max_update_distance: Optional[float] = None
    max_total_distance: Optional[float] = None
    row_sampling: Optional[float] = None
    column_sampling: Optional[float] = None
    constrain_center_of_mass: bool = False


@dataclass
class Result:
    """``SingleslicePtychography.Result`` (``Ptychography.swift:179-188``)."""
    object: np.ndarray
    probe: np.ndarray
    errors: np.ndarray
    positions: np.ndarray


def _split(z, shape=None):
    z = np.asarray(z)
    if shape is not None and z.size != int(np.prod(shape)):
        raise PtychographyError("array size")
    re = np.ascontiguousarray(np.real(z), dtype=np.float64).ravel()
    im = np.ascontiguousarray(np.imag(z), dtype=np.float64).ravel()
    return re, im


def _ptr(a, t=C.c_double):
    return a.ctypes.data_as(C.POINTER(t))


def _torch():
    import torch
    return torch


def _is_cuda_tensor(x):
    mod = type(x).__module__
    return mod.startswith("torch") and getattr(x, "is_cuda", False)


class _Inputs:
    """Keeps the ctypes structures and the arrays they point into alive for one call."""

    def __init__(self, amplitudes, positions, object_shape, probe_shape, iterations, step_size, normalization_minimum,
                 fix_probe, pure_phase_object, constrain_object_amplitude, fix_probe_center_of_mass,
                 constrain_probe_amplitude, probe_amplitude_relative_radius, probe_amplitude_relative_width,
                 fix_probe_aperture, probe_support_mask, error_normalization, position_correction, precision,
                 variant="auto", gather_tile=0, pass_shape=0):
        rows, columns = probe_shape
        positions = np.asarray(positions, np.float64).reshape(-1, 2) if np.size(positions) else np.zeros((0, 2))
        count = len(positions)
        on_device = _is_cuda_tensor(amplitudes)
        if on_device:  # a CUDA tensor (e.g. PtychographyPreparation.amplitudes(..., keep_on_device=True)): no upload
            if amplitudes.dtype != _torch().float32 or not amplitudes.is_contiguous():
                raise PtychographyError("device amplitudes must be a contiguous float32 tensor")
            size = amplitudes.numel()
            self.amplitudes = amplitudes
            amp_ptr = C.cast(C.c_void_p(amplitudes.data_ptr()), C.POINTER(C.c_float))
        else:
            amps = np.asarray(amplitudes)
            size = amps.size
            self.amplitudes = np.ascontiguousarray(amps, dtype=np.float32).ravel()
            amp_ptr = _ptr(self.amplitudes, C.c_float)
        if size != count * rows * columns:
            raise PtychographyError("amplitudes.count != positions * probe pixels")  # Ptychography.swift:248
        self.rows_ = np.ascontiguousarray(positions[:, 0])
        self.cols_ = np.ascontiguousarray(positions[:, 1])
        self.problem = L.Problem(rows, columns, object_shape[0], object_shape[1], count, amp_ptr, _ptr(self.rows_),
                                 _ptr(self.cols_), 1 if on_device else 0)
        self.params = L.Params()
        p = self.params
        p.iterations = int(iterations)
        p.step_size = float(step_size)
        p.normalization_minimum = float(normalization_minimum)
        p.fix_probe = int(bool(fix_probe))
        p.pure_phase_object = int(bool(pure_phase_object))
        p.constrain_object_amplitude = int(bool(constrain_object_amplitude))
        p.fix_probe_center_of_mass = int(bool(fix_probe_center_of_mass))
        p.constrain_probe_amplitude = int(bool(constrain_probe_amplitude))
        p.probe_amplitude_relative_radius = float(probe_amplitude_relative_radius)
        p.probe_amplitude_relative_width = float(probe_amplitude_relative_width)
        p.fix_probe_aperture = int(bool(fix_probe_aperture))
        self.mask = None
        if probe_support_mask is not None:
            m = np.asarray(probe_support_mask, bool).ravel()
            if m.size != rows * columns:
                raise PtychographyError("probeSupportMask.count != probe pixels")  # Ptychography.swift:256
            self.mask = np.ascontiguousarray(m.astype(np.uint8))
            p.probe_support_mask = _ptr(self.mask, C.c_ubyte)
        if isinstance(error_normalization, tuple):
            kind, mean = error_normalization
            if kind != "meanIntensity":
                raise PtychographyError("error normalisation")
            p.error_normalization = L.ERRORS_MEAN_INTENSITY
            p.mean_intensity = float(mean)
        elif error_normalization == "suppliedAmplitudeEnergy":
            p.error_normalization = L.ERRORS_SUPPLIED_AMPLITUDE_ENERGY
        else:
            raise PtychographyError("error normalisation")
        p.has_position_correction = 0 if position_correction is None else 1
        p.position_step_size = 0.5
        p.position_row_sampling = p.position_column_sampling = float("nan")
        if position_correction is not None:
            pc = position_correction
            p.position_step_size = float(pc.step_size)
            p.has_max_position_update_distance = int(pc.max_update_distance is not None)
            p.max_position_update_distance = float(pc.max_update_distance or 0.0)
            p.has_max_position_total_distance = int(pc.max_total_distance is not None)
            p.max_position_total_distance = float(pc.max_total_distance or 0.0)
            p.position_row_sampling = float("nan") if pc.row_sampling is None else float(pc.row_sampling)
            p.position_column_sampling = float("nan") if pc.column_sampling is None else float(pc.column_sampling)
            p.constrain_positions_center_of_mass = int(bool(pc.constrain_center_of_mass))
        self.positions_out = (np.zeros(count), np.zeros(count))
        p.position_rows_out = _ptr(self.positions_out[0])
        p.position_columns_out = _ptr(self.positions_out[1])
        if precision not in FORMS:
            raise PtychographyError(f"precision {precision!r}")
        p.form = FORMS[precision]
        variants = {"auto": L.VARIANT_AUTO, "generic": L.VARIANT_GENERIC, "global": L.VARIANT_GLOBAL}
        if variant not in variants:
            raise PtychographyError(f"variant {variant!r}")
        p.variant = variants[variant]
        if gather_tile not in (0, 1, 2, 3):
            raise PtychographyError(f"gather_tile {gather_tile!r}")
        p.gather_tile = int(gather_tile)
        if pass_shape not in (0, 1, 2, 3):
            raise PtychographyError(f"pass_shape {pass_shape!r}")
        p.pass_shape = int(pass_shape)
        self.cancel_flag = C.c_int(0)
        self.count = count


class SingleslicePtychography:
    """``SingleslicePtychography`` (``Ptychography.swift:176-407``) on the GPU."""

    Result = Result

    @staticmethod
    def reconstruct(amplitudes, positions, object, probe, iterations: int = 8, step_size: float = 0.5,
                    normalization_minimum: float = 1.0, fix_probe: bool = False, pure_phase_object: bool = False,
                    constrain_object_amplitude: bool = True, fix_probe_center_of_mass: bool = False,
                    constrain_probe_amplitude: bool = False, probe_amplitude_relative_radius: float = 0.5,
                    probe_amplitude_relative_width: float = 0.05, fix_probe_aperture: bool = False,
                    probe_support_mask=None, error_normalization="suppliedAmplitudeEnergy",
                    position_correction=None, precision: str = "fp32",
                    is_cancelled: Optional[Callable[[], bool]] = None,
                    progress: Optional[Callable[[int, int], None]] = None, device: int = 0,
                    variant: str = "auto", gather_tile: int = 0) -> Result:
        """Reconstructs from corner-centred amplitudes ``[position][row][column]``; see ``include/cubo_ptycho.h``.

        ``object`` and ``probe`` are complex 2-D arrays (``PtychographyArray``); ``positions`` is ``(P, 2)`` rows and
        columns in object pixels.  ``error_normalization`` is ``"suppliedAmplitudeEnergy"`` or
        ``("meanIntensity", m)``.  ``precision`` is ``"fp32"``, ``"split_bf16"`` (128 x 128 detectors) or ``"fp64"``;
        FP32 and FP64 take detectors with sides up to 4096.  ``variant`` picks the position-pass kernel:
        ``"auto"`` (the specialised one for the detector size), ``"generic"`` (the any-size shared-memory transform)
        or ``"global"`` (the pass through global memory that detectors too large for one CTA use).
        ``is_cancelled`` is polled before every iteration and raises ``CancellationError``; ``progress(completed,
        total)`` runs after each iteration.
        """
        obj = np.asarray(object)
        prb = np.asarray(probe)
        if obj.ndim != 2 or prb.ndim != 2:
            raise PtychographyError("object and probe must be 2-D")
        ctx = context(device)
        inp = _Inputs(amplitudes, positions, obj.shape, prb.shape, iterations, step_size, normalization_minimum,
                      fix_probe, pure_phase_object, constrain_object_amplitude, fix_probe_center_of_mass,
                      constrain_probe_amplitude, probe_amplitude_relative_radius, probe_amplitude_relative_width,
                      fix_probe_aperture, probe_support_mask, error_normalization, position_correction, precision,
                      variant, gather_tile)
        if is_cancelled is not None and is_cancelled():
            raise CancellationError("cancelled")
        cb = None
        if is_cancelled is not None or progress is not None:
            def _progress(done, total, _user):
                if progress is not None:
                    progress(done, total)
                if is_cancelled is not None and is_cancelled():
                    inp.cancel_flag.value = 1
            cb = L.PROGRESS_FN(_progress)
            inp.params.progress = cb
            inp.params.cancel = C.pointer(inp.cancel_flag)
        ore, oim = _split(obj)
        pre, pim = _split(prb)
        errors = np.zeros(max(int(iterations), 1))
        st = ctx.lib.cubo_ptycho_reconstruct(ctx.handle, C.byref(inp.problem), C.byref(inp.params), _ptr(ore),
                                             _ptr(oim), _ptr(pre), _ptr(pim), _ptr(errors))
        ctx.check(st)
        pos = np.column_stack(inp.positions_out) if inp.count else np.zeros((0, 2))
        return Result((ore + 1j * oim).reshape(obj.shape), (pre + 1j * pim).reshape(prb.shape),
                      errors[: int(iterations)].copy(), pos)


@dataclass
class MixedstateResult:
    """``MixedstatePtychography.Result`` (``PtychographyEngines.swift:126-134``)."""
    object: np.ndarray
    probes: np.ndarray  # (states, rows, columns)
    errors: np.ndarray


class MixedstatePtychography:
    """``MixedstatePtychography`` (``PtychographyEngines.swift:121-298``) on the GPU, FP64: several incoherent probe
    states on one object; see ``cubo_ptycho_mixed_reconstruct`` in ``include/cubo_ptycho.h``."""

    Result = MixedstateResult

    @staticmethod
    def reconstruct(amplitudes, positions, object, probes, iterations: int = 8, step_size: float = 0.5,
                    normalization_minimum: float = 1.0, fix_probe: bool = False, pure_phase_object: bool = False,
                    fix_probe_center_of_mass: bool = False, constrain_probe_amplitude: bool = False,
                    probe_amplitude_relative_radius: float = 0.5, probe_amplitude_relative_width: float = 0.05,
                    orthogonalize_probes: bool = True, fix_probe_aperture: bool = False, probe_support_mask=None,
                    error_normalization="suppliedAmplitudeEnergy", zero_far_field_pixel_error: str = "reference",
                    device: int = 0) -> MixedstateResult:
        """``probes`` is ``(states, rows, columns)`` complex (``PtychographyStack``); ``zero_far_field_pixel_error``
        is ``"reference"`` (an infinite error term, py4DSTEM) or ``"finite"``."""
        obj = np.asarray(object)
        prb = np.asarray(probes)
        if obj.ndim != 2 or prb.ndim != 3:
            raise PtychographyError("object must be 2-D and probes (states, rows, columns)")
        if zero_far_field_pixel_error not in ("reference", "finite"):
            raise PtychographyError(f"zero_far_field_pixel_error {zero_far_field_pixel_error!r}")
        ctx = context(device)
        inp = _Inputs(amplitudes, positions, obj.shape, prb.shape[1:], iterations, step_size, normalization_minimum,
                      fix_probe, pure_phase_object, True, fix_probe_center_of_mass, constrain_probe_amplitude,
                      probe_amplitude_relative_radius, probe_amplitude_relative_width, fix_probe_aperture,
                      probe_support_mask, error_normalization, None, "fp64")
        mixed = L.MixedParams()
        ctx.lib.cubo_ptycho_mixed_params_default(C.byref(mixed))
        mixed.states = int(prb.shape[0])
        mixed.orthogonalize_probes = int(bool(orthogonalize_probes))
        mixed.zero_pixel_error = L.ZERO_PIXEL_REFERENCE if zero_far_field_pixel_error == "reference" \
            else L.ZERO_PIXEL_FINITE
        ore, oim = _split(obj)
        pre, pim = _split(prb)
        errors = np.zeros(max(int(iterations), 1))
        ctx.check(ctx.lib.cubo_ptycho_mixed_reconstruct(ctx.handle, C.byref(inp.problem), C.byref(inp.params),
                                                        C.byref(mixed), _ptr(ore), _ptr(oim), _ptr(pre), _ptr(pim),
                                                        _ptr(errors)))
        return MixedstateResult((ore + 1j * oim).reshape(obj.shape), (pre + 1j * pim).reshape(prb.shape),
                                errors[: int(iterations)].copy())

    @staticmethod
    def orthogonalize(probes, device: int = 0) -> np.ndarray:
        """``MixedstatePtychography.orthogonalize`` on the device: the eigenvectors of the states' Gram matrix, by
        decreasing intensity (each state's overall phase is free)."""
        prb = np.asarray(probes)
        if prb.ndim != 3:
            raise PtychographyError("probes must be (states, rows, columns)")
        ctx = context(device)
        re, im = _split(prb)
        ctx.check(ctx.lib.cubo_ptycho_orthogonalize(ctx.handle, prb.shape[0], prb.shape[1], prb.shape[2], _ptr(re),
                                                    _ptr(im)))
        return (re + 1j * im).reshape(prb.shape)

    @staticmethod
    def initial_probes(first, count: int, seed: int) -> np.ndarray:
        """``MixedstatePtychography.initialProbes`` (``PtychographyEngines.swift:270-298``), host-side set-up: state 0 is
        ``first``; each further state is the previous one times ``exp(-2 pi i ((u - 1/2) f_row + (v - 1/2) f_col))``
        with u, v drawn from NumPy's legacy ``RandomState(seed)`` (what the reference's generator reproduces)."""
        if not (0 < count < 4096):
            raise PtychographyError("count")
        first = np.asarray(first, np.complex128)
        rows, columns = first.shape
        rng = np.random.RandomState(seed)
        f = lambda n: np.where(np.arange(n) < (n + 1) // 2, np.arange(n), np.arange(n) - n) / n
        fr, fc = f(rows), f(columns)
        out = [first]
        for _ in range(1, count):
            u, v = rng.rand(), rng.rand()
            phase = -2 * np.pi * (u - 0.5) * fr[:, None] - 2 * np.pi * (v - 0.5) * fc[None, :]
            out.append(out[-1] * (np.cos(phase) + 1j * np.sin(phase)))
        return np.stack(out)


@dataclass
class MultisliceResult:
    """``MultislicePtychography.Result`` (``PtychographyEngines.swift:460-466``)."""
    object: np.ndarray  # (slices, rows, columns), entrance first
    probe: np.ndarray
    errors: np.ndarray


def _multislice_params(slices, slice_thicknesses, wavelength, row_sampling, column_sampling, identical_slices):
    """The ``cubo_ptycho_multislice_params`` of a call and the thickness array it points into (kept alive by the
    caller)."""
    thick = np.ascontiguousarray(np.asarray(slice_thicknesses, np.float64).ravel())
    if len(thick) != int(slices) - 1:
        raise PtychographyError("sliceThicknesses.count != slices - 1")  # PtychographyEngines.swift:477
    m = L.MultisliceParams()
    m.slices = int(slices)
    m.slice_thicknesses = _ptr(thick) if len(thick) else None
    m.wavelength = float(wavelength)
    m.row_sampling = float(row_sampling)
    m.column_sampling = float(column_sampling)
    m.identical_slices = int(bool(identical_slices))
    return m, thick


class MultislicePtychography:
    """``MultislicePtychography`` (``PtychographyEngines.swift:420-588``) on the GPU, FP64: a stack of object slices
    with Fresnel propagation between them; see ``cubo_ptycho_multislice_reconstruct`` in ``include/cubo_ptycho.h``."""

    Result = MultisliceResult

    @staticmethod
    def propagators(rows: int, columns: int, row_sampling: float, column_sampling: float, wavelength: float,
                    slice_thicknesses) -> np.ndarray:
        """``MultislicePtychography.propagators``: one ``(rows, columns)`` Fresnel kernel
        ``exp(-i pi lambda dz (kr^2 + kc^2))`` per thickness (host arithmetic; no device needed)."""
        thick = np.ascontiguousarray(np.asarray(slice_thicknesses, np.float64).ravel())
        count = len(thick)
        size = max(count, 1) * max(int(rows), 1) * max(int(columns), 1)
        re, im = np.zeros(size), np.zeros(size)
        st = L.load().cubo_ptycho_propagators(int(rows), int(columns), float(row_sampling), float(column_sampling),
                                         float(wavelength), count, _ptr(thick) if count else None, _ptr(re), _ptr(im))
        if st != 0:
            raise PtychographyError("propagators")
        return (re + 1j * im).reshape(count, int(rows), int(columns))

    @staticmethod
    def reconstruct(amplitudes, positions, object, probe, slice_thicknesses, wavelength: float, row_sampling: float,
                    column_sampling: float, iterations: int = 8, step_size: float = 0.5,
                    normalization_minimum: float = 1.0, fix_probe: bool = False, pure_phase_object: bool = False,
                    identical_slices: bool = False, fix_probe_center_of_mass: bool = False,
                    constrain_probe_amplitude: bool = False, probe_amplitude_relative_radius: float = 0.5,
                    probe_amplitude_relative_width: float = 0.05, fix_probe_aperture: bool = False,
                    probe_support_mask=None, error_normalization="suppliedAmplitudeEnergy",
                    device: int = 0) -> MultisliceResult:
        """``object`` is ``(slices, rows, columns)`` complex (entrance first), ``slice_thicknesses`` the
        ``slices - 1`` gaps, in the units of ``wavelength`` and the samplings."""
        obj = np.asarray(object)
        prb = np.asarray(probe)
        if obj.ndim != 3 or prb.ndim != 2:
            raise PtychographyError("object must be (slices, rows, columns) and probe 2-D")
        ctx = context(device)
        inp = _Inputs(amplitudes, positions, obj.shape[1:], prb.shape, iterations, step_size, normalization_minimum,
                      fix_probe, pure_phase_object, True, fix_probe_center_of_mass, constrain_probe_amplitude,
                      probe_amplitude_relative_radius, probe_amplitude_relative_width, fix_probe_aperture,
                      probe_support_mask, error_normalization, None, "fp64")
        multi, thick = _multislice_params(obj.shape[0], slice_thicknesses, wavelength, row_sampling,
                                          column_sampling, identical_slices)
        ore, oim = _split(obj)
        pre, pim = _split(prb)
        errors = np.zeros(max(int(iterations), 1))
        ctx.check(ctx.lib.cubo_ptycho_multislice_reconstruct(ctx.handle, C.byref(inp.problem), C.byref(inp.params),
                                                             C.byref(multi), _ptr(ore), _ptr(oim), _ptr(pre),
                                                             _ptr(pim), _ptr(errors)))
        del thick
        return MultisliceResult((ore + 1j * oim).reshape(obj.shape), (pre + 1j * pim).reshape(prb.shape),
                                errors[: int(iterations)].copy())


class Plan:
    """A device-resident reconstruction (``cubo_ptycho_plan_*``): upload once, iterate, read the state back."""

    def __init__(self, amplitudes, positions, object_shape, probe_shape, ctx: Optional[Context] = None, **kwargs):
        """``mixed_states=S`` makes a mixed-state plan (``cubo_ptycho_mixed_plan_create``, FP64; with
        ``orthogonalize_probes`` and ``zero_far_field_pixel_error``): its state holds S probes.
        ``multislice=dict(slices=L, slice_thicknesses=..., wavelength=..., row_sampling=..., column_sampling=...[,
        identical_slices=...])`` makes a multislice plan (``cubo_ptycho_multislice_plan_create``, FP64): its object
        holds L slices of ``object_shape``."""
        self.ctx = ctx or context(kwargs.pop("device", 0))
        states = kwargs.pop("mixed_states", None)
        multislice = kwargs.pop("multislice", None)
        orthogonalize_probes = kwargs.pop("orthogonalize_probes", True)
        zero_error = kwargs.pop("zero_far_field_pixel_error", "reference")
        if states is not None and multislice is not None:
            raise PtychographyError("one engine per plan")
        if states is not None or multislice is not None:
            kwargs["precision"] = "fp64"
            kwargs.setdefault("constrain_object_amplitude", True)
        defaults = dict(iterations=0, step_size=0.5, normalization_minimum=1.0, fix_probe=False,
                        pure_phase_object=False, constrain_object_amplitude=True, fix_probe_center_of_mass=False,
                        constrain_probe_amplitude=False, probe_amplitude_relative_radius=0.5,
                        probe_amplitude_relative_width=0.05, fix_probe_aperture=False, probe_support_mask=None,
                        error_normalization="suppliedAmplitudeEnergy", position_correction=None, precision="fp32",
                        variant="auto", gather_tile=0, pass_shape=0)
        defaults.update(kwargs)
        self.inputs = _Inputs(amplitudes, positions, tuple(object_shape), tuple(probe_shape), **defaults)
        self.object_shape = tuple(object_shape)
        if multislice is not None:
            self.object_shape = (int(multislice["slices"]),) + self.object_shape
        self.probe_shape = tuple(probe_shape) if states is None else (int(states),) + tuple(probe_shape)
        h = C.c_void_p()
        if multislice is not None:
            ms = dict(multislice)
            multi, self._thicknesses = _multislice_params(ms["slices"], ms["slice_thicknesses"], ms["wavelength"],
                                                          ms["row_sampling"], ms["column_sampling"],
                                                          ms.get("identical_slices", False))
            self.ctx.check(self.ctx.lib.cubo_ptycho_multislice_plan_create(
                self.ctx.handle, C.byref(self.inputs.problem), C.byref(self.inputs.params), C.byref(multi),
                C.byref(h)))
        elif states is None:
            self.ctx.check(self.ctx.lib.cubo_ptycho_plan_create(self.ctx.handle, C.byref(self.inputs.problem),
                                                                C.byref(self.inputs.params), C.byref(h)))
        else:
            mixed = L.MixedParams()
            self.ctx.lib.cubo_ptycho_mixed_params_default(C.byref(mixed))
            mixed.states = int(states)
            mixed.orthogonalize_probes = int(bool(orthogonalize_probes))
            mixed.zero_pixel_error = L.ZERO_PIXEL_REFERENCE if zero_error == "reference" else L.ZERO_PIXEL_FINITE
            self.ctx.check(self.ctx.lib.cubo_ptycho_mixed_plan_create(self.ctx.handle, C.byref(self.inputs.problem),
                                                                      C.byref(self.inputs.params), C.byref(mixed),
                                                                      C.byref(h)))
        self.handle = h

    def set_state(self, obj, probe):
        ore, oim = _split(obj, self.object_shape)
        pre, pim = _split(probe, self.probe_shape)
        self.ctx.check(self.ctx.lib.cubo_ptycho_plan_set_state(self.handle, _ptr(ore), _ptr(oim), _ptr(pre), _ptr(pim)))

    def get_state(self):
        no = int(np.prod(self.object_shape))
        npb = int(np.prod(self.probe_shape))
        ore, oim, pre, pim = np.zeros(no), np.zeros(no), np.zeros(npb), np.zeros(npb)
        self.ctx.check(self.ctx.lib.cubo_ptycho_plan_get_state(self.handle, _ptr(ore), _ptr(oim), _ptr(pre), _ptr(pim)))
        return (ore + 1j * oim).reshape(self.object_shape), (pre + 1j * pim).reshape(self.probe_shape)

    def positions(self) -> np.ndarray:
        """The current scan positions (P, 2): the given ones, moved by position correction when it is on."""
        count = self.inputs.count
        rows, columns = np.zeros(max(count, 1)), np.zeros(max(count, 1))
        self.ctx.check(self.ctx.lib.cubo_ptycho_plan_get_positions(self.handle, _ptr(rows), _ptr(columns)))
        return np.column_stack([rows[:count], columns[:count]])

    def iterate(self, iterations: int):
        errors = np.zeros(max(iterations, 1))
        self.ctx.check(self.ctx.lib.cubo_ptycho_plan_iterate(self.handle, iterations, _ptr(errors)))
        return errors[:iterations]

    def enqueue(self, iterations: int):
        self.ctx.check(self.ctx.lib.cubo_ptycho_plan_enqueue(self.handle, iterations))

    def errors(self, count: int):
        out = np.zeros(max(count, 1))
        self.ctx.check(self.ctx.lib.cubo_ptycho_plan_errors(self.handle, count, _ptr(out)))
        return out[:count]

    # ---- sharded iterations (cubo_ptycho_plan_enqueue_gradients / _gradient_buffers / _apply_gradients)
    def enqueue_gradients(self):
        """This plan's band of the positions: position pass and gathers, the sums left for the other bands' to be added."""
        self.ctx.check(self.ctx.lib.cubo_ptycho_plan_enqueue_gradients(self.handle))

    def apply_gradients(self):
        """The updates from the gradient sums of every band (after they have been summed into this plan's buffers)."""
        self.ctx.check(self.ctx.lib.cubo_ptycho_plan_apply_gradients(self.handle))

    def gradient_tensors(self):
        """Zero-copy torch views of the buffers one sharded iteration sums over the bands: ``grad_object``,
        ``weight_object``, ``grad_probe``, ``weight_probe`` and ``loss`` (valid after the first enqueue_gradients)."""
        import torch
        ptrs = [C.c_void_p() for _ in range(5)]
        real = C.c_int(0)
        self.ctx.check(self.ctx.lib.cubo_ptycho_plan_gradient_buffers(self.handle, *[C.byref(x) for x in ptrs],
                                                                      C.byref(real)))
        objects = int(np.prod(self.object_shape))
        n = int(self.probe_shape[-1] * self.probe_shape[-2])
        states = int(self.probe_shape[0]) if len(self.probe_shape) == 3 else 1
        t = "<f4" if real.value == 4 else "<f8"

        class _View:  # the CUDA array interface over one of the plan's device buffers
            def __init__(self, ptr, shape, typestr):
                self.__cuda_array_interface__ = {"shape": shape, "typestr": typestr, "data": (ptr, False),
                                                 "version": 3, "strides": None}

        dev = torch.device("cuda", self.ctx.device)
        return {"grad_object": torch.as_tensor(_View(ptrs[0].value, (objects, 2), t), device=dev),
                "weight_object": torch.as_tensor(_View(ptrs[1].value, (objects,), t), device=dev),
                "grad_probe": torch.as_tensor(_View(ptrs[2].value, (states * n, 2), "<f8"), device=dev),
                "weight_probe": torch.as_tensor(_View(ptrs[3].value, (n,), "<f8"), device=dev),
                "loss": torch.as_tensor(_View(ptrs[4].value, (1,), "<f8"), device=dev)}

    def forward(self) -> float:
        """The unnormalised loss sum (|F| - A)^2 of the current state (``cubo_ptycho_plan_forward``)."""
        loss = C.c_double(0)
        self.ctx.check(self.ctx.lib.cubo_ptycho_plan_forward(self.handle, C.byref(loss)))
        return loss.value

    def backward(self, recompute_exit_waves: bool = False):
        """``(loss, grad_object, grad_probe)``: dL/dRe + i dL/dIm of the forward loss (``cubo_ptycho_plan_backward``)."""
        no = int(np.prod(self.object_shape))
        npb = int(np.prod(self.probe_shape))
        gore, goim, gpre, gpim = np.zeros(no), np.zeros(no), np.zeros(npb), np.zeros(npb)
        loss = C.c_double(0)
        self.ctx.check(self.ctx.lib.cubo_ptycho_plan_backward(self.handle, 1 if recompute_exit_waves else 0,
                                                              C.byref(loss), _ptr(gore), _ptr(goim), _ptr(gpre),
                                                              _ptr(gpim)))
        return (loss.value, (gore + 1j * goim).reshape(self.object_shape),
                (gpre + 1j * gpim).reshape(self.probe_shape))

    def set_timing(self, enabled: bool):
        self.ctx.check(self.ctx.lib.cubo_ptycho_plan_set_timing(self.handle, 1 if enabled else 0))

    def kernel_stats(self):
        cap = 32
        names = (C.c_char_p * cap)()
        ms = (C.c_double * cap)()
        launches = (C.c_longlong * cap)()
        count = C.c_int(0)
        self.ctx.check(self.ctx.lib.cubo_ptycho_plan_kernel_stats(self.handle, cap, names, ms, launches, C.byref(count)))
        return {names[i].decode(): (ms[i], launches[i]) for i in range(count.value)}

    @property
    def launch_count(self) -> int:
        return int(self.ctx.lib.cubo_ptycho_plan_launch_count(self.handle))

    def close(self):
        if getattr(self, "handle", None):
            self.ctx.lib.cubo_ptycho_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many independent reconstructions advanced together (``cubo_ptycho_batch_*``): one iteration of all of them is
    captured once into a CUDA graph and replayed.

    ``items`` is a list of dicts with ``amplitudes``, ``positions``, ``object``, ``probe`` and optional keyword
    parameters of ``SingleslicePtychography.reconstruct`` (``step_size``, ``precision``, ...).
    """

    def __init__(self, items, ctx: Optional[Context] = None):
        self.ctx = ctx or context(0)
        keys = ("iterations", "step_size", "normalization_minimum", "fix_probe", "pure_phase_object",
                "constrain_object_amplitude", "fix_probe_center_of_mass", "constrain_probe_amplitude",
                "probe_amplitude_relative_radius", "probe_amplitude_relative_width", "fix_probe_aperture",
                "probe_support_mask", "error_normalization", "position_correction", "precision", "variant",
                "gather_tile", "pass_shape")
        defaults = dict(iterations=0, step_size=0.5, normalization_minimum=1.0, fix_probe=False,
                        pure_phase_object=False, constrain_object_amplitude=True, fix_probe_center_of_mass=False,
                        constrain_probe_amplitude=False, probe_amplitude_relative_radius=0.5,
                        probe_amplitude_relative_width=0.05, fix_probe_aperture=False, probe_support_mask=None,
                        error_normalization="suppliedAmplitudeEnergy", position_correction=None, precision="fp32",
                        variant="auto", gather_tile=0, pass_shape=0)
        self.inputs, self.shapes = [], []
        for it in items:
            kw = dict(defaults)
            kw.update({k: v for k, v in it.items() if k in keys})
            obj, prb = np.asarray(it["object"]), np.asarray(it["probe"])
            self.inputs.append(_Inputs(it["amplitudes"], it["positions"], obj.shape, prb.shape, **kw))
            self.shapes.append((obj.shape, prb.shape))
        n = len(self.inputs)
        problems = (L.Problem * n)(*[i.problem for i in self.inputs])
        params = (L.Params * n)(*[i.params for i in self.inputs])
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.cubo_ptycho_batch_create(self.ctx.handle, n, problems, params, C.byref(h)))
        self.handle = h
        for i, it in enumerate(items):
            self.set_state(i, it["object"], it["probe"])

    def __len__(self):
        return len(self.inputs)

    def set_state(self, index, obj, probe):
        os_, ps = self.shapes[index]
        ore, oim = _split(obj, os_)
        pre, pim = _split(probe, ps)
        self.ctx.check(self.ctx.lib.cubo_ptycho_batch_set_state(self.handle, index, _ptr(ore), _ptr(oim), _ptr(pre),
                                                                _ptr(pim)))

    def get_state(self, index):
        os_, ps = self.shapes[index]
        no, npb = int(np.prod(os_)), int(np.prod(ps))
        ore, oim, pre, pim = np.zeros(no), np.zeros(no), np.zeros(npb), np.zeros(npb)
        self.ctx.check(self.ctx.lib.cubo_ptycho_batch_get_state(self.handle, index, _ptr(ore), _ptr(oim), _ptr(pre),
                                                                _ptr(pim)))
        return (ore + 1j * oim).reshape(os_), (pre + 1j * pim).reshape(ps)

    def run(self, iterations: int, synchronize: bool = True):
        self.ctx.check(self.ctx.lib.cubo_ptycho_batch_run(self.handle, iterations, 1 if synchronize else 0))

    def errors(self, index, count):
        out = np.zeros(max(count, 1))
        self.ctx.check(self.ctx.lib.cubo_ptycho_batch_errors(self.handle, index, count, _ptr(out)))
        return out[:count]

    @property
    def launches_per_iteration(self) -> int:
        return int(self.ctx.lib.cubo_ptycho_batch_launches_per_iteration(self.handle))

    def close(self):
        if getattr(self, "handle", None):
            self.ctx.lib.cubo_ptycho_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class PtychographyAmplitudes:
    """``PtychographyAmplitudes`` (``PtychographyPreparation.swift:62-75``): square-root amplitudes of a cube,
    corner-centred, ``[position][row][column]`` (Float32 here: the engine's input), with the mean intensities."""
    values: object                 # numpy float32 array, or a CUDA tensor when kept on the device
    position_count: int
    detector_rows: int
    detector_columns: int
    mean_intensity: float          # mean over positions of the summed shifted intensity, negatives included
    clipped_mean_intensity: float  # the same with negative shifted values set to zero first

    @property
    def error_normalization(self):
        """py4DSTEM's error normalisation for the engines: ``.meanIntensity(meanIntensity)``."""
        return ("meanIntensity", self.mean_intensity)


class PtychographyPreparation:
    """``PtychographyPreparation.amplitudes(from:origins:shift:)`` (``PtychographyPreparation.swift:142-183``) on the
    device: every pattern shifted so its origin sits on the corner pixel (bilinear or periodic cubic B-spline, wrapped,
    FP64), then ``sqrt(max(., 0))``; see ``cubo_ptycho_prepare_amplitudes`` in ``include/cubo_ptycho.h``."""

    SHIFTS = {"bilinear": L.SHIFT_BILINEAR, "cubicSpline": L.SHIFT_CUBIC_SPLINE}

    @staticmethod
    def amplitudes(cube, origins, shift: str = "cubicSpline", keep_on_device: bool = False,
                   ctx: Optional[Context] = None, device: int = 0, out=None) -> PtychographyAmplitudes:
        """``cube``: ``[position][row][column]`` (or ``[scan row][scan column][row][column]``), Float32 values, a numpy
        array or a CUDA tensor.  ``origins``: ``(row, column)`` for every pattern (``PtychographyOrigins.uniform``) or
        ``(rows, columns)`` arrays with one value per position (``.perPosition``).  ``keep_on_device``: return the
        amplitudes as a CUDA tensor (for ``reconstruct`` / ``Plan`` without a host round trip).  ``out``: a contiguous
        Float32 CUDA tensor of ``count * rows * columns`` values on the context's device to write the amplitudes into
        (implies ``keep_on_device``; repeated calls then allocate no device memory for the result)."""
        if shift not in PtychographyPreparation.SHIFTS:
            raise PtychographyError(f"shift {shift!r}")
        ctx = ctx or context(device)
        cuda_in = _is_cuda_tensor(cube)
        shape = tuple(cube.shape)
        if len(shape) == 4:
            shape = (shape[0] * shape[1], shape[2], shape[3])
        if len(shape) != 3:
            raise PtychographyError("cube must be [position][row][column]")
        count, rows, columns = shape
        o_rows, o_cols = origins
        if np.ndim(o_rows) == 0 and np.ndim(o_cols) == 0:
            o_rows = np.full(count, float(o_rows))
            o_cols = np.full(count, float(o_cols))
        o_rows = np.ascontiguousarray(o_rows, np.float64).ravel()
        o_cols = np.ascontiguousarray(o_cols, np.float64).ravel()
        if o_rows.size != count or o_cols.size != count:
            raise PtychographyError("one origin per position")  # PtychographyPreparation.swift:157
        mean, clipped = C.c_double(), C.c_double()
        code = PtychographyPreparation.SHIFTS[shift]
        if out is not None:
            keep_on_device = True
            if not (_is_cuda_tensor(out) and str(out.dtype) == "torch.float32" and out.is_contiguous()
                    and out.numel() == count * rows * columns and out.device.index == ctx.device):
                raise PtychographyError("out must be a contiguous Float32 CUDA tensor of count * rows * columns values "
                                        "on the context's device")
        if cuda_in or keep_on_device:
            torch = _torch()
            dev = torch.device("cuda", ctx.device)
            src = cube if cuda_in else torch.from_numpy(np.ascontiguousarray(cube, np.float32))
            src = src.to(dev, torch.float32).contiguous().reshape(count, rows, columns)
            out = (torch.empty((count, rows, columns), dtype=torch.float32, device=dev) if out is None
                   else out.view(count, rows, columns))
            torch.cuda.synchronize(dev)
            ctx.check(ctx.lib.cubo_ptycho_prepare_amplitudes_device(
                ctx.handle, count, rows, columns, C.c_void_p(src.data_ptr()), _ptr(o_rows), _ptr(o_cols), code,
                C.c_void_p(out.data_ptr()), C.byref(mean), C.byref(clipped)))
            values = out if keep_on_device else out.cpu().numpy()
        else:
            src = np.ascontiguousarray(cube, np.float32).reshape(count, rows, columns)
            values = np.empty((count, rows, columns), np.float32)
            ctx.check(ctx.lib.cubo_ptycho_prepare_amplitudes(
                ctx.handle, count, rows, columns, src.ctypes.data_as(C.c_void_p), _ptr(o_rows), _ptr(o_cols), code,
                values.ctypes.data_as(C.c_void_p), C.byref(mean), C.byref(clipped)))
        return PtychographyAmplitudes(values, count, rows, columns, mean.value, clipped.value)


class PtychographyProbe:
    """``PtychographyProbe.build`` (``Ptychography.swift:142-172``), evaluated on the device in FP64."""

    @staticmethod
    def build(rows: int, columns: int, row_sampling: float, column_sampling: float, wavelength: float, cutoff: float,
              rolloff: float = 0.002, defocus: float = 0.0, astigmatism: float = 0.0, astigmatism_angle: float = 0.0,
              spherical_aberration: float = 0.0, higher_order: Sequence = (), device: int = 0) -> np.ndarray:
        """``higher_order`` rows are ``(radialOrder, angularOrder, sine, coefficient)``."""
        ctx = context(device)
        t = np.ascontiguousarray(np.asarray(higher_order, np.float64).reshape(-1, 4))
        re = np.zeros(rows * columns)
        im = np.zeros(rows * columns)
        st = ctx.lib.cubo_ptycho_probe_build(ctx.handle, rows, columns, row_sampling, column_sampling, wavelength,
                                             cutoff, rolloff, defocus, astigmatism, astigmatism_angle,
                                             spherical_aberration, len(t), _ptr(t), _ptr(re), _ptr(im))
        ctx.check(st)
        return (re + 1j * im).reshape(rows, columns)


def electron_wavelength(energy_ev: float) -> float:
    """Relativistic electron wavelength in angstrom from CODATA constants."""
    h, m, e, c = 6.62607015e-34, 9.1093837015e-31, 1.602176634e-19, 299792458.0
    v = energy_ev * e
    return h / np.sqrt(2 * m * v * (1 + v / (2 * m * c * c))) * 1e10
