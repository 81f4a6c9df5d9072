"""FP64 NumPy restatement of CuboPtycho's single-slice gradient descent — TEST INFRASTRUCTURE ONLY.

This module is an oracle: only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import it,
and only to check or time against the CUDA path.  Nothing in ``cubokit_b200`` imports it; the product has no CPU fallback.

It restates, in vectorised NumPy (``np.fft`` is pocketfft in double, NumPy's fft/ifft convention, as CuboKit's
``FFT2D``), the arithmetic of (paths inside the CuboKit project):
  * ``Sources/CuboPtycho/Ptychography.swift:142-172``  ``PtychographyProbe.build``
  * ``Sources/CuboPtycho/Ptychography.swift:218-406``  ``SingleslicePtychography.reconstruct`` (Double path)
  * ``Sources/CuboPtycho/Ptychography.swift:474``      ``frequency``
  * ``Sources/CuboPtycho/PtychographyConstraints.swift:9-83``  probe constraints
  * ``Sources/CuboPtycho/PtychographyPreparation.swift:244-259``  ``initialProbe`` energy scaling
  * ``Sources/CuboPtycho/PtychographyPreparation.swift:142-183,296-344``  ``amplitudes(from:origins:shift:)``: the
    bilinear and periodic cubic-spline pattern shifts, square-root amplitudes and mean intensities
  * ``Sources/CuboPtycho/PtychographyEngines.swift:121-267,270-298``  ``MixedstatePtychography`` (reconstruct,
    orthogonalize, initialProbes: NumPy's own legacy ``RandomState`` draws)
  * ``Sources/CuboPtycho/PtychographyEngines.swift:427-589``  ``MultislicePtychography`` (propagators, reconstruct)
  * ``Sources/CuboPtycho/Ptychography.swift:53-85,260-264,371-377,398-401,411-472``  position correction
    (``PtychographyPositionCorrection``: the per-position 2 x 2 least-squares step, its limits, the centre-of-mass
    constraint)

Pinned against the py4DSTEM fixtures of CuboKit's own tests (``tests/golden/*.npz``) by ``tests/test_oracle.py``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

try:  # scipy's erf is vectorised; math.erf is the fallback
    from scipy.special import erf as _erf
except Exception:  # pragma: no cover
    _erf = np.vectorize(math.erf)


class PtychographyError(ValueError):
    """``PtychographyError.invalidInput`` (``Ptychography.swift:24-27``)."""


def frequency(k, n):
    """``fftfreq`` sample ``k`` of ``n`` (``Ptychography.swift:474``)."""
    k = np.asarray(k)
    return np.where(k < (n + 1) // 2, k, k - n) / n


def fftfreq_grid(rows, columns):
    return frequency(np.arange(rows), rows), frequency(np.arange(columns), columns)


@dataclass
class AberrationTerm:
    """``PtychographyAberrationTerm`` (``Ptychography.swift:101-133``)."""
    radial_order: int
    angular_order: int
    sine: bool
    coefficient: float

    @staticmethod
    def polar(radial_order, angular_order, magnitude, azimuth):
        if angular_order == 0:
            return [AberrationTerm(radial_order, 0, False, magnitude)]
        m = float(angular_order)
        return [AberrationTerm(radial_order, angular_order, False, magnitude * math.cos(m * azimuth)),
                AberrationTerm(radial_order, angular_order, True, magnitude * math.sin(m * azimuth))]

    def valid(self):
        return (math.isfinite(self.coefficient) and 1 <= self.radial_order <= 64 and self.angular_order >= 0
                and (not self.sine or self.angular_order > 0))

    def phase(self, alpha, azimuth):
        radial = alpha ** (self.radial_order + 1) / (self.radial_order + 1)
        if self.angular_order == 0:
            return self.coefficient * radial
        angle = self.angular_order * azimuth
        return self.coefficient * radial * (np.sin(angle) if self.sine else np.cos(angle))


def probe_build(rows, columns, row_sampling, column_sampling, wavelength, cutoff, rolloff=0.002, defocus=0.0,
                astigmatism=0.0, astigmatism_angle=0.0, spherical_aberration=0.0, higher_order=()):
    """Corner-centred unit-norm probe (``Ptychography.swift:142-172``)."""
    vals = [row_sampling, column_sampling, wavelength, cutoff]
    if not (rows > 1 and columns > 1 and all(math.isfinite(v) and v > 0 for v in vals)
            and math.isfinite(rolloff) and rolloff >= 0
            and all(math.isfinite(v) for v in (defocus, astigmatism, astigmatism_angle, spherical_aberration))
            and all(t.valid() for t in higher_order)):
        raise PtychographyError("invalid probe parameters")
    fr, fc = fftfreq_grid(rows, columns)
    qr = (fr / row_sampling)[:, None] * np.ones((1, columns))
    qc = np.ones((rows, 1)) * (fc / column_sampling)[None, :]
    alpha = np.hypot(qr, qc) * wavelength
    angle = np.arctan2(qc, qr)
    if rolloff > 0:
        soft = np.where(alpha > cutoff, 0.0, 0.5 * (1 + np.cos(np.pi * (alpha - cutoff + rolloff) / rolloff)))
        aperture = np.where(alpha > cutoff - rolloff, soft, 1.0)
    else:
        aperture = np.where(alpha < cutoff, 1.0, 0.0)
    a2 = alpha * alpha
    phase = a2 / 2 * (-defocus + astigmatism * np.cos(2 * (angle - astigmatism_angle))) + a2 * a2 / 4 * spherical_aberration
    for t in higher_order:
        phase = phase + t.phase(alpha, angle)
    chi = 2 * np.pi / wavelength * phase
    spec = aperture * np.cos(chi) - 1j * aperture * np.sin(chi)
    p = np.fft.ifft2(spec)
    norm = math.sqrt(float(np.sum(p.real ** 2 + p.imag ** 2)))
    if not (norm > 0 and math.isfinite(norm)):
        raise PtychographyError("probe without intensity")
    return p / norm


def initial_probe(rows, columns, sampling_row, sampling_column, wavelength, semiangle, rolloff=2.0, defocus=0.0,
                  astigmatism=0.0, astigmatism_angle=0.0, spherical_aberration=0.0, higher_order=(), mean_intensity=1.0):
    """Probe scaled so ``sum |fft2(probe)|^2 == mean_intensity`` (``PtychographyPreparation.swift:244-259``)."""
    if not (math.isfinite(mean_intensity) and mean_intensity > 0):
        raise PtychographyError("mean intensity")
    p = probe_build(rows, columns, sampling_row, sampling_column, wavelength, semiangle / 1e3, rolloff / 1e3, defocus,
                    astigmatism, astigmatism_angle, spherical_aberration, higher_order)
    energy = float(np.sum(np.abs(np.fft.fft2(p)) ** 2))
    return p * math.sqrt(mean_intensity / energy)


# ---------------------------------------------------------------- probe constraints (PtychographyConstraints.swift)

def probe_center_of_mass(p):
    """``PtychographyConstraints.swift:9-18``."""
    rows, columns = p.shape
    w = p.real ** 2 + p.imag ** 2
    total = float(w.sum())
    if not (total > 0 and math.isfinite(total)):
        return None
    fr, fc = fftfreq_grid(rows, columns)
    return float((fr * rows) @ w.sum(axis=1)) / total, float(w.sum(axis=0) @ (fc * columns)) / total


def fourier_shift(p, row, column):
    """``PtychographyConstraints.swift:21-31``: ``out[x] = in[x - shift]``."""
    rows, columns = p.shape
    fr, fc = fftfreq_grid(rows, columns)
    phase = -2 * np.pi * (fr[:, None] * row + fc[None, :] * column)
    return np.fft.ifft2(np.fft.fft2(p) * (np.cos(phase) + 1j * np.sin(phase)))


def center_of_mass_constraint(p):
    com = probe_center_of_mass(p)
    return p if com is None else fourier_shift(p, -com[0], -com[1])


def amplitude_constraint(p, radius, width):
    """``PtychographyConstraints.swift:40-55``."""
    rows, columns = p.shape
    before = float(np.sum(p.real ** 2 + p.imag ** 2))
    sigma = math.sqrt(math.pi) / width
    fr, fc = fftfreq_grid(rows, columns)
    d = np.hypot(fr[:, None], fc[None, :]) - radius
    mask = 0.5 * (1 - _erf(sigma * d / (1 - d * d)))
    q = p * mask
    after = float(np.sum(q.real ** 2 + q.imag ** 2))
    if not (before > 0 and after > 0):
        return q
    return q * math.sqrt(before / after)


def aperture_constraint(p, aperture):
    """``PtychographyConstraints.swift:59-71``."""
    before = float(np.sum(p.real ** 2 + p.imag ** 2))
    f = np.fft.fft2(p)
    ph = np.arctan2(f.imag, f.real)
    q = np.fft.ifft2(aperture * np.cos(ph) + 1j * aperture * np.sin(ph))
    after = float(np.sum(q.real ** 2 + q.imag ** 2))
    if not (before > 0 and after > 0):
        return q
    return q * math.sqrt(before / after)


# ---------------------------------------------------------------- the engine

def round_half_even(x):
    return np.round(x)  # numpy rounds half to even


def patch_indices(rows, columns, object_rows, object_columns, rr, cc):
    """Periodic corner-centred patch indices ``Ptychography.swift:321-336`` for integer centres ``rr, cc`` (P,)."""
    ro = np.arange(rows)
    ro = np.where(ro < (rows + 1) // 2, ro, ro - rows)
    co = np.arange(columns)
    co = np.where(co < (columns + 1) // 2, co, co - columns)
    r = np.mod(rr[:, None] + ro[None, :], object_rows)
    c = np.mod(cc[:, None] + co[None, :], object_columns)
    return (r[:, :, None] * object_columns + c[:, None, :]).reshape(len(rr), rows * columns)


def shifted_probes(probe_spectrum, dr, dc):
    """``Ptychography.swift:303-320``: ``ifft2(spectrum * ramp(dr, dc))`` for each position, grouped by its fraction."""
    rows, columns = probe_spectrum.shape
    fr, fc = fftfreq_grid(rows, columns)
    out = np.empty((len(dr), rows, columns), np.complex128)
    keys = {}
    for i, key in enumerate(zip(dr.tolist(), dc.tolist())):
        keys.setdefault(key, []).append(i)
    for (a, b), idx in keys.items():
        ar = -2 * np.pi * fr * a
        ac = -2 * np.pi * fc * b
        ramp = (np.cos(ar) + 1j * np.sin(ar))[:, None] * (np.cos(ac) + 1j * np.sin(ac))[None, :]
        out[idx] = np.fft.ifft2(probe_spectrum * ramp)
    return out


def error_divisor(amplitudes, count, error_normalization, mean_intensity):
    """``Ptychography.swift:40-47``."""
    if error_normalization == "meanIntensity":
        d = mean_intensity * count
    else:
        d = float(np.sum(np.asarray(amplitudes, np.float64) ** 2))
    if not (math.isfinite(d) and d > 0):
        raise PtychographyError("error normalisation")
    return d


def validate(amplitudes, positions, object_shape, probe_shape, iterations, step_size, normalization_minimum,
             radius, width, probe_support_mask):
    """The refusals of ``Ptychography.swift:247-259``."""
    n = probe_shape[0] * probe_shape[1]
    count = len(positions)
    a = np.asarray(amplitudes, np.float64)
    pos = np.asarray(positions, np.float64).reshape(-1, 2) if count else np.zeros((0, 2))
    ok = (count > 0 and a.size == count * n and np.all(np.isfinite(a)) and np.all(a >= 0)
          and iterations >= 0 and math.isfinite(step_size) and step_size > 0
          and math.isfinite(normalization_minimum) and 0 <= normalization_minimum <= 1
          and np.all(np.isfinite(pos)) and np.all(np.abs(pos) < float((2 ** 63 - 1) // 4))
          and math.isfinite(radius) and 0 <= radius <= 0.5 and math.isfinite(width) and 0 < width <= 0.5
          and object_shape[0] >= probe_shape[0] and object_shape[1] >= probe_shape[1]
          and (probe_support_mask is None or np.asarray(probe_support_mask).size == n))
    if not ok:
        raise PtychographyError("invalid input")


@dataclass
class PositionCorrection:
    """``PtychographyPositionCorrection`` (``Ptychography.swift:53-72``); distances in Å, ``None`` = unlimited."""
    step_size: float = 0.5
    max_update_distance: float | None = None
    max_total_distance: float | None = None
    row_sampling: float | None = None
    column_sampling: float | None = None
    constrain_center_of_mass: bool = False

    def pixel_distances(self):
        """``pixelDistances`` (``Ptychography.swift:74-84``): (update, total) in pixels, or a refusal."""
        if not math.isfinite(self.step_size):
            raise PtychographyError("position step")
        scale = 1.0
        if self.max_update_distance is not None or self.max_total_distance is not None:
            r, c = self.row_sampling, self.column_sampling
            if r is None or c is None or not (math.isfinite(r) and r > 0 and math.isfinite(c) and c > 0):
                raise PtychographyError("samplings")
            scale = math.sqrt(r * r + c * c)
        for d in (self.max_update_distance, self.max_total_distance):
            if d is not None and not (math.isfinite(d) and d > 0):
                raise PtychographyError("distance")
        return ((math.inf if self.max_update_distance is None else self.max_update_distance) / scale,
                (math.inf if self.max_total_distance is None else self.max_total_distance) / scale)


def position_update(before, after, spectrum, amp, positions, initial, step, limits):
    """``positionUpdate`` (``Ptychography.swift:411-472``) for all positions at once.  ``before`` / ``after``: the
    object (flat) the forward model used and the one with the update added; ``spectrum``: the forward model's probe
    spectrum (R, C); ``amp`` (P, n).  Returns the new positions (P, 2)."""
    rows, columns = spectrum.shape
    n = rows * columns
    object_rows, object_columns = before.shape if before.ndim == 2 else (None, None)
    before, after = before.reshape(-1), after.reshape(-1)
    count = len(positions)
    rr = round_half_even(positions[:, 0])
    cc = round_half_even(positions[:, 1])
    dr, dc = positions[:, 0] - rr, positions[:, 1] - cc
    fr, fc = fftfreq_grid(rows, columns)
    phase = -2 * np.pi * (fr[None, :, None] * dr[:, None, None] + fc[None, None, :] * dc[:, None, None])
    s = np.fft.ifft2(spectrum[None] * (np.cos(phase) + 1j * np.sin(phase))).reshape(count, n)
    ri, ci = rr.astype(np.int64), cc.astype(np.int64)

    def far(obj, row_step, column_step):  # :424-436
        idx = patch_indices(rows, columns, object_rows, object_columns, ri + row_step, ci + column_step)
        return np.fft.fft2((s * obj[idx]).reshape(count, rows, columns)).reshape(count, n)

    f, fdx, fdy = far(before, 0, 0), far(after, 1, 0), far(after, 0, 1)
    difference = amp * amp - (f.real ** 2 + f.imag ** 2)
    dx = 2 * ((f.real - fdx.real) * f.real + (f.imag - fdx.imag) * f.imag)
    dy = 2 * ((f.real - fdy.real) * f.real + (f.imag - fdy.imag) * f.imag)
    axx, axy, ayy = np.sum(dx * dx, 1), np.sum(dx * dy, 1), np.sum(dy * dy, 1)
    bx, by = np.sum(dx * difference, 1), np.sum(dy * difference, 1)
    out = positions.copy()
    for i in range(count):  # :447-470
        det = axx[i] * ayy[i] - axy[i] * axy[i]
        u0 = u1 = 0.0
        if det != 0 and math.isfinite(det):
            u0 = (ayy[i] * bx[i] - axy[i] * by[i]) / det * step
            u1 = (axx[i] * by[i] - axy[i] * bx[i]) / det * step
        if not (math.isfinite(u0) and math.isfinite(u1)):
            continue
        norm = math.hypot(u0, u1)
        if norm > limits[0]:
            u0 /= norm / limits[0]
            u1 /= norm / limits[0]
        if math.isfinite(limits[1]):
            if math.hypot(positions[i, 0] - initial[i, 0] - u0, positions[i, 1] - initial[i, 1] - u1) > limits[1]:
                u0 = u1 = 0.0
        row, column = positions[i, 0] - u0, positions[i, 1] - u1
        if not (abs(row) < float((2 ** 63 - 1) // 4) and abs(column) < float((2 ** 63 - 1) // 4)):
            raise PtychographyError("position")
        out[i] = (row, column)
    return out


def reconstruct(amplitudes, positions, obj, probe, iterations=8, step_size=0.5, normalization_minimum=1.0,
                fix_probe=False, pure_phase_object=False, constrain_object_amplitude=True,
                fix_probe_center_of_mass=False, constrain_probe_amplitude=False,
                probe_amplitude_relative_radius=0.5, probe_amplitude_relative_width=0.05,
                fix_probe_aperture=False, probe_support_mask=None, error_normalization="suppliedAmplitudeEnergy",
                mean_intensity=None, progress=None, position_correction: PositionCorrection | None = None):
    """``SingleslicePtychography.reconstruct`` Double path (``Ptychography.swift:218-406``).

    ``amplitudes`` (P, R, C) or flat; ``positions`` (P, 2) rows/columns in object pixels; ``obj`` (OR, OC) and
    ``probe`` (R, C) complex.  Returns ``(object, probe, errors)``, and the corrected positions (P, 2) as a fourth value
    when ``position_correction`` is given.
    """
    obj = np.array(obj, np.complex128)
    probe = np.array(probe, np.complex128)
    rows, columns = probe.shape
    n = rows * columns
    positions = np.asarray(positions, np.float64).reshape(-1, 2)
    count = len(positions)
    validate(amplitudes, positions, obj.shape, probe.shape, iterations, step_size, normalization_minimum,
             probe_amplitude_relative_radius, probe_amplitude_relative_width, probe_support_mask)
    limits = position_correction.pixel_distances() if position_correction is not None else None
    amp = np.asarray(amplitudes, np.float64).reshape(count, n)
    divisor = error_divisor(amp, count, error_normalization, mean_intensity)
    initial_aperture = np.abs(np.fft.fft2(probe)) if fix_probe_aperture else None
    object_rows, object_columns = obj.shape
    initial = positions.copy()
    initial_mean = (np.sum(initial[:, 0]) / count, np.sum(initial[:, 1]) / count)
    current = positions.copy()
    mask = None if probe_support_mask is None else np.asarray(probe_support_mask, bool).reshape(rows, columns)
    m = normalization_minimum
    errors = []
    o = obj.reshape(-1).copy()
    p = probe.copy()
    for it in range(iterations):
        rr = round_half_even(current[:, 0])
        cc = round_half_even(current[:, 1])
        dr = current[:, 0] - rr
        dc = current[:, 1] - cc
        idx = patch_indices(rows, columns, object_rows, object_columns, rr.astype(np.int64), cc.astype(np.int64))
        spectrum = np.fft.fft2(p)
        s = shifted_probes(spectrum, dr, dc).reshape(count, n)
        op = o[idx]
        psi = (s * op).reshape(count, rows, columns)
        f = np.fft.fft2(psi).reshape(count, n)
        mag = np.abs(f)
        error = float(np.sum((amp - mag) ** 2))
        with np.errstate(divide="ignore", invalid="ignore"):
            scale = np.where(mag > 0, amp / np.where(mag > 0, mag, 1.0), 0.0)
        proj = np.where(mag > 0, scale * f - f, amp + 0j)
        d = np.fft.ifft2(proj.reshape(count, rows, columns)).reshape(count, n)
        grad_o = np.zeros(o.size, np.complex128)
        pn = np.zeros(o.size)
        np.add.at(grad_o, idx.ravel(), (np.conj(s) * d).ravel())
        np.add.at(pn, idx.ravel(), (s.real ** 2 + s.imag ** 2).ravel())
        grad_p = np.sum(np.conj(op) * d, axis=0).reshape(rows, columns)
        on = np.sum(op.real ** 2 + op.imag ** 2, axis=0).reshape(rows, columns)
        max_pn, max_on = pn.max(), on.max()

        def inverse(local, maximum):
            return 1 / np.sqrt(1e-16 + ((1 - m) * local) ** 2 + (m * maximum) ** 2)

        before = o
        o = o + step_size * inverse(pn, max_pn) * grad_o
        if position_correction is not None:  # :371-377, with the updated object, before the amplitude cap
            current = position_update(before.reshape(object_rows, object_columns), o.reshape(object_rows, object_columns),
                                      spectrum, amp, current, initial, position_correction.step_size, limits)
        if constrain_object_amplitude or pure_phase_object:
            a = np.abs(o)
            target = np.ones_like(a) if pure_phase_object else np.minimum(a, 1.0)
            with np.errstate(divide="ignore", invalid="ignore"):
                o = np.where(a > 0, o * (target / np.where(a > 0, a, 1.0)), target + 0j)
        if not fix_probe:
            p = p + step_size * inverse(on, max_on) * grad_p
            if fix_probe_center_of_mass:
                p = center_of_mass_constraint(p)
            if fix_probe_aperture:
                p = aperture_constraint(p, initial_aperture)
            if constrain_probe_amplitude:
                p = amplitude_constraint(p, probe_amplitude_relative_radius, probe_amplitude_relative_width)
        if mask is not None:
            p = np.where(mask, p, 0)
        if position_correction is not None and position_correction.constrain_center_of_mass:  # :398-401
            mean = (np.sum(current[:, 0]) / count, np.sum(current[:, 1]) / count)
            current = np.stack([current[:, 0] - (mean[0] - initial_mean[0]),
                                current[:, 1] - (mean[1] - initial_mean[1])], axis=1)
        errors.append(error / divisor)
        if progress is not None:
            progress(it + 1, iterations)
    if position_correction is not None:
        return o.reshape(object_rows, object_columns), p, np.asarray(errors), current
    return o.reshape(object_rows, object_columns), p, np.asarray(errors)


# ---------------------------------------------------------------- mixed state (PtychographyEngines.swift)

def orthogonalize(probes):
    """``MixedstatePtychography.orthogonalize`` (``PtychographyEngines.swift:265-269,300-323``): the states become the
    eigenvectors of their Gram matrix ``G[i][j] = sum conj(p_i) p_j``, ``new_i = sum_j V[j][i] p_j``, by decreasing
    eigenvalue (ties: the later index first, NumPy's ascending argsort reversed).  Eigenvector phases are LAPACK's."""
    p = np.asarray(probes, np.complex128)
    states = p.shape[0]
    flat = p.reshape(states, -1)
    g = np.conj(flat) @ flat.T
    values, vectors = np.linalg.eigh(g)
    mixed = vectors.T @ flat
    order = sorted(range(states), key=lambda i: (-values[i], -i))
    return mixed[order].reshape(p.shape)


def initial_probes(first, count, seed):
    """``MixedstatePtychography.initialProbes`` (``PtychographyEngines.swift:270-298``): state 0 is ``first``; each further
    state is the previous one times exp(-2 pi i ((u - 1/2) f_row + (v - 1/2) f_col)), u then v drawn from
    ``np.random.RandomState(seed)``."""
    if not (0 < count < 4096):
        raise PtychographyError("count")
    first = np.asarray(first, np.complex128)
    rows, columns = first.shape
    rng = np.random.RandomState(seed)
    fr, fc = fftfreq_grid(rows, columns)
    out = [first]
    for _ in range(1, count):
        u, v = rng.rand(), rng.rand()
        phase = -2 * np.pi * (u - 0.5) * fr[:, None] - 2 * np.pi * (v - 0.5) * fc[None, :]
        out.append(out[-1] * (np.cos(phase) + 1j * np.sin(phase)))
    return np.stack(out)


def mixedstate_reconstruct(amplitudes, positions, obj, probes, iterations=8, step_size=0.5, normalization_minimum=1.0,
                           fix_probe=False, pure_phase_object=False, fix_probe_center_of_mass=False,
                           constrain_probe_amplitude=False, probe_amplitude_relative_radius=0.5,
                           probe_amplitude_relative_width=0.05, orthogonalize_probes=True, fix_probe_aperture=False,
                           probe_support_mask=None, error_normalization="suppliedAmplitudeEnergy", mean_intensity=None,
                           zero_pixel_error="reference"):
    """``MixedstatePtychography.reconstruct`` (``PtychographyEngines.swift:146-262``): several incoherent probe states on
    one object; the far-field intensity is the sum over states.  ``probes`` (S, R, C).  Returns ``(object, probes,
    errors)``."""
    obj = np.array(obj, np.complex128)
    p = np.array(probes, np.complex128)
    states, rows, columns = p.shape
    n = rows * columns
    positions = np.asarray(positions, np.float64).reshape(-1, 2)
    count = len(positions)
    validate(amplitudes, positions, obj.shape, (rows, columns), iterations, step_size, normalization_minimum,
             probe_amplitude_relative_radius, probe_amplitude_relative_width, probe_support_mask)
    amp = np.asarray(amplitudes, np.float64).reshape(count, n)
    divisor = error_divisor(amp, count, error_normalization, mean_intensity)
    initial_aperture = np.abs(np.fft.fft2(p[0])) if fix_probe_aperture else None
    object_rows, object_columns = obj.shape
    rr = round_half_even(positions[:, 0])
    cc = round_half_even(positions[:, 1])
    dr, dc = positions[:, 0] - rr, positions[:, 1] - cc
    idx = patch_indices(rows, columns, object_rows, object_columns, rr.astype(np.int64), cc.astype(np.int64))
    mask = None if probe_support_mask is None else np.asarray(probe_support_mask, bool).reshape(rows, columns)
    m = normalization_minimum
    o = obj.reshape(-1).copy()
    errors = []

    def norm(local, maximum):
        return 1 / np.sqrt(1e-16 + ((1 - m) * local) ** 2 + (m * maximum) ** 2)

    for it in range(iterations):
        op = o[idx]                                                   # (P, n)
        shifted = np.stack([shifted_probes(np.fft.fft2(p[s]), dr, dc).reshape(count, n) for s in range(states)])
        far = np.fft.fft2((shifted * op[None]).reshape(states, count, rows, columns)).reshape(states, count, n)
        intensity = np.sum(far.real ** 2 + far.imag ** 2, axis=0)     # (P, n)
        amplitude = np.sqrt(intensity)
        zero = amplitude == 0
        with np.errstate(divide="ignore", invalid="ignore"):
            factor = np.where(zero, 0.0, amp / np.where(zero, 1.0, amplitude) - 1)
        terms = np.where(zero, np.inf if zero_pixel_error == "reference" else amp * amp, (amp - amplitude) ** 2)
        error = float(np.sum(terms))
        e = np.fft.ifft2((far * factor[None]).reshape(states, count, rows, columns)).reshape(states, count, n)
        grad_o = np.zeros(o.size, np.complex128)
        pn = np.zeros(o.size)
        np.add.at(grad_o, idx.ravel(), np.sum(np.conj(shifted) * e, axis=0).ravel())
        np.add.at(pn, idx.ravel(), np.sum(shifted.real ** 2 + shifted.imag ** 2, axis=0).ravel())
        grad_p = np.sum(np.conj(op)[None] * e, axis=1).reshape(states, rows, columns)
        on = np.sum(op.real ** 2 + op.imag ** 2, axis=0).reshape(rows, columns)
        o = o + step_size * norm(pn, pn.max()) * grad_o
        a = np.abs(o)                                                 # the threshold, always (:112-116)
        target = np.ones_like(a) if pure_phase_object else np.minimum(a, 1.0)
        ph = np.arctan2(o.imag, o.real)
        o = target * np.cos(ph) + 1j * target * np.sin(ph)
        if not fix_probe:
            p = p + step_size * norm(on, on.max())[None] * grad_p
            if fix_probe_center_of_mass:
                com = probe_center_of_mass(p[0])
                if com is not None:
                    p = np.stack([fourier_shift(p[s], -com[0], -com[1]) for s in range(states)])
            if fix_probe_aperture:
                p[0] = aperture_constraint(p[0], initial_aperture)
            if constrain_probe_amplitude:
                p = np.stack([amplitude_constraint(p[s], probe_amplitude_relative_radius,
                                                   probe_amplitude_relative_width) for s in range(states)])
        if mask is not None:
            p = np.where(mask[None], p, 0)
        if orthogonalize_probes and states > 1:
            p = orthogonalize(p)
        errors.append(error / divisor)
    return o.reshape(object_rows, object_columns), p, np.asarray(errors)


# ---------------------------------------------------------------- multislice (PtychographyEngines.swift)

def propagators(rows, columns, row_sampling, column_sampling, wavelength, slice_thicknesses):
    """``MultislicePtychography.propagators`` (``PtychographyEngines.swift:427-442``): exp(-i pi lambda dz (kr^2 + kc^2))
    with k = frequency / sampling, one (rows, columns) grid per thickness."""
    ok = (rows > 1 and columns > 1 and math.isfinite(row_sampling) and row_sampling > 0
          and math.isfinite(column_sampling) and column_sampling > 0 and math.isfinite(wavelength) and wavelength > 0
          and len(slice_thicknesses) > 0 and all(math.isfinite(d) for d in slice_thicknesses))
    if not ok:
        raise PtychographyError("propagators")
    fr, fc = fftfreq_grid(rows, columns)
    k2 = (fr / row_sampling)[:, None] ** 2 + (fc / column_sampling)[None, :] ** 2
    out = []
    for dz in slice_thicknesses:
        phase = -np.pi * wavelength * dz * k2
        out.append(np.cos(phase) + 1j * np.sin(phase))
    return np.stack(out)


def multislice_reconstruct(amplitudes, positions, obj, probe, slice_thicknesses, wavelength, row_sampling,
                           column_sampling, iterations=8, step_size=0.5, normalization_minimum=1.0, fix_probe=False,
                           pure_phase_object=False, identical_slices=False, fix_probe_center_of_mass=False,
                           constrain_probe_amplitude=False, probe_amplitude_relative_radius=0.5,
                           probe_amplitude_relative_width=0.05, fix_probe_aperture=False, probe_support_mask=None,
                           error_normalization="suppliedAmplitudeEnergy", mean_intensity=None):
    """``MultislicePtychography.reconstruct`` (``PtychographyEngines.swift:458-588``): ``obj`` (L, OR, OC) slices,
    entrance first; ``slice_thicknesses`` L - 1 values (A).  Returns ``(slices, probe, errors)``."""
    obj = np.array(obj, np.complex128)
    probe = np.array(probe, np.complex128)
    slices, object_rows, object_columns = obj.shape
    rows, columns = probe.shape
    n = rows * columns
    positions = np.asarray(positions, np.float64).reshape(-1, 2)
    count = len(positions)
    validate(amplitudes, positions, (object_rows, object_columns), probe.shape, iterations, step_size,
             normalization_minimum, probe_amplitude_relative_radius, probe_amplitude_relative_width,
             probe_support_mask)
    if len(slice_thicknesses) != slices - 1:
        raise PtychographyError("slice thicknesses")
    amp = np.asarray(amplitudes, np.float64).reshape(count, n)
    divisor = error_divisor(amp, count, error_normalization, mean_intensity)
    props = propagators(rows, columns, row_sampling, column_sampling, wavelength,
                        list(slice_thicknesses) if len(slice_thicknesses) else [0.0])
    initial_aperture = np.abs(np.fft.fft2(probe)) if fix_probe_aperture else None
    rr = round_half_even(positions[:, 0])
    cc = round_half_even(positions[:, 1])
    dr, dc = positions[:, 0] - rr, positions[:, 1] - cc
    idx = patch_indices(rows, columns, object_rows, object_columns, rr.astype(np.int64), cc.astype(np.int64))
    mask = None if probe_support_mask is None else np.asarray(probe_support_mask, bool).reshape(rows, columns)
    m = normalization_minimum
    o = obj.reshape(slices, -1).copy()
    p = probe.copy()
    errors = []

    def norm(local, maximum):
        return 1 / np.sqrt(1e-16 + ((1 - m) * local) ** 2 + (m * maximum) ** 2)

    def propagate(x, s, conjugate):
        f = np.fft.fft2(x.reshape(count, rows, columns))
        f = f * (np.conj(props[s]) if conjugate else props[s])[None]
        return np.fft.ifft2(f).reshape(count, n)

    for it in range(iterations):
        current = shifted_probes(np.fft.fft2(p), dr, dc).reshape(count, n)
        waves, patches = [], []
        for s in range(slices):                                        # :503-515
            waves.append(current)
            patch = o[s][idx]
            patches.append(patch)
            exit_wave = current * patch
            if s + 1 < slices:
                current = propagate(exit_wave, s, False)
        f = np.fft.fft2(exit_wave.reshape(count, rows, columns)).reshape(count, n)
        magnitude = np.abs(f)
        error = float(np.sum((amp - magnitude) ** 2))
        angle = np.arctan2(f.imag, f.real)
        chi = np.fft.ifft2((amp * np.cos(angle) - f.real + 1j * (amp * np.sin(angle) - f.imag))
                           .reshape(count, rows, columns)).reshape(count, n)
        grads, weights = [None] * slices, [None] * slices
        for s in range(slices - 1, -1, -1):                            # :526-545
            g = np.zeros(object_rows * object_columns, np.complex128)
            w = np.zeros(object_rows * object_columns)
            np.add.at(g, idx.ravel(), (np.conj(waves[s]) * chi).ravel())
            np.add.at(w, idx.ravel(), (waves[s].real ** 2 + waves[s].imag ** 2).ravel())
            grads[s], weights[s] = g, w
            chi = chi * np.conj(patches[s])
            if s > 0:
                chi = propagate(chi, s - 1, True)
        grad_p = np.sum(chi, axis=0).reshape(rows, columns)
        on = np.sum(patches[0].real ** 2 + patches[0].imag ** 2, axis=0).reshape(rows, columns)
        for s in range(slices):
            o[s] = o[s] + step_size * norm(weights[s], weights[s].max()) * grads[s]
        if not fix_probe:
            p = p + step_size * norm(on, on.max()) * grad_p
        if identical_slices:
            o[:] = np.sum(o, axis=0) / slices
        a = np.abs(o)
        target = np.ones_like(a) if pure_phase_object else np.minimum(a, 1.0)
        ph = np.arctan2(o.imag, o.real)
        o = target * np.cos(ph) + 1j * target * np.sin(ph)
        if not fix_probe:
            if fix_probe_center_of_mass:
                p = center_of_mass_constraint(p)
            if fix_probe_aperture:
                p = aperture_constraint(p, initial_aperture)
            if constrain_probe_amplitude:
                p = amplitude_constraint(p, probe_amplitude_relative_radius, probe_amplitude_relative_width)
        if mask is not None:
            p = np.where(mask, p, 0)
        errors.append(error / divisor)
    return o.reshape(slices, object_rows, object_columns), p, np.asarray(errors)


def loss_and_gradients(amplitudes, positions, obj, probe):
    """The real loss ``L = sum_p sum_k (|F_k| - A_k)^2`` and its gradients, for INTEGER positions.

    With the unnormalised forward FFT, ``dL/dRe O + i dL/dIm O = -2 n * sum_p conj(S) dpsi`` and likewise for the probe
    with ``conj(O) dpsi`` (the accumulations of ``Ptychography.swift:351-358``).  Returns ``(L, gO, gP)``.
    """
    obj = np.asarray(obj, np.complex128)
    probe = np.asarray(probe, np.complex128)
    rows, columns = probe.shape
    n = rows * columns
    positions = np.asarray(positions, np.float64).reshape(-1, 2)
    count = len(positions)
    amp = np.asarray(amplitudes, np.float64).reshape(count, n)
    rr = round_half_even(positions[:, 0]).astype(np.int64)
    cc = round_half_even(positions[:, 1]).astype(np.int64)
    idx = patch_indices(rows, columns, obj.shape[0], obj.shape[1], rr, cc)
    o = obj.reshape(-1)
    s = np.broadcast_to(probe.reshape(1, n), (count, n))
    op = o[idx]
    f = np.fft.fft2((s * op).reshape(count, rows, columns)).reshape(count, n)
    mag = np.abs(f)
    loss = float(np.sum((mag - amp) ** 2))
    with np.errstate(divide="ignore", invalid="ignore"):
        scale = np.where(mag > 0, amp / np.where(mag > 0, mag, 1.0), 0.0)
    proj = np.where(mag > 0, scale * f - f, amp + 0j)
    d = np.fft.ifft2(proj.reshape(count, rows, columns)).reshape(count, n)
    go = np.zeros(o.size, np.complex128)
    np.add.at(go, idx.ravel(), (np.conj(s) * d).ravel())
    gp = np.sum(np.conj(op) * d, axis=0)
    return loss, (-2 * n * go).reshape(obj.shape), (-2 * n * gp).reshape(rows, columns)


# ---------------------------------------------------------------------------------------------------- preprocessing

@dataclass
class PreparedAmplitudes:
    """``PtychographyAmplitudes`` (``PtychographyPreparation.swift:62-75``)."""
    values: np.ndarray            # [position][row][column], sqrt(max(shifted, 0))
    mean_intensity: float         # mean over positions of the summed shifted intensity, negatives included
    clipped_mean_intensity: float  # the same with negative shifted values set to zero first


def _bilinear_shift(p, origin_row, origin_column):
    """``shiftPattern(.bilinear)`` (``PtychographyPreparation.swift:301-315``): out[i, j] = p[i + origin_row,
    j + origin_column], bilinear, wrapped."""
    rows, columns = p.shape
    xr = np.arange(rows) + origin_row
    fr = np.floor(xr)
    tr = (xr - fr)[:, None]
    r0 = np.mod(fr.astype(np.int64), rows)
    r1 = np.mod(fr.astype(np.int64) + 1, rows)
    xc = np.arange(columns) + origin_column
    fc = np.floor(xc)
    tc = (xc - fc)[None, :]
    c0 = np.mod(fc.astype(np.int64), columns)
    c1 = np.mod(fc.astype(np.int64) + 1, columns)
    return (p[np.ix_(r0, c0)] * (1 - tr) * (1 - tc) + p[np.ix_(r1, c0)] * tr * (1 - tc)
            + p[np.ix_(r0, c1)] * (1 - tr) * tc + p[np.ix_(r1, c1)] * tr * tc)


def _cubic_weights(origin, n):
    """Per output index i: the four wrapped taps floor(x) - 1 .. floor(x) + 2 of x = i + origin and the cubic B-spline
    weights of the fraction (``PtychographyPreparation.swift:330-334``)."""
    x = np.arange(n) + origin
    f = np.floor(x)
    t = x - f
    w = np.stack([(1 - t) ** 3 / 6, (3 * t ** 3 - 6 * t ** 2 + 4) / 6, (-3 * t ** 3 + 3 * t ** 2 + 3 * t + 1) / 6,
                  t ** 3 / 6], axis=1)
    idx = np.mod(f.astype(np.int64)[:, None] + np.arange(-1, 3)[None, :], n)
    return idx, w


def _cubic_spline_shift(p, origin_row, origin_column):
    """``shiftPattern(.cubicSpline)`` (``PtychographyPreparation.swift:317-342``): periodic cubic B-spline coefficients
    by division in Fourier space (the kernel's DFT is (4 + 2 cos(2 pi k / n)) / 6 per axis), then 4 x 4 taps."""
    rows, columns = p.shape
    hr = (4 + 2 * np.cos(2 * np.pi * np.arange(rows) / rows)) / 6
    hc = (4 + 2 * np.cos(2 * np.pi * np.arange(columns) / columns)) / 6
    coef = np.fft.ifft2(np.fft.fft2(p) / (hr[:, None] * hc[None, :])).real
    ri, rw = _cubic_weights(origin_row, rows)
    ci, cw = _cubic_weights(origin_column, columns)
    out = np.zeros((rows, columns))
    for a in range(4):
        for b in range(4):
            out += rw[:, a][:, None] * cw[:, b][None, :] * coef[np.ix_(ri[:, a], ci[:, b])]
    return out


def prepare_amplitudes(cube, origin_rows, origin_columns, shift="cubicSpline"):
    """``PtychographyPreparation.amplitudes(from:origins:shift:)`` (``PtychographyPreparation.swift:142-183``).

    ``cube`` is ``[position][row][column]`` (Float32 values, taken to Double); ``origin_rows/columns`` one origin per
    position (a uniform origin repeated).  Each pattern is shifted so its origin sits on the corner, and the result is
    ``sqrt(max(shifted, 0))`` with the mean intensities over positions (unclipped and clipped)."""
    cube = np.asarray(cube, np.float32).astype(np.float64)
    if cube.ndim != 3:
        raise PtychographyError("cube must be [position][row][column]")
    count, rows, columns = cube.shape
    origin_rows = np.asarray(origin_rows, np.float64).ravel()
    origin_columns = np.asarray(origin_columns, np.float64).ravel()
    if not (count > 0 and rows > 1 and columns > 1):
        raise PtychographyError("cube shape")
    if origin_rows.size != count or origin_columns.size != count:
        raise PtychographyError("one origin per position")
    for o in (origin_rows, origin_columns):
        if not (np.all(np.isfinite(o)) and np.all(np.abs(o) < 1e9)):
            raise PtychographyError("origin")
    if not np.all(np.isfinite(cube)):
        raise PtychographyError("cube value not finite")
    if shift not in ("bilinear", "cubicSpline"):
        raise PtychographyError("shift")
    fn = _bilinear_shift if shift == "bilinear" else _cubic_spline_shift
    out = np.empty_like(cube)
    total = clipped = 0.0
    for i in range(count):
        shifted = fn(cube[i], origin_rows[i], origin_columns[i])
        total += float(shifted.sum())
        clipped += float(np.maximum(shifted, 0).sum())
        out[i] = np.sqrt(np.maximum(shifted, 0))
    return PreparedAmplitudes(out, total / count, clipped / count)
