"""Well-conditioned synthetic scenes for precision-agreement tests.

Restated from the scenes CuboKit uses to hold its Float32 engine to its Double engine
(``Tests/CuboPtychoTests/SinglePrecisionTests.swift:16-56`` and ``:160-199``): amplitudes are the exact forward model of
a known smooth phase object read through a known probe, so the iteration is consistent and converges.  The forward
model here uses ``np.fft`` in double (the reference test uses a naive DFT; both are the same transform).
"""
from __future__ import annotations

import numpy as np


def frequency(k, n):
    k = np.asarray(k)
    return np.where(k < (n + 1) // 2, k, k - n) / n


def _patch(rows, columns, size, rr, cc):
    ro = np.arange(rows)
    ro = np.where(ro < (rows + 1) // 2, ro, ro - rows)
    co = np.arange(columns)
    co = np.where(co < (columns + 1) // 2, co, co - columns)
    r = np.mod(rr + ro, size)
    c = np.mod(cc + co, size)
    return r[:, None] * size + c[None, :]


def gaussian_scene(d=32, size=80, count=36):
    """``SinglePrecisionTests.scene``: d x d Gaussian probe (unit norm), 0.9-amplitude smooth phase truth, a 6 x 6 integer
    raster with pitch 8 starting at 20, unit start object."""
    r = np.arange(d)
    rr = np.minimum(r, d - r).astype(np.float64)
    probe = np.exp(-(rr[:, None] ** 2 + rr[None, :] ** 2) / 40)
    probe = probe / np.sqrt(np.sum(probe ** 2))
    y, x = np.indices((size, size)).astype(np.float64)
    phase = 0.6 * np.sin(y / 9) * np.cos(x / 7) + 0.3 * np.sin((y + x) / 5)
    truth = 0.9 * np.exp(1j * phase)
    positions = np.array([[20 + (i // 6) * 8, 20 + (i % 6) * 8] for i in range(count)], np.float64)
    amps = np.empty((count, d, d))
    flat = truth.ravel()
    for p in range(count):
        idx = _patch(d, d, size, int(positions[p, 0]), int(positions[p, 1]))
        amps[p] = np.abs(np.fft.fft2(probe * flat[idx]))
    return dict(amplitudes=amps, positions=positions, object=np.ones((size, size), np.complex128),
                probe=probe.astype(np.complex128), truth=truth)


def nonsquare_scene(rows=32, columns=48, size=96):
    """``SinglePrecisionNonSquareTests.agreesWithDouble``: a complex Gaussian probe, 12 fractional positions (pitches
    7.37 and 9.61), amplitudes from the Fourier-shifted probe times the truth."""
    r = np.arange(rows)
    c = np.arange(columns)
    rr = np.minimum(r, rows - r).astype(np.float64)[:, None]
    cc = np.minimum(c, columns - c).astype(np.float64)[None, :]
    g = np.exp(-(rr * rr / 20 + cc * cc / 60))
    probe = g + 1j * (0.04 * rr * g)
    probe = probe / np.sqrt(np.sum(np.abs(probe) ** 2))
    y, x = np.indices((size, size)).astype(np.float64)
    ph = 0.5 * np.sin(y / 6) * np.cos(x / 11) + 0.2 * np.sin((y + 2 * x) / 8)
    truth = 0.9 * np.exp(1j * ph)
    positions = np.array([[30 + (i // 4) * 7.37, 30 + (i % 4) * 9.61] for i in range(12)])
    spectrum = np.fft.fft2(probe)
    fr = frequency(np.arange(rows), rows)[:, None]
    fc = frequency(np.arange(columns), columns)[None, :]
    amps = np.empty((len(positions), rows, columns))
    flat = truth.ravel()
    for p, (pr, pc) in enumerate(positions):
        rr0, cc0 = np.round(pr), np.round(pc)
        dr, dc = pr - rr0, pc - cc0
        a = -2 * np.pi * (fr * dr + fc * dc)
        s = np.fft.ifft2(spectrum * (np.cos(a) + 1j * np.sin(a)))
        idx = _patch(rows, columns, size, int(rr0), int(cc0))
        amps[p] = np.abs(np.fft.fft2(s * flat[idx]))
    return dict(amplitudes=amps, positions=positions, object=np.ones((size, size), np.complex128), probe=probe,
                truth=truth)


def raster_scene(scan=8, det=32, step=4, seed=11, phase_range=0.5, weak_phase=0.02, shape=None):
    """A small raster scene in the style of the benchmark recipe: integer raster positions with ``step`` px pitch starting
    at (det/2, det/2), an object of side ``scan*step + det`` whose truth is a smooth seeded phase (0..phase_range rad),
    a band-limited Gaussian-aperture probe, noise-free amplitudes, and a start object with a weak seeded random phase."""
    rng = np.random.default_rng(seed)
    rows, columns = (det, det) if shape is None else shape
    size_r = scan * step + rows
    size_c = scan * step + columns
    noise = rng.standard_normal((size_r, size_c))
    ky = frequency(np.arange(size_r), size_r)[:, None]
    kx = frequency(np.arange(size_c), size_c)[None, :]
    sigma = 3.0
    field = np.real(np.fft.ifft2(np.fft.fft2(noise) * np.exp(-2 * (np.pi * sigma) ** 2 * (ky ** 2 + kx ** 2))))
    field = (field - field.min()) / (field.max() - field.min()) * phase_range
    truth = np.exp(1j * field)
    fr = frequency(np.arange(rows), rows)[:, None]
    fc = frequency(np.arange(columns), columns)[None, :]
    q = np.hypot(fr, fc)
    aperture = 0.5 * (1 - np.tanh((q - 0.2) / 0.02))
    probe = np.fft.ifft2(aperture * np.exp(-1j * 40.0 * q ** 2))
    probe = probe / np.sqrt(np.sum(np.abs(probe) ** 2)) * np.sqrt(1e4 / (rows * columns))
    positions = np.array([[rows // 2 + step * i, columns // 2 + step * j] for i in range(scan) for j in range(scan)],
                         np.float64)
    flat = truth.ravel()
    amps = np.empty((len(positions), rows, columns))
    for p, (pr, pc) in enumerate(positions):
        ro = np.arange(rows)
        ro = np.where(ro < (rows + 1) // 2, ro, ro - rows)
        co = np.arange(columns)
        co = np.where(co < (columns + 1) // 2, co, co - columns)
        idx = (np.mod(int(pr) + ro, size_r)[:, None] * size_c + np.mod(int(pc) + co, size_c)[None, :])
        amps[p] = np.abs(np.fft.fft2(probe * flat[idx]))
    start = np.exp(1j * rng.normal(0, weak_phase, (size_r, size_c)))
    return dict(amplitudes=amps.astype(np.float32).astype(np.float64), positions=positions, object=start, probe=probe,
                truth=truth)
