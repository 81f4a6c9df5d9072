"""Seeded synthetic single-slice ptychography datasets (no public dataset is involved).

Recipe: a unit-amplitude object whose phase is a periodic Gaussian-filtered (sigma = 3 px) field of seeded standard
normals, min-max scaled to [0, phase_range] rad; a probe from PtychographyProbe.build (on the device, FP64) at the given
voltage, aperture, rolloff and defocus, scaled so each noise-free pattern holds `dose` electrons
(sum |fft2(P)|^2 = n sum |P|^2 = dose, the energy scaling of PtychographyPreparation.initialProbe); an integer raster of
`step` px starting at (R/2, C/2); amplitudes sqrt(Poisson(|fft2(P * O[patch])|^2)) in Float32; and a start object of
unit amplitude with a seeded weak phase N(0, 0.02 rad).

The angular sampling is 64/N mrad per detector pixel, so the object pixel is wavelength / (dk N) = 0.3076 A at 300 kV for
every detector size N.  The far-field synthesis runs on the GPU with torch (input generation, outside every timed
region).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .ptycho import PtychographyProbe, electron_wavelength


@dataclass
class Dataset:
    amplitudes: np.ndarray      # (P, R, C) float32
    positions: np.ndarray       # (P, 2) float64
    object_start: np.ndarray    # (OR, OC) complex128
    probe: np.ndarray           # (R, C) complex128
    truth: np.ndarray           # (OR, OC) complex128
    config: dict


def phase_field(rows, columns, seed, sigma=3.0, phase_range=0.5):
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal((rows, columns))
    ky = np.fft.fftfreq(rows)[:, None]
    kx = np.fft.fftfreq(columns)[None, :]
    field = np.real(np.fft.ifft2(np.fft.fft2(noise) * np.exp(-2 * (np.pi * sigma) ** 2 * (ky ** 2 + kx ** 2))))
    return (field - field.min()) / (field.max() - field.min()) * phase_range


def probe(n, kv=300.0, cutoff_mrad=20.0, rolloff_mrad=2.0, defocus=100.0, dose=1e5, device=0):
    wavelength = electron_wavelength(kv * 1e3)
    dk = 64.0 / n * 1e-3  # rad per detector pixel
    sampling = wavelength / (dk * n)
    p = PtychographyProbe.build(n, n, sampling, sampling, wavelength, cutoff_mrad * 1e-3, rolloff_mrad * 1e-3,
                                defocus=defocus, device=device)
    return p * np.sqrt(dose / (n * n * np.sum(np.abs(p) ** 2))), sampling


def raster(scan, n, step=4):
    return np.array([[n // 2 + step * i, n // 2 + step * j] for i in range(scan) for j in range(scan)], np.float64)


def amplitudes_torch(probe_arr, truth, positions, seed, batch=2048, pinned=False, device=0):
    """sqrt(Poisson(|fft2(P * O[patch])|^2)) in Float32 for every position (torch on the GPU)."""
    import torch
    dev = torch.device(f"cuda:{device}")
    R, C = probe_arr.shape
    OR, OC = truth.shape
    P = len(positions)
    out = torch.empty((P, R, C), dtype=torch.float32, pin_memory=pinned)
    pr = torch.as_tensor(probe_arr, dtype=torch.complex128, device=dev)
    ob = torch.as_tensor(truth, dtype=torch.complex128, device=dev).reshape(-1)
    ro = torch.arange(R, device=dev)
    ro = torch.where(ro < (R + 1) // 2, ro, ro - R)
    co = torch.arange(C, device=dev)
    co = torch.where(co < (C + 1) // 2, co, co - C)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    pos = torch.as_tensor(np.round(positions).astype(np.int64), device=dev)
    for b in range(0, P, batch):
        e = min(P, b + batch)
        rr = torch.remainder(pos[b:e, 0, None] + ro[None, :], OR)
        cc = torch.remainder(pos[b:e, 1, None] + co[None, :], OC)
        idx = rr[:, :, None] * OC + cc[:, None, :]
        wave = pr[None] * ob[idx]
        inten = torch.abs(torch.fft.fft2(wave)) ** 2
        counts = torch.poisson(inten, generator=gen)
        out[b:e] = torch.sqrt(counts).to(torch.float32).cpu()
    return out


def dataset(scan, n, dose=1e5, step=4, seed_object=1, seed_noise=2, seed_start=3, defocus=100.0, pinned=False, device=0):
    size = scan * step + n
    truth = np.exp(1j * phase_field(size, size, seed_object))
    prb, sampling = probe(n, dose=dose, defocus=defocus, device=device)
    positions = raster(scan, n, step)
    amps = amplitudes_torch(prb, truth, positions, seed_noise, pinned=pinned, device=device)
    rng = np.random.default_rng(seed_start)
    start = np.exp(1j * rng.normal(0, 0.02, (size, size)))
    return Dataset(amps.numpy(), positions, start, prb, truth,
                   dict(scan=scan, detector=n, object=size, dose=dose, step=step, sampling_A=sampling,
                        defocus_A=defocus, kv=300, cutoff_mrad=20, rolloff_mrad=2))
