"""The allocation-free loss entry point, through the C ABI, against the FP64 oracle and the allocating engine.

``cubo_ptycho_loss_fp32_noalloc`` serves callers that cannot call cudaMalloc: an application whose device memory is
owned by its own pool allocator, or a loop that must not allocate while it runs.  Its only scratch is a fixed device
array inside the library.  These tests give it device buffers (allocated here by the test, as such a caller's allocator
would) and check its loss, on two calls in a row (the second call reuses the scratch array the first one left filled),
within the relative 1e-5 the FP32-form tests use for errors, against:

- the FP64 NumPy oracle's loss ``sum (|F| - A)^2`` (``numpy_oracle.loss_and_gradients``, the squared amplitude residual
  of Ptychography.swift:338-342), on a power-of-two detector, a non-power-of-two one (48 x 40) and one whose lengths
  have prime factors the shared-memory transform takes by direct DFT (22 x 21), with scan centres that are negative or
  beyond the object (wrapped periodically);
- the first-iteration residual of ``cubo_ptycho_reconstruct`` times that call's normalisation.

This file is named so pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from tests import scenes

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _loss_twice(amps, rows_c, cols_c, obj, probe):
    """Two calls of the entry point in a row on the same inputs; returns both losses."""
    import torch

    from cubokit_b200 import _lib

    lib = _lib.load()
    dev = torch.device("cuda", 0)
    d_amps = torch.as_tensor(np.ascontiguousarray(amps, np.float32), device=dev).contiguous()
    d_rows = torch.as_tensor(np.asarray(rows_c, np.int32), device=dev)
    d_cols = torch.as_tensor(np.asarray(cols_c, np.int32), device=dev)
    d_obj = torch.as_tensor(np.stack([obj.real, obj.imag], -1).astype(np.float32), device=dev).contiguous()
    d_probe = torch.as_tensor(np.stack([probe.real, probe.imag], -1).astype(np.float32), device=dev).contiguous()
    R, Cn = probe.shape
    OR, OC = obj.shape
    out = []
    for call in range(2):
        d_loss = torch.full((1,), -1.0, dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        st = lib.cubo_ptycho_loss_fp32_noalloc(R, Cn, OR, OC, len(rows_c), _ptr(d_amps), _ptr(d_rows), _ptr(d_cols),
                                                _ptr(d_obj), _ptr(d_probe), _ptr(d_loss), None)
        assert st == 0, (call, st)
        torch.cuda.synchronize()
        out.append(float(d_loss.item()))
    return out


def _scene(rows, columns, object_rows, object_columns, centres, seed):
    """A smooth random object, a Gaussian-windowed random-phase probe and amplitudes of a perturbed truth with 10 %
    multiplicative noise, so that the residual is far above FP32 round-off."""
    rng = np.random.default_rng(seed)
    y, x = np.indices((object_rows, object_columns))
    obj = (0.9 + 0.1 * np.cos(y / 5.0)) * np.exp(1j * (0.4 * np.sin(x / 7.0) + 0.2 * np.cos((x + y) / 9.0)))
    r = np.minimum(np.arange(rows), rows - np.arange(rows))[:, None]
    c = np.minimum(np.arange(columns), columns - np.arange(columns))[None, :]
    probe = np.exp(-(r * r / (rows * rows / 12.0) + c * c / (columns * columns / 12.0))) * np.exp(
        1j * rng.uniform(-0.3, 0.3, (rows, columns)))
    truth = obj * np.exp(1j * 0.05 * rng.standard_normal(obj.shape))
    from oracle import numpy_oracle as no
    rr = np.array([p[0] for p in centres], np.int64)
    cc = np.array([p[1] for p in centres], np.int64)
    idx = no.patch_indices(rows, columns, object_rows, object_columns, rr, cc)
    f = np.fft.fft2((probe.reshape(1, -1) * truth.reshape(-1)[idx]).reshape(len(rr), rows, columns))
    amps = (np.abs(f) * (1 + 0.1 * rng.standard_normal(f.shape))).clip(min=0)
    return amps.astype(np.float32), rr, cc, obj, probe


@pytest.mark.parametrize("rows,columns", [(32, 32), (48, 40), (22, 21)])
def test_noalloc_loss_matches_the_fp64_oracle_on_two_calls(rows, columns):
    from oracle import numpy_oracle as no

    OR, OC = 3 * rows, 2 * columns + 5
    # interior centres, negative ones and ones beyond the object: the window wraps periodically
    centres = [(OR // 2, OC // 2), (-3, 5), (OR + 7, -(OC + 2)), (2, OC - 1), (-(2 * OR) - 1, 3 * OC + 4),
               (OR // 3, OC // 4)]
    amps, rr, cc, obj, probe = _scene(rows, columns, OR, OC, centres, seed=rows * 100 + columns)
    expected, _, _ = no.loss_and_gradients(amps.astype(np.float64), np.stack([rr, cc], -1).astype(np.float64),
                                           obj.astype(np.complex64).astype(np.complex128),
                                           probe.astype(np.complex64).astype(np.complex128))
    for call, got in enumerate(_loss_twice(amps, rr, cc, obj, probe)):
        assert abs(got - expected) <= 1e-5 * abs(expected), (rows, columns, call, got, expected)


def test_noalloc_loss_matches_reconstruct_on_two_calls():
    import cubokit_b200 as cb

    s = scenes.raster_scene(scan=8, det=32, step=4, seed=21)
    amps = s["amplitudes"].astype(np.float32)
    obj = s["object"]
    probe = s["probe"]
    ref = cb.SingleslicePtychography.reconstruct(amps, s["positions"], obj, probe, iterations=1)
    expected = float(ref.errors[0]) * float(np.sum(amps.astype(np.float64) ** 2))
    rows_c = np.round(s["positions"][:, 0]).astype(np.int32)
    cols_c = np.round(s["positions"][:, 1]).astype(np.int32)
    for call, got in enumerate(_loss_twice(amps, rows_c, cols_c, obj, probe)):
        assert abs(got - expected) <= 1e-5 * abs(expected), (call, got, expected)


def test_noalloc_refuses_sizes_beyond_its_scratch_and_misaligned_buffers():
    from cubokit_b200 import _lib

    lib = _lib.load()
    dummy = C.c_void_p(16)  # never dereferenced: the checks come before any launch
    st = lib.cubo_ptycho_loss_fp32_noalloc(32, 32, 64, 64, (1 << 20) + 1, dummy, dummy, dummy, dummy, dummy, dummy, None)
    assert st == _lib.INVALID_INPUT
    odd = C.c_void_p(20)  # 4-byte but not 8-byte aligned: not a complex64 or double address
    st = lib.cubo_ptycho_loss_fp32_noalloc(32, 32, 64, 64, 4, dummy, dummy, dummy, odd, dummy, dummy, None)
    assert st == _lib.INVALID_INPUT
    st = lib.cubo_ptycho_loss_fp32_noalloc(2, 8193, 64, 8200, 4, dummy, dummy, dummy, dummy, dummy, dummy, None)
    assert st == _lib.UNSUPPORTED
