"""The allocation-free loss entry point against the allocating one, through the C ABI.

``cubo_ptycho_loss_fp32_noalloc`` serves callers that cannot call cudaMalloc: an application whose device memory is
owned by its own pool allocator, or a loop that must not allocate while it runs.  Its only scratch is a fixed device
array inside the library.  This test gives it device buffers (allocated here by the test, as such a caller's allocator
would) and checks its loss against the first-iteration residual of ``cubo_ptycho_reconstruct`` times that call's
normalisation, within the relative 1e-5 the FP32-form tests use for errors, on two calls in a row (the second call
reuses the scratch array the first one left filled).  This file is named so pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from tests import scenes

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def test_noalloc_loss_matches_reconstruct_on_two_calls():
    import torch

    import cubokit_b200 as cb
    from cubokit_b200 import _lib

    s = scenes.raster_scene(scan=8, det=32, step=4, seed=21)
    amps = s["amplitudes"].astype(np.float32)
    obj = s["object"]
    probe = s["probe"]
    ref = cb.SingleslicePtychography.reconstruct(amps, s["positions"], obj, probe, iterations=1)
    expected = float(ref.errors[0]) * float(np.sum(amps.astype(np.float64) ** 2))

    lib = _lib.load()
    dev = torch.device("cuda", 0)
    d_amps = torch.as_tensor(amps, device=dev).contiguous()
    d_rows = torch.as_tensor(np.round(s["positions"][:, 0]).astype(np.int32), device=dev)
    d_cols = torch.as_tensor(np.round(s["positions"][:, 1]).astype(np.int32), device=dev)
    d_obj = torch.as_tensor(np.stack([obj.real, obj.imag], -1).astype(np.float32), device=dev).contiguous()
    d_probe = torch.as_tensor(np.stack([probe.real, probe.imag], -1).astype(np.float32), device=dev).contiguous()
    R, Cn = probe.shape
    OR, OC = obj.shape
    for call in range(2):
        d_loss = torch.full((1,), -1.0, dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        st = lib.cubo_ptycho_loss_fp32_noalloc(R, Cn, OR, OC, len(s["positions"]), _ptr(d_amps), _ptr(d_rows),
                                                _ptr(d_cols), _ptr(d_obj), _ptr(d_probe), _ptr(d_loss), None)
        assert st == 0, (call, st)
        torch.cuda.synchronize()
        got = float(d_loss.item())
        assert abs(got - expected) <= 1e-5 * abs(expected), (call, got, expected)


def test_noalloc_refuses_sizes_beyond_its_scratch():
    from cubokit_b200 import _lib

    lib = _lib.load()
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    st = lib.cubo_ptycho_loss_fp32_noalloc(32, 32, 64, 64, (1 << 20) + 1, dummy, dummy, dummy, dummy, dummy, dummy, None)
    assert st == _lib.INVALID_INPUT
