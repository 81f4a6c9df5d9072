"""The tcgen05 helpers (cubokit_b200/csrc/umma.cuh) on a B200: one complex 128 x 128 x 128 split-BF16 product.

The harness (tests/cuda/umma_probe.cu) keeps W in tensor memory (A operand) and B in shared memory (B operand, K-major or
MN-major), exactly as the split-BF16 DFT kernel does.  Expected values are the FP64 sums of the same three bf16 split
products (hi*hi + hi*lo + lo*hi); the tensor core accumulates in FP32, so the bound is FP32 roundoff of a 128-term sum.
"""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "cuda" / "umma_probe.cu"
LIB = ROOT / "tests" / "cuda" / "libumma_probe.so"


def _lib():
    deps = [SRC, ROOT / "cubokit_b200" / "csrc" / "umma.cuh"]
    if not LIB.exists() or any(d.stat().st_mtime > LIB.stat().st_mtime for d in deps):
        from cubokit_b200.build import ARCH, nvcc
        subprocess.run([nvcc(), *ARCH, "-O2", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
                        "-I", str(ROOT / "cubokit_b200" / "csrc"), str(SRC), "-o", str(LIB)], check=True)
    lib = C.CDLL(str(LIB))
    lib.umma_probe_complex.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]
    lib.umma_probe_complex.restype = C.c_int
    lib.umma_probe_complex_strided.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_uint32, C.c_uint32,
                                               C.c_void_p]
    lib.umma_probe_complex_strided.restype = C.c_int
    return lib


def bf16_split(x):
    """hi = bf16(x) (round to nearest even), lo = bf16(x - hi); returns bit patterns and values."""
    x = np.asarray(x, np.float32)

    def rnd(v):
        u = v.view(np.uint32).astype(np.uint64)
        bits = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)
        return bits, (bits.astype(np.uint32) << 16).view(np.float32)

    hb, hv = rnd(x)
    lb, lv = rnd((x - hv).astype(np.float32))
    return hb, lb, hv.astype(np.float64), lv.astype(np.float64)


def planes(z):
    rh, rl, rhv, rlv = bf16_split(z.real)
    ih, il, ihv, ilv = bf16_split(z.imag)
    return np.ascontiguousarray(np.stack([rh, rl, ih, il])), (rhv, rlv, ihv, ilv)


@pytest.mark.parametrize("lbo,sbo", [(128, 2048), (144, 2304)])
@pytest.mark.parametrize("mn_major,conj", [(False, False), (True, False), (False, True), (True, True)])
def test_split_bf16_complex_product(mn_major, conj, lbo, sbo):
    """Packed core matrices (LBO 128) and core matrices 144 bytes apart along K (16 bytes of padding, the layout whose
    4-byte stores of consecutive K by consecutive lanes hit 32 different banks)."""
    lib = _lib()
    n = 128
    k = np.arange(n)
    w = np.exp(-2j * np.pi * np.outer(k, k) / n)  # the DFT matrix, W[m][k]
    rng = np.random.default_rng(5)
    b = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))  # logical B[k][n]
    wp, (wrh, wrl, wih, wil) = planes(w)
    bp, (brh, brl, bih, bil) = planes(b)
    out = np.zeros((2, n, n), np.float32)
    st = lib.umma_probe_complex_strided(wp.ctypes.data, bp.ctypes.data, int(mn_major), int(conj), 0, lbo, sbo,
                                        out.ctypes.data)
    assert st == 0, st
    mm = lambda p, q: p @ q
    s = -1.0 if conj else 1.0
    rr = mm(wrh, brh) + mm(wrh, brl) + mm(wrl, brh)
    ii = mm(wih, bih) + mm(wih, bil) + mm(wil, bih)
    ri = mm(wrh, bih) + mm(wrh, bil) + mm(wrl, bih)
    ir = mm(wih, brh) + mm(wih, brl) + mm(wil, brh)
    expect_re = rr - s * ii
    expect_im = ri + s * ir
    scale = np.max(np.abs(expect_re)) + np.max(np.abs(expect_im))
    assert np.max(np.abs(out[0] - expect_re)) <= 1e-5 * scale
    assert np.max(np.abs(out[1] - expect_im)) <= 1e-5 * scale
    # and the split product is a faithful complex product: relative error vs the exact FP64 W @ B
    exact = (np.conj(w) if conj else w) @ b
    rel = np.max(np.abs(out[0] + 1j * out[1] - exact)) / np.max(np.abs(exact))
    assert rel < 2e-5, rel


def test_a_wait_that_nothing_completes_runs_out_with_a_status():
    """The bounded-wait path: no MMA is issued and nothing arrives on the barrier; the kernel must give up after its
    time limit (0.2 s here), free its tensor memory and report status 1, leaving the context usable."""
    lib = _lib()
    n = 128
    planes = np.zeros((4, n, n), np.uint16)
    out = np.zeros((2, n, n), np.float32)
    assert lib.umma_probe_complex(planes.ctypes.data, planes.ctypes.data, 0, 0, 1, out.ctypes.data) == 1
    # the context is still usable: a normal product right after
    w = np.ones((4, n, n), np.uint16)
    assert lib.umma_probe_complex(w.ctypes.data, w.ctypes.data, 0, 0, 0, out.ctypes.data) == 0
