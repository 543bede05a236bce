"""The fused FFT stage (both passes of a direction in one persistent launch, layer chunk by layer
chunk; pfsoft_tune_fft_fused) against the two separate passes: the same arithmetic on the same
values, so the transforms agree bit for bit, for every plan family (ping-pong radix plans at
N = 64, 128, 256; in-place plans at N = 32, 96, 192, 384, 512; lengths that cannot be fused fall
back to two passes), single transforms and batch plans alike."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _coeffs(lib, B, seed):
    c = torch.empty(B * (4 * B * B - 1) // 3, dtype=torch.complex128, device="cuda")
    assert lib.pfsoft_cuda_random_coeffs(c.data_ptr(), B, seed, 1, 1.0, torch.cuda.current_stream().cuda_stream) == 0
    return c


def _round_trip(lib, B, c):
    s = torch.cuda.current_stream().cuda_stream
    g = torch.empty((2 * B,) * 3, dtype=torch.complex128, device="cuda")
    f = torch.empty_like(c)
    assert lib.pfsoft_cuda_idsoft(c.data_ptr(), B, g.data_ptr(), None, 0, s) == 0, lib.pfsoft_last_error()
    assert lib.pfsoft_cuda_dsoft(g.data_ptr(), B, f.data_ptr(), None, 0, s) == 0, lib.pfsoft_last_error()
    torch.cuda.synchronize()
    return g, f


@pytest.mark.parametrize("B", [5, 16, 32, 48, 64, 96, 128, 192, 256])
def test_fused_equals_two_passes(lib, B):
    c = _coeffs(lib, B, 500 + B)
    try:
        assert lib.pfsoft_tune_fft_fused(0, 0) == 0
        g2, f2 = _round_trip(lib, B, c)
        assert lib.pfsoft_tune_fft_fused(0, 1) == 0
        g1, f1 = _round_trip(lib, B, c)
    finally:
        lib.pfsoft_tune_fft_fused(0, 0)   # the library default
    assert torch.equal(g1, g2), f"B={B}: iDSOFT grids differ"
    assert torch.equal(f1, f2), f"B={B}: DSOFT coefficients differ"
    assert (torch.linalg.vector_norm(f1 - c) / torch.linalg.vector_norm(c)).item() <= 1e-13


@pytest.mark.parametrize("split", [0, 2])
def test_fused_batch_equals_two_passes(lib, split):
    bws = [32, 48, 48, 64, 96, 128, 128, 17]
    cs = [_coeffs(lib, B, 900 + i) for i, B in enumerate(bws)]
    s = torch.cuda.current_stream().cuda_stream
    out = {}
    try:
        for fused in (0, 1):
            assert lib.pfsoft_tune_fft_fused(0, fused) == 0
            plan = ctypes.c_void_p()
            assert lib.pfsoft_batch_create((ctypes.c_int * len(bws))(*bws), len(bws), 0, split | 1,
                                           ctypes.byref(plan)) == 0, lib.pfsoft_last_error()
            gs = [torch.empty((2 * B,) * 3, dtype=torch.complex128, device="cuda") for B in bws]
            fs = [torch.empty_like(c) for c in cs]
            cp = (ctypes.c_void_p * len(bws))(*[t.data_ptr() for t in cs])
            gp = (ctypes.c_void_p * len(bws))(*[t.data_ptr() for t in gs])
            fp = (ctypes.c_void_p * len(bws))(*[t.data_ptr() for t in fs])
            assert lib.pfsoft_batch_idsoft(plan, cp, gp, s) == 0
            assert lib.pfsoft_batch_dsoft(plan, gp, fp, s) == 0
            torch.cuda.synchronize()
            assert lib.pfsoft_batch_status(plan) == 0
            lib.pfsoft_batch_destroy(plan)
            out[fused] = (gs, fs)
    finally:
        lib.pfsoft_tune_fft_fused(0, 0)   # the library default
    for i, B in enumerate(bws):
        assert torch.equal(out[0][0][i], out[1][0][i]), f"B={B}: grids differ"
        assert torch.equal(out[0][1][i], out[1][1][i]), f"B={B}: coefficients differ"
