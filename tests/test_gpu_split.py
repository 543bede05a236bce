"""Split-precision DWT (PFSOFT_BATCH_SPLIT): tensor-core digit products against the FP64 path,
the compiled reference's golden vectors, and mixed plans where some bandwidths stay on FP64.

Tolerance: relative L2 error <= 1e-11 against FP64 results (the engine's stated bound for the
split path; the digit arithmetic itself gives about 1e-13)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SPLIT = 2
REL_TOL = 1e-11


def _rel(a, b):
    import torch
    return (torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)).item()


def _run(lib, bws, coeffs, flags):
    """IDSOFT then DSOFT of every transform through one batch plan; returns (grids, coeffs)."""
    import torch
    s = torch.cuda.current_stream().cuda_stream
    grids = [torch.empty((2 * B,) * 3, dtype=torch.complex128, device="cuda") for B in bws]
    back = [torch.empty_like(c) for c in coeffs]
    plan = ctypes.c_void_p()
    arr = (ctypes.c_int * len(bws))(*bws)
    assert lib.pfsoft_batch_create(arr, len(bws), 0, flags, ctypes.byref(plan)) == 0, lib.pfsoft_last_error()
    cp = (ctypes.c_void_p * len(bws))(*[t.data_ptr() for t in coeffs])
    gp = (ctypes.c_void_p * len(bws))(*[t.data_ptr() for t in grids])
    bp = (ctypes.c_void_p * len(bws))(*[t.data_ptr() for t in back])
    assert lib.pfsoft_batch_idsoft(plan, cp, gp, s) == 0
    assert lib.pfsoft_batch_dsoft(plan, gp, bp, s) == 0
    torch.cuda.synchronize()
    assert lib.pfsoft_batch_status(plan) == 0
    lib.pfsoft_batch_destroy(plan)
    return grids, back


def _coeffs(lib, bws, seed0=300, kind=1, power=1.0):
    import torch
    s = torch.cuda.current_stream().cuda_stream
    out = []
    for i, B in enumerate(bws):
        c = torch.empty(B * (4 * B * B - 1) // 3, dtype=torch.complex128, device="cuda")
        assert lib.pfsoft_cuda_random_coeffs(c.data_ptr(), B, seed0 + i, kind, power, s) == 0
        out.append(c)
    return out


def test_supported_bandwidths(lib):
    assert [B for B in range(1, 300) if lib.pfsoft_split_supported(B)] == list(range(16, 129, 16))


@pytest.mark.parametrize("B,T", [(16, 1), (16, 4), (32, 6), (64, 4), (128, 5)])
def test_split_matches_fp64(lib, B, T):
    bws = [B] * T
    cs = _coeffs(lib, bws, seed0=1000 * B + T)
    g64, c64 = _run(lib, bws, cs, 0)
    gsp, csp = _run(lib, bws, cs, SPLIT)
    for t in range(T):
        eg, ec = _rel(gsp[t], g64[t]), _rel(csp[t], c64[t])
        assert eg <= REL_TOL, f"B={B} t={t}: iDSOFT grid rel L2 {eg:.2e}"
        assert ec <= REL_TOL, f"B={B} t={t}: DSOFT coefficients rel L2 {ec:.2e}"
        assert _rel(csp[t], cs[t]) <= REL_TOL   # round trip


def test_split_against_reference_golden(lib, golden):
    """B = 16: the reference's IDSOFT grid and DSOFT coefficients (tests/golden) through the
    split path, four copies in one plan."""
    import torch
    g = golden[16]
    f = torch.from_numpy(g["coeffs_in"].astype(np.complex128)).to("cuda")
    grid_ref = torch.from_numpy(g["grid"].astype(np.complex128)).to("cuda")
    fref = torch.from_numpy(g["coeffs_out"].astype(np.complex128)).to("cuda")
    grids, back = _run(lib, [16] * 4, [f.clone() for _ in range(4)], SPLIT)
    for t in range(4):
        assert _rel(grids[t].reshape(-1), grid_ref.reshape(-1)) <= REL_TOL
    # forward alone on the reference's grid
    s = torch.cuda.current_stream().cuda_stream
    plan = ctypes.c_void_p()
    assert lib.pfsoft_batch_create((ctypes.c_int * 4)(*[16] * 4), 4, 0, SPLIT, ctypes.byref(plan)) == 0
    gsrc = [grid_ref.reshape(32, 32, 32).contiguous().clone() for _ in range(4)]
    outs = [torch.empty_like(fref) for _ in range(4)]
    gp = (ctypes.c_void_p * 4)(*[x.data_ptr() for x in gsrc])
    op = (ctypes.c_void_p * 4)(*[x.data_ptr() for x in outs])
    assert lib.pfsoft_batch_dsoft(plan, gp, op, s) == 0
    torch.cuda.synchronize()
    assert lib.pfsoft_batch_status(plan) == 0
    lib.pfsoft_batch_destroy(plan)
    for t in range(4):
        assert _rel(outs[t], fref) <= REL_TOL


def test_mixed_plan_split_and_fp64(lib):
    """Bandwidths the split kernel takes (16, 32, 64) and ones it leaves to FP64 (24, 40) in one plan."""
    bws = [16, 24, 32, 32, 40, 64, 64, 64, 64, 16]
    cs = _coeffs(lib, bws, seed0=77, kind=2, power=1.5)
    g64, c64 = _run(lib, bws, cs, 0)
    gsp, csp = _run(lib, bws, cs, SPLIT)
    for t, B in enumerate(bws):
        assert _rel(gsp[t], g64[t]) <= REL_TOL, f"B={B}"
        assert _rel(csp[t], c64[t]) <= REL_TOL, f"B={B}"
