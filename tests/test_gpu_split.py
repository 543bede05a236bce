"""Split-precision DWT (PFSOFT_BATCH_SPLIT): exact 8-bit digit products on the tensor cores
against the FP64 path, the compiled reference's golden vectors, the oracle, mixed plans of
uneven bandwidths, and the kernel's bounded-wait exit.

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
    assert [B for B in range(0, 300) if lib.pfsoft_split_supported(B)] == list(range(1, 257))


@pytest.mark.parametrize("B,T", [(1, 1), (3, 2), (16, 1), (16, 4), (32, 6), (37, 3), (64, 4), (100, 2), (128, 5),
                                 (192, 2), (256, 2)])
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


def test_split_against_oracle(lib, oracle):
    """B = 20 and 33 (odd sizes, partial chunks and tiles): split-path grids and coefficients
    against the long-double oracle's IDSOFT / DSOFT of the same inputs."""
    import torch
    from oracle import oracle as orc
    for B in (20, 33):
        c = orc.coeffs_uniform(B, seed=B)
        dc = torch.from_numpy(c).to("cuda")
        grids, back = _run(lib, [B, B], [dc.clone(), dc.clone()], SPLIT)
        g_ref = oracle.idsoft(c, B)
        f_ref = oracle.dsoft(grids[0].cpu().numpy())
        for t in range(2):
            assert orc.rel_l2(grids[t].cpu().numpy(), g_ref) <= REL_TOL, f"B={B} grid"
        assert orc.rel_l2(back[0].cpu().numpy(), f_ref) <= REL_TOL, f"B={B} coefficients"


def test_bounded_wait_exit(lib):
    """A split launch whose first wait (before any MMA) runs out leaves cleanly: the plan's status
    reads PFSOFT_ETIMEOUT, the context stays usable, and a new plan then runs clean."""
    import torch
    bws = [16, 16]
    cs = _coeffs(lib, bws, seed0=5)
    s = torch.cuda.current_stream().cuda_stream
    grids = [torch.empty((32,) * 3, dtype=torch.complex128, device="cuda") for _ in bws]
    plan = ctypes.c_void_p()
    assert lib.pfsoft_batch_create((ctypes.c_int * 2)(*bws), 2, 0, SPLIT | 1, ctypes.byref(plan)) == 0
    cp = (ctypes.c_void_p * 2)(*[t.data_ptr() for t in cs])
    gp = (ctypes.c_void_p * 2)(*[t.data_ptr() for t in grids])
    try:
        assert lib.pfsoft_test_split_wait_ns(1_000_000) == 0      # 1 ms
        assert lib.pfsoft_batch_idsoft(plan, cp, gp, s) == 0
        torch.cuda.synchronize()
    finally:
        lib.pfsoft_test_split_wait_ns(0)
    assert lib.pfsoft_batch_status(plan) == 3                       # PFSOFT_ETIMEOUT
    lib.pfsoft_batch_destroy(plan)
    g64, c64 = _run(lib, bws, cs, 0)
    gsp, csp = _run(lib, bws, cs, SPLIT)
    for t in range(2):
        assert _rel(gsp[t], g64[t]) <= REL_TOL
        assert _rel(csp[t], c64[t]) <= REL_TOL


def test_mixed_plan_split_and_fp64(lib):
    """Uneven bandwidths in one split plan, every group in the one split launch, against the FP64
    plan (which runs B <= 128 fused and larger ones per transform)."""
    bws = [16, 24, 32, 32, 40, 64, 64, 64, 64, 16, 97, 130, 130]
    cs = _coeffs(lib, bws, seed0=77, kind=2, power=1.5)
    g64, c64 = _run(lib, bws, cs, 0)
    gsp, csp = _run(lib, bws, cs, SPLIT)
    for t, B in enumerate(bws):
        assert _rel(gsp[t], g64[t]) <= REL_TOL, f"B={B}"
        assert _rel(csp[t], c64[t]) <= REL_TOL, f"B={B}"
