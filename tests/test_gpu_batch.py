"""GPU tests of the batched engine (pfsoft_batch_*): uneven bandwidths in one plan, through the
C ABI, against the single-transform entry points and the oracle. Tolerances as the other parity
tests: relative L2 <= 1e-13 per transform; round trips within the reference's 1e-11."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as orc

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

REL_TOL = 1e-13


def _ptrs(tensors):
    arr = (ctypes.c_void_p * len(tensors))(*[t.data_ptr() for t in tensors])
    return arr


def _single(lib, fn, src, B):
    s = torch.cuda.current_stream().cuda_stream
    if fn == "idsoft":
        N = 2 * B
        out = torch.empty((N, N, N), dtype=torch.complex128, device="cuda")
        assert lib.pfsoft_cuda_idsoft(src.data_ptr(), B, out.data_ptr(), None, 0, s) == 0, lib.pfsoft_last_error()
    else:
        out = torch.empty(orc.coef_count(B), dtype=torch.complex128, device="cuda")
        assert lib.pfsoft_cuda_dsoft(src.data_ptr(), B, out.data_ptr(), None, 0, s) == 0, lib.pfsoft_last_error()
    return out


@pytest.mark.parametrize("tpc,flags", [(1, 0), (2, 0), (4, 0), (0, 1)])
def test_batch_matches_single_transforms(lib, tpc, flags):
    bws = [5, 8, 8, 16, 12, 32, 32, 32, 24, 64, 8]
    coeffs = [torch.from_numpy(orc.coeffs_uniform(B, seed=300 + i)).cuda() for i, B in enumerate(bws)]
    grids = [torch.full((2 * B,) * 3, complex(np.nan, np.nan), dtype=torch.complex128, device="cuda") for B in bws]
    back = [torch.full((orc.coef_count(B),), complex(np.nan, np.nan), dtype=torch.complex128, device="cuda") for B in bws]
    plan = ctypes.c_void_p()
    arr = (ctypes.c_int * len(bws))(*bws)
    assert lib.pfsoft_batch_create(arr, len(bws), tpc, flags, ctypes.byref(plan)) == 0, lib.pfsoft_last_error()
    s = torch.cuda.current_stream().cuda_stream
    try:
        for rep in range(2):   # second run replays the captured graph
            assert lib.pfsoft_batch_idsoft(plan, _ptrs(coeffs), _ptrs(grids), s) == 0, lib.pfsoft_last_error()
            assert lib.pfsoft_batch_dsoft(plan, _ptrs(grids), _ptrs(back), s) == 0, lib.pfsoft_last_error()
            torch.cuda.synchronize()
            for i, B in enumerate(bws):
                g_ref = _single(lib, "idsoft", coeffs[i], B)
                f_ref = _single(lib, "dsoft", grids[i], B)
                torch.cuda.synchronize()
                assert orc.rel_l2(grids[i].cpu().numpy(), g_ref.cpu().numpy()) <= REL_TOL, (B, rep)
                assert orc.rel_l2(back[i].cpu().numpy(), f_ref.cpu().numpy()) <= REL_TOL, (B, rep)
                d = (back[i] - coeffs[i]).abs().max().item()
                assert d <= 1e-11, (B, d)
    finally:
        lib.pfsoft_batch_destroy(plan)


def test_batch_against_oracle_and_large_bandwidth(lib, oracle):
    # one group above the fused limit (B = 136) runs the per-transform DWT inside the batch
    bws = [136, 6, 6]
    coeffs = [torch.from_numpy(orc.coeffs_uniform(B, seed=400 + i)).cuda() for i, B in enumerate(bws)]
    grids = [torch.empty((2 * B,) * 3, dtype=torch.complex128, device="cuda") for B in bws]
    back = [torch.empty(orc.coef_count(B), dtype=torch.complex128, device="cuda") for B in bws]
    plan = ctypes.c_void_p()
    arr = (ctypes.c_int * len(bws))(*bws)
    assert lib.pfsoft_batch_create(arr, len(bws), 0, 0, ctypes.byref(plan)) == 0, lib.pfsoft_last_error()
    s = torch.cuda.current_stream().cuda_stream
    try:
        assert lib.pfsoft_batch_idsoft(plan, _ptrs(coeffs), _ptrs(grids), s) == 0, lib.pfsoft_last_error()
        assert lib.pfsoft_batch_dsoft(plan, _ptrs(grids), _ptrs(back), s) == 0, lib.pfsoft_last_error()
        torch.cuda.synchronize()
        for i, B in enumerate(bws):
            c = coeffs[i].cpu().numpy()
            assert (back[i].cpu().numpy() - c).__abs__().max() <= 1e-11
            if B <= 16:
                assert orc.rel_l2(grids[i].cpu().numpy(), oracle.idsoft(c, B)) <= REL_TOL
    finally:
        lib.pfsoft_batch_destroy(plan)


def test_batch_rejects_bad_arguments(lib):
    plan = ctypes.c_void_p()
    arr = (ctypes.c_int * 2)(8, 0)
    assert lib.pfsoft_batch_create(arr, 2, 0, 0, ctypes.byref(plan)) == 1
    arr = (ctypes.c_int * 1)(8)
    assert lib.pfsoft_batch_create(arr, 1, 3, 0, ctypes.byref(plan)) == 1


def test_python_batch_plan(lib):
    """pfsoftlib_b200.BatchPlan: same results as the single-transform entry points, split mode
    within 1e-11, argument checks raise before any launch."""
    import torch

    from pfsoftlib_b200 import BatchPlan, PfsoftError

    bws = [16, 8, 16, 32, 5]
    s = torch.cuda.current_stream().cuda_stream
    cs = []
    for i, B in enumerate(bws):
        c = torch.empty(B * (4 * B * B - 1) // 3, dtype=torch.complex128, device="cuda")
        assert lib.pfsoft_cuda_random_coeffs(c.data_ptr(), B, 40 + i, 1, 1.0, s) == 0
        cs.append(c)
    grids = [torch.empty((2 * B,) * 3, dtype=torch.complex128, device="cuda") for B in bws]
    back = [torch.empty_like(c) for c in cs]
    with BatchPlan(bws) as plan:
        assert plan.transforms_per_cta in (1, 2, 4) and plan.workspace_bytes > 0
        plan.idsoft(cs, grids)
        plan.dsoft(grids, back)
    for B, c, g, f in zip(bws, cs, grids, back):
        assert orc.rel_l2(g.cpu().numpy(), _single(lib, "idsoft", c, B).cpu().numpy()) <= REL_TOL
        assert orc.rel_l2(f.cpu().numpy(), _single(lib, "dsoft", g, B).cpu().numpy()) <= REL_TOL
    with BatchPlan(bws, split=True) as plan:
        sg = [torch.empty_like(g) for g in grids]
        plan.idsoft(cs, sg)
        plan.status()
    for g, h in zip(grids, sg):
        assert (torch.linalg.vector_norm(h - g) / torch.linalg.vector_norm(g)).item() <= 1e-11
    plan = BatchPlan([8, 8])
    with pytest.raises(ValueError):
        plan.dsoft(grids[:2], back[:2])           # sizes do not match B = 8
    with pytest.raises(ValueError):
        plan.dsoft(grids[:1], back[:1])           # wrong count
    with pytest.raises(PfsoftError):
        BatchPlan([0])
    plan.close()
