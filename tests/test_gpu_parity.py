"""GPU parity tests: the CUDA engine, called through its C ABI, against the reference's own
outputs (golden fixtures and the compiled reference) and the long-double oracle.

Tolerances (FP64 engine vs reference / oracle): relative L2 <= 1e-13 and max-abs <= 1e-12 on
coefficients; round trips meet the reference's own criterion |d re|, |d im| <= 1e-11
(examples/example.cpp:44-74)."""
import numpy as np
import pytest

from oracle import oracle as orc

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

REL_TOL = 1e-13
ABS_TOL = 1e-12


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def stream():
    return torch.cuda.current_stream().cuda_stream


def gpu_dsoft(lib, grid, B, ws=None):
    g = dev(grid.astype(np.complex128))
    out = torch.empty(orc.coef_count(B), dtype=torch.complex128, device="cuda")
    wp, wb = (ws.data_ptr(), ws.numel() * ws.element_size()) if ws is not None else (None, 0)
    rc = lib.pfsoft_cuda_dsoft(g.data_ptr(), B, out.data_ptr(), wp, wb, stream())
    assert rc == 0, lib.pfsoft_last_error()
    torch.cuda.synchronize()
    return out.cpu().numpy(), g.cpu().numpy()


def gpu_idsoft(lib, coeffs, B):
    c = dev(coeffs.astype(np.complex128))
    N = 2 * B
    out = torch.full((N, N, N), complex(np.nan, np.nan), dtype=torch.complex128, device="cuda")
    rc = lib.pfsoft_cuda_idsoft(c.data_ptr(), B, out.data_ptr(), None, 0, stream())
    assert rc == 0, lib.pfsoft_last_error()
    torch.cuda.synchronize()
    return out.cpu().numpy()


def random_grid(B, seed):
    rng = np.random.default_rng(seed)
    N = 2 * B
    return rng.uniform(-1, 1, (N, N, N)) + 1j * rng.uniform(-1, 1, (N, N, N))


@pytest.mark.parametrize("B", [2, 4, 8, 16])
def test_dsoft_matches_reference_golden(lib, golden, B):
    g = golden[B]
    f, after = gpu_dsoft(lib, g["grid"], B)
    assert orc.rel_l2(f, g["coeffs_out"]) <= REL_TOL
    assert orc.max_abs(f, g["coeffs_out"]) <= ABS_TOL
    np.testing.assert_array_equal(after, g["grid"])   # input not modified


@pytest.mark.parametrize("B", [2, 4, 8, 16])
def test_idsoft_matches_reference_golden(lib, golden, B):
    g = golden[B]
    grid = gpu_idsoft(lib, g["coeffs_in"], B)
    assert orc.rel_l2(grid, g["grid"]) <= REL_TOL
    assert orc.max_abs(grid, g["grid"]) <= ABS_TOL


@pytest.mark.parametrize("B", [1, 3, 5, 6, 7, 12, 17, 24, 37, 48])
def test_dsoft_matches_oracle_any_grid(lib, oracle, B):
    # generic (not band-limited) grids, FFT lengths 2, 6, 10, 12, 14, 24, 48, 96; 34 and 74 (prime
    # factors 17 and 37) run the Bluestein pass
    grid = random_grid(B, seed=100 + B)
    f, _ = gpu_dsoft(lib, grid, B)
    ref = oracle.dsoft(grid)
    assert orc.rel_l2(f, ref) <= REL_TOL
    assert orc.max_abs(f, ref) <= ABS_TOL


@pytest.mark.parametrize("B", [1, 3, 5, 7, 12, 17, 24, 37, 48])
def test_idsoft_matches_oracle(lib, oracle, B):
    c = orc.coeffs_uniform(B, seed=200 + B)
    grid = gpu_idsoft(lib, c, B)
    ref = oracle.idsoft(c, B)
    assert orc.rel_l2(grid, ref) <= REL_TOL
    assert orc.max_abs(grid, ref) <= ABS_TOL * max(1, B)


@pytest.mark.parametrize("B", [16, 32, 64, 96, 128, 137, 192, 251])
def test_round_trip_reference_criterion(lib, B):
    c = orc.coeffs_uniform(B, seed=B)
    grid = gpu_idsoft(lib, c, B)
    f, _ = gpu_dsoft(lib, grid, B)
    d = f - c
    assert np.abs(d.real).max() <= 1e-11 and np.abs(d.imag).max() <= 1e-11
    assert orc.rel_l2(f, c) <= 1e-13


@pytest.mark.skipif(not orc.Reference.available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("B", [32, 64, 128])
def test_matches_compiled_reference(lib, B):
    ref = orc.Reference()
    threads = ref.max_threads()
    c = orc.coeffs_decaying(B, seed=B, power=1.0, normal_mag=True)
    g_ref = ref.idsoft(c, B, threads)
    g_gpu = gpu_idsoft(lib, c, B)
    assert orc.rel_l2(g_gpu, g_ref) <= REL_TOL
    f_ref = ref.dsoft(g_ref, threads)
    f_gpu, _ = gpu_dsoft(lib, g_ref, B)
    assert orc.rel_l2(f_gpu, f_ref) <= REL_TOL
    assert orc.max_abs(f_gpu, f_ref) <= ABS_TOL


@pytest.mark.skipif(not orc.Reference.available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("B", [192, 256])
def test_forward_matches_compiled_reference_large(lib, B):
    """DSOFT at B = 192 and 256 against the compiled reference's CPU DSOFT of the same grid (the
    grid is the GPU iDSOFT of device-generated coefficients, |f| = (1+l)^-1 |N(0,1)|)."""
    s = stream()
    c = torch.empty(B * (4 * B * B - 1) // 3, dtype=torch.complex128, device="cuda")
    assert lib.pfsoft_cuda_random_coeffs(c.data_ptr(), B, 77 + B, 1, 1.0, s) == 0
    g = torch.empty((2 * B,) * 3, dtype=torch.complex128, device="cuda")
    f = torch.empty_like(c)
    assert lib.pfsoft_cuda_idsoft(c.data_ptr(), B, g.data_ptr(), None, 0, s) == 0
    assert lib.pfsoft_cuda_dsoft(g.data_ptr(), B, f.data_ptr(), None, 0, s) == 0
    torch.cuda.synchronize()
    ref = orc.Reference()
    f_ref = ref.dsoft(g.cpu().numpy(), ref.max_threads())
    f_gpu = f.cpu().numpy()
    assert orc.rel_l2(f_gpu, f_ref) <= REL_TOL
    assert orc.max_abs(f_gpu, f_ref) <= ABS_TOL


@pytest.mark.skipif(not orc.Reference.available(), reason="reference build (oracle/_ref) not present")
def test_config_b16_seed0_against_reference(lib):
    """The plain round trip at B = 16 exactly as the workload states it: coefficients re, im
    U[-1, 1] from seed 0 (5,456 values); the GPU iDSOFT against the reference's IDSOFT, the GPU
    DSOFT of that grid against the reference's DSOFT of the same grid, and the round trip within
    the reference's own 1e-11 criterion (examples/example.cpp:44-74)."""
    B = 16
    c = orc.coeffs_uniform(B, seed=0)
    assert c.size == 5456
    ref = orc.Reference()
    grid = gpu_idsoft(lib, c, B)
    assert orc.rel_l2(grid, ref.idsoft(c, B, 1)) <= REL_TOL
    f, _ = gpu_dsoft(lib, grid, B)
    f_ref = ref.dsoft(grid, 1)
    assert orc.rel_l2(f, f_ref) <= REL_TOL and orc.max_abs(f, f_ref) <= ABS_TOL
    d = f - c
    assert np.abs(d.real).max() <= 1e-11 and np.abs(d.imag).max() <= 1e-11


def test_explicit_workspace_equals_library_workspace(lib):
    B = 10
    grid = random_grid(B, 7)
    ws = torch.empty(lib.pfsoft_workspace_bytes(B) // 8, dtype=torch.float64, device="cuda")
    a, _ = gpu_dsoft(lib, grid, B, ws=ws)
    b, _ = gpu_dsoft(lib, grid, B)
    np.testing.assert_array_equal(a, b)


def test_host_staged_matches_device(lib):
    B = 12
    c = orc.coeffs_uniform(B, seed=3)
    N = 2 * B
    g_host = np.zeros((N, N, N), dtype=np.complex128)
    assert lib.pfsoft_idsoft_host(c.ctypes.data, B, g_host.ctypes.data) == 0
    np.testing.assert_array_equal(g_host, gpu_idsoft(lib, c, B))
    f_host = np.zeros_like(c)
    assert lib.pfsoft_dsoft_host(g_host.ctypes.data, B, f_host.ctypes.data) == 0
    np.testing.assert_array_equal(f_host, gpu_dsoft(lib, g_host, B)[0])


def test_host_staged_pageable_large_matches_device(lib):
    """B = 96 (a 221 MB grid: the pageable copies go through the pinned bounce chunks, 16 MB
    each, in several rounds) on numpy (pageable) buffers, against the device entry points."""
    B = 96
    c = orc.coeffs_uniform(B, seed=9)
    N = 2 * B
    g_host = np.empty((N, N, N), dtype=np.complex128)
    assert lib.pfsoft_idsoft_host(c.ctypes.data, B, g_host.ctypes.data) == 0, lib.pfsoft_last_error()
    np.testing.assert_array_equal(g_host, gpu_idsoft(lib, c, B))
    f_host = np.empty_like(c)
    assert lib.pfsoft_dsoft_host(g_host.ctypes.data, B, f_host.ctypes.data) == 0, lib.pfsoft_last_error()
    np.testing.assert_array_equal(f_host, gpu_dsoft(lib, g_host, B)[0])


@pytest.mark.parametrize("cols,rows,lays", [(8, 8, 3), (32, 32, 5), (24, 40, 2), (7, 9, 3), (256, 256, 2), (512, 512, 1),
                                             (512, 384, 5), (384, 512, 6), (96, 192, 3), (192, 96, 2),
                                             (32, 96, 4), (502, 34, 1), (274, 22, 2), (257, 6, 2), (6, 257, 2)])
def test_layer_wise_fft_matches_numpy(lib, cols, rows, lays):
    rng = np.random.default_rng(cols * rows)
    x = rng.standard_normal((lays, cols, rows)) + 1j * rng.standard_normal((lays, cols, rows))
    t = dev(x)
    assert lib.pfsoft_cuda_layer_wise_dft2(cols, rows, lays, t.data_ptr(), 1.0, stream()) == 0
    torch.cuda.synchronize()
    y = t.cpu().numpy()
    ref = np.fft.fft2(x)
    assert orc.rel_l2(y, ref) <= 1e-14
    assert lib.pfsoft_cuda_layer_wise_idft2(cols, rows, lays, t.data_ptr(), 1.0 / (cols * rows), stream()) == 0
    torch.cuda.synchronize()
    assert orc.rel_l2(t.cpu().numpy(), x) <= 1e-14


@pytest.mark.parametrize("B", [2, 4, 8, 16])
def test_dwt_helpers_match_reference_golden(lib, golden, B):
    g = golden[B]
    w = torch.empty(2 * B, dtype=torch.float64, device="cuda")
    assert lib.pfsoft_cuda_quadrature_weights(B, w.data_ptr(), stream()) == 0
    np.testing.assert_allclose(w.cpu().numpy(), g["weights"], rtol=1e-14, atol=1e-16)
    for key, val in g.items():
        if not (key.startswith("wigner_") or key.startswith("wwigner_")):
            continue
        M, Mp = (int(x) for x in key.split("_")[1:])
        out = torch.empty(val.size, dtype=torch.float64, device="cuda")
        assert lib.pfsoft_cuda_wigner_d_matrix(B, M, Mp, int(key.startswith("ww")), out.data_ptr(), stream()) == 0
        d = out.cpu().numpy().reshape(val.shape)
        scale = max(1.0, float(np.abs(val).max()))
        assert np.abs(d - val).max() <= 1e-13 * scale, key


def test_wigner_matrix_large_orders_match_oracle(lib, oracle):
    # orders with seeds far below the FP64 range: the scaled recurrence must agree with the
    # long-double oracle wherever the values are representable
    B = 200
    for (M, Mp) in [(150, -150), (199, 0), (120, 119), (180, -3)]:
        J = max(abs(M), abs(Mp))
        out = torch.empty((B - J) * 2 * B, dtype=torch.float64, device="cuda")
        assert lib.pfsoft_cuda_wigner_d_matrix(B, M, Mp, 0, out.data_ptr(), stream()) == 0
        d = out.cpu().numpy().reshape(B - J, 2 * B)
        ref = oracle.wigner_d(B, M, Mp)
        assert np.abs(d - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())


def test_round_trip_b256(lib):
    """B = 256 (512^3 grid: the FFT passes run 4-vector tiles): IDSOFT then DSOFT."""
    B = 256
    s = stream()
    c = torch.empty(B * (4 * B * B - 1) // 3, dtype=torch.complex128, device="cuda")
    assert lib.pfsoft_cuda_random_coeffs(c.data_ptr(), B, 11, 2, 1.0, s) == 0
    g = torch.empty((2 * B,) * 3, dtype=torch.complex128, device="cuda")
    f = torch.empty_like(c)
    assert lib.pfsoft_cuda_idsoft(c.data_ptr(), B, g.data_ptr(), None, 0, s) == 0
    assert lib.pfsoft_cuda_dsoft(g.data_ptr(), B, f.data_ptr(), None, 0, s) == 0
    torch.cuda.synchronize()
    assert (torch.linalg.vector_norm(f - c) / torch.linalg.vector_norm(c)).item() <= 1e-13
