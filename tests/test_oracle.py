"""CPU tests of the checkers themselves: the C restatement (oracle/soft_oracle.c) against the
reference-generated golden fixtures, the FFT pieces against numpy.fft, and (when the reference
build is present) the reference build against the same fixtures."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as orc


@pytest.mark.parametrize("B", [2, 4, 8, 16])
def test_oracle_dsoft_matches_reference_golden(oracle, golden, B):
    g = golden[B]
    f = oracle.dsoft(g["grid"])
    assert orc.rel_l2(f, g["coeffs_out"]) < 5e-15
    assert orc.max_abs(f, g["coeffs_out"]) < 1e-14


@pytest.mark.parametrize("B", [2, 4, 8, 16])
def test_oracle_idsoft_matches_reference_golden(oracle, golden, B):
    g = golden[B]
    grid = oracle.idsoft(g["coeffs_in"], B)
    assert orc.rel_l2(grid, g["grid"]) < 5e-15


@pytest.mark.parametrize("B", [2, 4, 8, 16])
def test_reference_round_trip_known_answer(golden, B):
    # examples/example.cpp:44-74: |re|, |im| differences <= 1e-11 after IDSOFT -> DSOFT
    g = golden[B]
    d = g["coeffs_out"] - g["coeffs_in"]
    assert np.all(np.abs(d.real) <= 1e-11) and np.all(np.abs(d.imag) <= 1e-11)


@pytest.mark.parametrize("B", [2, 4, 8, 16])
def test_oracle_weights_and_wigner_match_golden(oracle, golden, B):
    g = golden[B]
    np.testing.assert_allclose(oracle.weights(B), g["weights"], rtol=0, atol=1e-16)
    for key, val in g.items():
        if key.startswith("wigner_") or key.startswith("wwigner_"):
            M, Mp = (int(x) for x in key.split("_")[1:])
            d = oracle.wigner_d(B, M, Mp, weighted=key.startswith("ww"))
            scale = max(1.0, float(np.abs(val).max()))
            assert np.abs(d - val).max() <= 1e-14 * scale, key


@pytest.mark.parametrize("N,lays", [(2, 2), (6, 3), (10, 2), (14, 2), (32, 4), (96, 2)])
def test_oracle_fft_matches_numpy(oracle, N, lays):
    rng = np.random.default_rng(N)
    x = rng.standard_normal((lays, N, N)) + 1j * rng.standard_normal((lays, N, N))
    np.testing.assert_allclose(oracle.fft2_layers(x, -1), np.fft.fft2(x), rtol=0, atol=1e-12 * N)
    np.testing.assert_allclose(oracle.fft2_layers(x, +1), np.fft.ifft2(x) * N * N, rtol=0, atol=1e-12 * N)


def test_oracle_symmetry_rule_against_reference_wigner_matrices(oracle):
    # the per-coefficient rule reproduces all eight cases of the reference at every (M, M'):
    # exercised end to end by the golden tests above at B = 16 (all 136 classes)
    B = 6
    c = orc.coeffs_uniform(B, seed=11)
    grid = oracle.idsoft(c, B)
    assert orc.max_abs(oracle.dsoft(grid), c) < 1e-13


def test_coefficient_layout_helpers():
    B = 5
    l, m1, m2 = orc.fill_order(B)
    idx = orc.coef_index(l, m1, m2)
    assert sorted(idx.tolist()) == list(range(orc.coef_count(B)))
    assert orc.coef_index(3, -3, 0) == orc.coef_offset(3) + 0 * 7 + 4


ref_only = pytest.mark.skipif(not orc.Reference.available(), reason="reference build (oracle/_ref) not present")


@ref_only
@pytest.mark.parametrize("B", [2, 4, 8, 16])
def test_reference_build_reproduces_golden(golden, B):
    ref = orc.Reference()
    g = golden[B]
    np.testing.assert_array_equal(ref.dsoft(g["grid"]), g["coeffs_out"])


@ref_only
@pytest.mark.parametrize("N", [4, 6, 10, 16, 30])
def test_fftw_standin_matches_numpy(N):
    lib = ctypes.CDLL(orc.REF_SO)
    rng = np.random.default_rng(N)
    x = rng.standard_normal((3, N, N)) + 1j * rng.standard_normal((3, N, N))
    y = np.ascontiguousarray(x.copy())
    lib.uzl_fftw_layer_wise_DFT2_grid3D(N, N, 3, y.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 2)
    np.testing.assert_allclose(y, np.fft.fft2(x), rtol=0, atol=1e-12 * N)
    lib.uzl_fftw_layer_wise_IDFT2_grid3D(N, N, 3, y.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 2)
    np.testing.assert_allclose(y, x * N * N, rtol=0, atol=1e-11 * N * N)
