"""Test infrastructure (oracle): Python access to the CPU checkers. NOT part of the product.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline / reference legs import
this module. The CUDA product (``pfsoftlib_b200``) never imports it.

Two checkers are exposed through ctypes:

* ``Oracle``    -- ``oracle/liboracle.so``, the project's long-double C restatement of
                   DSOFT / iDSOFT (``oracle/soft_oracle.c``).
* ``Reference`` -- ``oracle/_ref/libpfsoft_ref.so``, the reference's own sources
                   (src/fn_dsoft.cpp, src/fn_idsoft.cpp, ...) compiled unmodified, with a
                   project FFT in place of the absent FFTW 3.3.4 (``oracle/fft_standin.cpp``).

Plus numpy helpers for the packed layouts, the seeded input generators of the benchmark
workloads, and error metrics.

Layouts (shared with the product's C ABI):

* grid   -- complex128 array of shape (N, N, N) indexed [lay, col, row] (row fastest), i.e.
            element (row, col, lay) of ``grid3D`` at (lay*N + col)*N + row
            (include/PFSOFTlib_headers/grid3D_cx.hpp:293-303), N = 2B.
* coeffs -- complex128 vector of length B(4B^2-1)/3; degree l starts at l(4l^2-1)/3 and holds
            a column-major (2l+1)x(2l+1) block, row index M, column index M', negative orders
            stored at 2l+1+M (src/dsoft_fourier_coefficients.cpp:80-89).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libpfsoft_ref.so")

_dp = ctypes.POINTER(ctypes.c_double)


def _ptr(a: np.ndarray):
    assert a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


# ----------------------------------------------------------------------------- layouts

def coef_offset(l: int) -> int:
    return l * (4 * l * l - 1) // 3


def coef_count(B: int) -> int:
    return coef_offset(B)


def coef_index(l, m1, m2):
    """Packed index of f^l_{m1,m2} (vectorises over numpy arrays)."""
    l = np.asarray(l, dtype=np.int64)
    m1 = np.asarray(m1, dtype=np.int64)
    m2 = np.asarray(m2, dtype=np.int64)
    L = 2 * l + 1
    i1 = np.where(m1 >= 0, m1, L + m1)
    i2 = np.where(m2 >= 0, m2, L + m2)
    return l * (4 * l * l - 1) // 3 + i2 * L + i1


def fill_order(B: int):
    """(l, M, M') in the order ``rand(DSOFTFourierCoefficients&)`` fills them
    (include/PFSOFTlib_headers/random.hpp:105-116): l outer, then M, then M'."""
    ls, ms, mps = [], [], []
    for l in range(B):
        r = np.arange(-l, l + 1)
        M, Mp = np.meshgrid(r, r, indexing="ij")
        ls.append(np.full(M.size, l))
        ms.append(M.ravel())
        mps.append(Mp.ravel())
    return np.concatenate(ls), np.concatenate(ms), np.concatenate(mps)


def degrees(B: int) -> np.ndarray:
    """Degree l of every packed coefficient slot."""
    return np.concatenate([np.full((2 * l + 1) ** 2, l) for l in range(B)])


# ----------------------------------------------------------------------------- inputs

def coeffs_uniform(B: int, seed: int) -> np.ndarray:
    """Re and im i.i.d. U[-1, 1], drawn in the reference fill order (l -> M -> M', re then
    im) from numpy PCG64 with the given seed (examples/example.cpp uses U[-1,1])."""
    rng = np.random.default_rng(seed)
    v = rng.uniform(-1.0, 1.0, size=(coef_count(B), 2))
    l, m1, m2 = fill_order(B)
    out = np.empty(coef_count(B), dtype=np.complex128)
    out[coef_index(l, m1, m2)] = v[:, 0] + 1j * v[:, 1]
    return out


def coeffs_decaying(B: int, seed: int, power: float, normal_mag: bool = False) -> np.ndarray:
    """Uniform phase in [0, 2pi) and magnitude (1+l)^-power, times |N(0,1)| when
    ``normal_mag`` (the B=128 single-transform workload), drawn in the reference fill order."""
    rng = np.random.default_rng(seed)
    n = coef_count(B)
    l, m1, m2 = fill_order(B)
    mag = (1.0 + l) ** (-power)
    if normal_mag:
        mag = mag * np.abs(rng.standard_normal(n))
    phase = rng.uniform(0.0, 2.0 * np.pi, size=n)
    out = np.empty(n, dtype=np.complex128)
    out[coef_index(l, m1, m2)] = mag * np.exp(1j * phase)
    return out


# ----------------------------------------------------------------------------- metrics

def rel_l2(x: np.ndarray, ref: np.ndarray) -> float:
    den = float(np.linalg.norm(ref))
    return float(np.linalg.norm(x - ref)) / (den if den > 0 else 1.0)


def max_abs(x: np.ndarray, ref: np.ndarray) -> float:
    return float(np.max(np.abs(x - ref))) if x.size else 0.0


# ----------------------------------------------------------------------------- build

def build(ref_root: str | None = None, quiet: bool = True) -> None:
    """Build liboracle.so and, when a reference source tree is given (``ref_root``, else the
    PFSOFT_REFERENCE environment variable) and present, _ref/libpfsoft_ref.so."""
    targets = ["oracle"]
    ref_root = ref_root or os.environ.get("PFSOFT_REFERENCE", "")
    if ref_root and os.path.isdir(os.path.join(ref_root, "src")):
        targets.append("ref")
    cmd = ["make", "-s", "-C", HERE, f"REF={ref_root}"] + targets
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL if quiet else None)


# ----------------------------------------------------------------------------- C restatement

class Oracle:
    """The project's long-double C restatement (oracle/soft_oracle.c)."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build()
        lib = ctypes.CDLL(path)
        lib.oracle_dsoft.argtypes = [_dp, ctypes.c_int, _dp]
        lib.oracle_idsoft.argtypes = [_dp, ctypes.c_int, _dp]
        lib.oracle_quadrature_weights.argtypes = [ctypes.c_int, _dp]
        lib.oracle_wigner_d.argtypes = [ctypes.c_int] * 4 + [_dp]
        lib.oracle_fft2_layers.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp, ctypes.c_int]
        lib.oracle_dwt_forward.argtypes = [_dp, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, _dp]
        lib.oracle_dwt_inverse.argtypes = [_dp, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, _dp]
        self.lib = lib

    def dsoft(self, grid: np.ndarray) -> np.ndarray:
        N = grid.shape[0]
        B = N // 2
        g = np.ascontiguousarray(grid, dtype=np.complex128)
        out = np.empty(coef_count(B), dtype=np.complex128)
        self.lib.oracle_dsoft(_ptr(g.view(np.float64)), B, _ptr(out.view(np.float64)))
        return out

    def idsoft(self, coeffs: np.ndarray, B: int) -> np.ndarray:
        c = np.ascontiguousarray(coeffs, dtype=np.complex128)
        N = 2 * B
        out = np.empty((N, N, N), dtype=np.complex128)
        self.lib.oracle_idsoft(_ptr(c.view(np.float64)), B, _ptr(out.view(np.float64)))
        return out

    def dwt_forward(self, spectrum: np.ndarray, B: int, classes=None, out: np.ndarray | None = None) -> np.ndarray:
        """The DWT stage on the bin-major spectrum X[row][col][k] for `classes` (None: all),
        writing only their coefficients into `out` (zeros when not given)."""
        x = np.ascontiguousarray(spectrum, dtype=np.complex128).reshape(-1)
        out = np.zeros(coef_count(B), dtype=np.complex128) if out is None else out
        cl = None if classes is None else np.ascontiguousarray(classes, dtype=np.int32)
        self.lib.oracle_dwt_forward(_ptr(x.view(np.float64)), B, None if cl is None else cl.ctypes.data,
                                    -1 if cl is None else len(cl), _ptr(out.view(np.float64)))
        return out

    def dwt_inverse(self, coeffs: np.ndarray, B: int, classes=None, out: np.ndarray | None = None) -> np.ndarray:
        """The inverse DWT stage into the bin-major spectrum `out` (zeros when not given), writing
        only the beta columns of the bins of `classes` (None: all)."""
        c = np.ascontiguousarray(coeffs, dtype=np.complex128)
        N = 2 * B
        out = np.zeros(N ** 3, dtype=np.complex128) if out is None else out
        cl = None if classes is None else np.ascontiguousarray(classes, dtype=np.int32)
        self.lib.oracle_dwt_inverse(_ptr(c.view(np.float64)), B, None if cl is None else cl.ctypes.data,
                                    -1 if cl is None else len(cl), _ptr(out.view(np.float64)))
        return out

    def weights(self, B: int) -> np.ndarray:
        w = np.empty(2 * B)
        self.lib.oracle_quadrature_weights(B, _ptr(w))
        return w

    def wigner_d(self, B: int, M: int, Mp: int, weighted: bool = False) -> np.ndarray:
        J = max(abs(M), abs(Mp))
        out = np.empty((B - J, 2 * B))
        self.lib.oracle_wigner_d(B, M, Mp, int(weighted), _ptr(out))
        return out

    def fft2_layers(self, grid: np.ndarray, sign: int = -1) -> np.ndarray:
        g = np.ascontiguousarray(grid, dtype=np.complex128)
        lays, N = g.shape[0], g.shape[1]
        out = np.empty_like(g)
        self.lib.oracle_fft2_layers(N, lays, _ptr(g.view(np.float64)), _ptr(out.view(np.float64)), sign)
        return out


# ----------------------------------------------------------------------------- the reference

class Reference:
    """The reference's own DSOFT / IDSOFT / DWT, compiled from its sources."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (oracle/Makefile target 'ref')")
        lib = ctypes.CDLL(path)
        lib.ref_dsoft.argtypes = [_dp, ctypes.c_int, _dp, ctypes.c_int]
        lib.ref_idsoft.argtypes = [_dp, ctypes.c_int, _dp, ctypes.c_int]
        lib.ref_quadrature_weights.argtypes = [ctypes.c_int, _dp]
        lib.ref_wigner_d_matrix.argtypes = [ctypes.c_int] * 4 + [_dp]
        lib.ref_max_threads.restype = ctypes.c_int
        lib.ref_ctx_create.restype = ctypes.c_void_p
        lib.ref_ctx_create.argtypes = [ctypes.c_int]
        lib.ref_ctx_destroy.argtypes = [ctypes.c_void_p]
        for f in ("ref_ctx_set_grid", "ref_ctx_get_grid", "ref_ctx_set_coeffs", "ref_ctx_get_coeffs"):
            getattr(lib, f).argtypes = [ctypes.c_void_p, _dp]
        for f in ("ref_ctx_dsoft", "ref_ctx_idsoft"):
            getattr(lib, f).argtypes = [ctypes.c_void_p, ctypes.c_int]
            getattr(lib, f).restype = ctypes.c_double
        self.lib = lib

    @staticmethod
    def available(path: str = REF_SO) -> bool:
        return os.path.exists(path)

    def max_threads(self) -> int:
        return int(self.lib.ref_max_threads())

    def dsoft(self, grid: np.ndarray, threads: int = 1) -> np.ndarray:
        B = grid.shape[0] // 2
        g = np.ascontiguousarray(grid, dtype=np.complex128)
        out = np.empty(coef_count(B), dtype=np.complex128)
        self.lib.ref_dsoft(_ptr(g.view(np.float64)), B, _ptr(out.view(np.float64)), threads)
        return out

    def idsoft(self, coeffs: np.ndarray, B: int, threads: int = 1) -> np.ndarray:
        c = np.ascontiguousarray(coeffs, dtype=np.complex128)
        N = 2 * B
        out = np.empty((N, N, N), dtype=np.complex128)
        self.lib.ref_idsoft(_ptr(c.view(np.float64)), B, _ptr(out.view(np.float64)), threads)
        return out

    def weights(self, B: int) -> np.ndarray:
        w = np.empty(2 * B)
        self.lib.ref_quadrature_weights(B, _ptr(w))
        return w

    def wigner_d(self, B: int, M: int, Mp: int, weighted: bool = False) -> np.ndarray:
        J = max(abs(M), abs(Mp))
        out = np.empty((B - J, 2 * B))
        self.lib.ref_wigner_d_matrix(B, M, Mp, int(weighted), _ptr(out))
        return out


class ReferenceTimer:
    """Times the reference's DSOFT and IDSOFT on persistent containers (the shape of
    benchmark/benchmark_dsoft_for.cpp:157-186): only the transform call is inside the clock."""

    def __init__(self, ref: Reference, B: int, coeffs: np.ndarray):
        self.ref, self.B = ref, B
        self.ctx = ref.lib.ref_ctx_create(B)
        c = np.ascontiguousarray(coeffs, dtype=np.complex128)
        ref.lib.ref_ctx_set_coeffs(self.ctx, _ptr(c.view(np.float64)))

    def idsoft(self, threads: int) -> float:
        return float(self.ref.lib.ref_ctx_idsoft(self.ctx, threads))

    def dsoft(self, threads: int) -> float:
        return float(self.ref.lib.ref_ctx_dsoft(self.ctx, threads))

    def close(self) -> None:
        if self.ctx:
            self.ref.lib.ref_ctx_destroy(self.ctx)
            self.ctx = None


def wall(fn, *a, **k):
    t0 = time.perf_counter()
    r = fn(*a, **k)
    return r, time.perf_counter() - t0
