"""Host-side mirror of PFSOFTlib's public interface for the DSOFT / iDSOFT path.

Names, argument meaning and error behaviour follow the reference:

* ``grid3D``                    include/PFSOFTlib_headers/grid3D_cx.hpp:47-83
* ``DSOFTFourierCoefficients``  include/PFSOFTlib_headers/dsoft_fourier_coefficients.hpp:50-72
* ``FourierTransforms.DSOFT``   src/fn_dsoft.cpp:76      (sample taken "by value": not modified)
* ``FourierTransforms.IDSOFT``  src/fn_idsoft.cpp:72
* ``DWT.quadrature_weights / wigner_d_matrix / weighted_wigner_d_matrix``
                                include/PFSOFTlib_headers/fn_dwt.hpp:64,239,107

Argument checks that the reference reports with a warning and a silent return
(src/fn_dsoft.cpp:82-94 through cmake_aux/compiler_config.hpp.in:112-120) print the same kind
of warning to stderr and return. An order outside |M|,|M'| <= l, where the reference calls
exit(EXIT_FAILURE) (src/dsoft_fourier_coefficients.cpp:82), raises IndexError instead.

Containers live either on the host (numpy, the default) or on the GPU (``device="cuda"``,
torch tensors used as plain device buffers). Host containers go through the host-staged entry
points (copy in, transform, copy out); device containers use the stream-ordered entry points on
torch's current CUDA stream. Every transform runs in the CUDA library; there is no CPU path.
"""
from __future__ import annotations

import sys

import numpy as np

from . import _lib


def _warn(func: str, msg: str) -> None:
    sys.stderr.write(f"** [PFSOFTLib warning] {func}(): {msg} **\n")


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _dev_ptr(t) -> int:
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("device buffer must be a contiguous CUDA tensor")
    return t.data_ptr()


def _stream_ptr():
    import torch

    return torch.cuda.current_stream().cuda_stream


def coef_count(B: int) -> int:
    return B * (4 * B * B - 1) // 3


def coef_index(l: int, M: int, Mp: int) -> int:
    L = 2 * l + 1
    i1 = M if M >= 0 else L + M
    i2 = Mp if Mp >= 0 else L + Mp
    return l * (4 * l * l - 1) // 3 + i2 * L + i1


def _cell_format(values):
    """Width and notation of the reference's complex grid / matrix printers (grid3D_cx.hpp:429-523,
    matrix_cx.hpp:545-620): 20, fixed; the last value in print order whose real or imaginary
    magnitude reaches 10, 100 or 1000 sets 22, 24 or 28 (the last in scientific notation)."""
    width, sci = 20, False
    for v in values:
        a, b = abs(v.real), abs(v.imag)
        if a >= 10 or b >= 10:
            width, sci = 22, False
        if a >= 100 or b >= 100:
            width, sci = 24, False
        if a >= 1000 or b >= 1000:
            width, sci = 28, True
    return width, sci


def _cell(v, width, sci):
    f = "%.4e" if sci else "%.4f"
    im = v.imag
    text = (f % v.real) + (" - " if im < 0 else " + ") + (f % (0.0 if im == 0 else abs(im))) + "i"
    return text.rjust(width)


class grid3D:
    """Complex (2B)^3 sample grid, element (row, col, lay) at (lay*cols + col)*rows + row.

    ``mem`` is the storage: a numpy complex128 array of shape (lays, cols, rows), or a torch
    complex128 CUDA tensor of that shape when ``device="cuda"``. New grids are zero-filled,
    as ``new complex<double>[n]`` is in the reference (complex.hpp:117-120).
    """

    def __init__(self, rows, cols=None, lays=None, initial=0, device: str = "cpu"):
        if cols is None and lays is None:
            cols = lays = rows
        self.rows, self.cols, self.lays = int(rows), int(cols), int(lays)
        shape = (self.lays, self.cols, self.rows)
        if device == "cpu":
            self.mem = np.full(shape, initial, dtype=np.complex128)
        else:
            import torch

            self.mem = torch.full(shape, complex(initial), dtype=torch.complex128, device=device)

    @classmethod
    def wrap(cls, array) -> "grid3D":
        """Use an existing (lays, cols, rows) complex128 array or CUDA tensor as storage."""
        g = cls.__new__(cls)
        g.lays, g.cols, g.rows = (int(s) for s in array.shape)
        g.mem = array
        return g

    @property
    def on_device(self) -> bool:
        return _is_torch(self.mem) and self.mem.is_cuda

    def __call__(self, row, col, lay):
        return self.mem[lay, col, row]

    def __getitem__(self, idx):
        row, col, lay = idx
        return self.mem[lay, col, row]

    def __setitem__(self, idx, value):
        row, col, lay = idx
        self.mem[lay, col, row] = value

    def copy(self) -> "grid3D":
        return grid3D.wrap(self.mem.clone() if _is_torch(self.mem) else self.mem.copy())

    def __str__(self) -> str:
        """The reference's ``operator<<`` text (grid3D_cx.hpp:429-523): a blank line, then per
        layer ``layer[z]`` and one line per grid row."""
        m = self.mem.cpu().numpy() if _is_torch(self.mem) else np.asarray(self.mem)
        order = [complex(m[z, y, x]) for z in range(self.lays) for x in range(self.rows) for y in range(self.cols)]
        width, sci = _cell_format(order)
        out = ["\n"]
        for z in range(self.lays):
            out.append(f"layer[{z}]\n")
            for x in range(self.rows):
                out.append("".join(_cell(complex(m[z, y, x]), width, sci) for y in range(self.cols)) + "\n")
            out.append("\n")
        return "".join(out)

    def _layer_wise(self, scale: complex, inverse: bool):
        if not self.on_device:
            raise ValueError("layer-wise DFT runs on device grids (device='cuda')")
        import torch

        lib = _lib.load()
        f = lib.pfsoft_cuda_layer_wise_idft2 if inverse else lib.pfsoft_cuda_layer_wise_dft2
        s = complex(scale)
        real_scale = s.real if s.imag == 0 else 1.0
        _lib.check(f(self.cols, self.rows, self.lays, _dev_ptr(self.mem), real_scale, _stream_ptr()))
        if s.imag != 0:
            self.mem.mul_(torch.tensor(s, dtype=torch.complex128, device=self.mem.device))

    def layer_wise_DFT2(self, scale=1.0, threads: int = 1):
        """grid3D_cx.hpp:309-366: in-place unnormalised 2D DFT of every layer, then * scale."""
        self._layer_wise(scale, inverse=False)

    def layer_wise_IDFT2(self, scale=1.0, threads: int = 1):
        """grid3D_cx.hpp:370-427: in-place unnormalised inverse 2D DFT of every layer, then * scale."""
        self._layer_wise(scale, inverse=True)


class DSOFTFourierCoefficients:
    """Coefficients f^l_{M,M'} for 0 <= l < B, |M|, |M'| <= l, packed contiguously: degree l at
    l(4l^2-1)/3, a column-major (2l+1)x(2l+1) block, negative orders at 2l+1+M."""

    def __init__(self, bandwidth: int = 0, device: str = "cpu"):
        self.bandwidth = int(bandwidth)
        n = coef_count(self.bandwidth) if self.bandwidth > 0 else 0
        if device == "cpu":
            self.mem = np.zeros(n, dtype=np.complex128)
        else:
            import torch

            self.mem = torch.zeros(n, dtype=torch.complex128, device=device)

    @classmethod
    def wrap(cls, array, bandwidth: int) -> "DSOFTFourierCoefficients":
        if array.shape[0] != coef_count(bandwidth):
            raise ValueError("coefficient vector length does not match the bandwidth")
        fc = cls.__new__(cls)
        fc.bandwidth = int(bandwidth)
        fc.mem = array
        return fc

    @property
    def on_device(self) -> bool:
        return _is_torch(self.mem) and self.mem.is_cuda

    def _index(self, l, M, Mp) -> int:
        if not (0 <= l < self.bandwidth) or M > l or Mp > l or M < -l or Mp < -l:
            raise IndexError("illegal parameter for DSOFTFourierCoefficients. Condition |M|,|Mp| <= l violated.")
        return coef_index(l, M, Mp)

    def __call__(self, l, M, Mp):
        return self.mem[self._index(l, M, Mp)]

    def __getitem__(self, idx):
        return self.mem[self._index(*idx)]

    def __setitem__(self, idx, value):
        self.mem[self._index(*idx)] = value

    def __str__(self) -> str:
        """The reference's ``operator<<`` text (src/dsoft_fourier_coefficients.cpp:124-137): per
        degree a title line and the (2l+1)^2 block, rows = M, columns = M'."""
        m = self.mem.cpu().numpy() if _is_torch(self.mem) else np.asarray(self.mem)
        out = ["\n"]
        for l in range(self.bandwidth):
            out.append(f"DSOFTFourierCoefficients[M_{{0,1,2,...,-2,-1}} x M'_{{0,1,2,...,-2,-1}}] ~> [l = {l}]\n\n")
            L, base = 2 * l + 1, l * (4 * l * l - 1) // 3
            blk = m[base:base + L * L].reshape(L, L)   # [column M'][row M]
            width, sci = _cell_format(complex(blk[j, i]) for i in range(L) for j in range(L))
            for i in range(L):
                out.append("".join(_cell(complex(blk[j, i]), width, sci) for j in range(L)) + "\n")
            out.append("\n")
        return "".join(out)


class FourierTransforms:
    """pfsoft::FourierTransforms (include/PFSOFTlib_headers/fn_fourier_transforms.hpp:75-78)."""

    @staticmethod
    def DSOFT(sample: grid3D, fc: DSOFTFourierCoefficients, threads: int | None = None) -> None:
        """Forward SO(3) Fourier transform: fc <- DSOFT(sample). ``sample`` is not modified.
        ``threads`` is accepted for interface parity and has no effect."""
        if sample.rows != sample.cols or sample.rows != sample.lays:
            _warn("DSOFT", "all DSOFT sample grid dimensions should be equal.")
            return
        if sample.rows & 1:
            _warn("DSOFT", "DSOFT sample grid dimensions are not even.")
            return
        B = sample.cols // 2
        if B != fc.bandwidth:
            _warn("DSOFT", "DSOFT Fourier coefficients container bandwidth does not match to sample grid bandwidth.")
            return
        _transform(True, sample, fc, B)

    @staticmethod
    def IDSOFT(fc: DSOFTFourierCoefficients, synthesis: grid3D, threads: int | None = None) -> None:
        """Inverse SO(3) Fourier transform: synthesis <- IDSOFT(fc)."""
        if synthesis.rows != synthesis.cols or synthesis.rows != synthesis.lays:
            _warn("IDSOFT", "all IDSOFT synthesis grid dimensions should be equal.")
            return
        if synthesis.rows & 1:
            _warn("IDSOFT", "IDSOFT synthesis grid dimensions are not even.")
            return
        B = synthesis.cols // 2
        if B != fc.bandwidth:
            _warn("IDSOFT", "IDSOFT Fourier coefficients container bandwidth does not match to synthesis grid bandwidth.")
            return
        _transform(False, synthesis, fc, B)


def _transform(forward: bool, grid: grid3D, fc: DSOFTFourierCoefficients, B: int) -> None:
    lib = _lib.load()
    if grid.on_device != fc.on_device:
        raise ValueError("grid and coefficients must both be on the host or both on the GPU")
    if grid.on_device:
        gp, cp = _dev_ptr(grid.mem), _dev_ptr(fc.mem)
        if forward:
            _lib.check(lib.pfsoft_cuda_dsoft(gp, B, cp, None, 0, _stream_ptr()))
        else:
            _lib.check(lib.pfsoft_cuda_idsoft(cp, B, gp, None, 0, _stream_ptr()))
        return
    g = grid.mem
    c = fc.mem
    if not (g.flags.c_contiguous and c.flags.c_contiguous):
        raise ValueError("host buffers must be C-contiguous")
    if forward:
        _lib.check(lib.pfsoft_dsoft_host(g.ctypes.data, B, c.ctypes.data))
    else:
        _lib.check(lib.pfsoft_idsoft_host(c.ctypes.data, B, g.ctypes.data))


class DWT:
    """pfsoft::DWT helpers (include/PFSOFTlib_headers/fn_dwt.hpp), evaluated on the GPU.
    Results are returned as numpy arrays (host) after the device computation."""

    @staticmethod
    def quadrature_weights(bandwidth: int) -> np.ndarray:
        import torch

        w = torch.empty(2 * bandwidth, dtype=torch.float64, device="cuda")
        lib = _lib.load()
        _lib.check(lib.pfsoft_cuda_quadrature_weights(bandwidth, w.data_ptr(), _stream_ptr()))
        return w.cpu().numpy()

    @staticmethod
    def _matrix(bandwidth: int, M: int, Mp: int, weighted: bool) -> np.ndarray:
        import torch

        J = max(abs(M), abs(Mp))
        out = torch.empty((bandwidth - J) * 2 * bandwidth, dtype=torch.float64, device="cuda")
        lib = _lib.load()
        _lib.check(lib.pfsoft_cuda_wigner_d_matrix(bandwidth, M, Mp, int(weighted), out.data_ptr(), _stream_ptr()))
        return out.view(bandwidth - J, 2 * bandwidth).cpu().numpy()

    @staticmethod
    def wigner_d_matrix(bandwidth: int, M: int, Mp: int) -> np.ndarray:
        """Rows l = J..B-1, columns beta_k (k < 2B), of the reference's d-matrix."""
        return DWT._matrix(bandwidth, M, Mp, False)

    @staticmethod
    def weighted_wigner_d_matrix(bandwidth: int, M: int, Mp: int) -> np.ndarray:
        return DWT._matrix(bandwidth, M, Mp, True)
