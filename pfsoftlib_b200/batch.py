"""Batch plans (C ABI ``pfsoft_batch_*``): many transforms of any bandwidths in one execution.

    plan = BatchPlan([32, 64, 64, 128], split=False)
    plan.idsoft(coeff_tensors, grid_tensors)      # lists of complex128 CUDA tensors, caller's order
    plan.dsoft(grid_tensors, coeff_tensors)
    plan.close()

A plan groups its transforms by bandwidth, runs the FFT passes batched per bandwidth and one
persistent DWT launch over every (bandwidth, order class, transform block) item, and replays the
whole sequence from a CUDA graph. Create it once per bandwidth mix (it builds tables, work lists
and the graph) and reuse it with any buffers. ``split=True`` runs the DWT of bandwidths 16..128
(multiples of 16) on the tensor cores in split precision (relative error about 1e-13 against the
FP64 path). Calls are ordered on torch's current stream unless ``stream`` is given.
"""
from __future__ import annotations

import ctypes

from . import _lib

NO_GRAPH, SPLIT = 1, 2


def _stream_handle(stream):
    import torch

    if stream is None:
        stream = torch.cuda.current_stream()
    return stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)


def _check_tensors(ts, n, what):
    import torch

    if len(ts) != n:
        raise ValueError(f"expected {n} {what} tensors, got {len(ts)}")
    for t in ts:
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.complex128 and t.is_contiguous()):
            raise TypeError(f"{what} must be contiguous complex128 CUDA tensors")


class BatchPlan:
    def __init__(self, bandwidths, transforms_per_cta: int = 0, split: bool = False, graph: bool = True):
        self._lib = _lib.load()
        self.bandwidths = [int(b) for b in bandwidths]
        flags = (0 if graph else NO_GRAPH) | (SPLIT if split else 0)
        h = ctypes.c_void_p()
        arr = (ctypes.c_int * len(self.bandwidths))(*self.bandwidths)
        _lib.check(self._lib.pfsoft_batch_create(arr, len(self.bandwidths), int(transforms_per_cta), flags,
                                                 ctypes.byref(h)))
        self._h = h

    @property
    def transforms_per_cta(self) -> int:
        return self._lib.pfsoft_batch_transforms_per_cta(self._h)

    @property
    def workspace_bytes(self) -> int:
        return self._lib.pfsoft_batch_workspace_bytes(self._h)

    def _tables(self, inputs, outputs, in_what, out_what, in_len, out_len):
        n = len(self.bandwidths)
        _check_tensors(inputs, n, in_what)
        _check_tensors(outputs, n, out_what)
        for B, x, y in zip(self.bandwidths, inputs, outputs):
            if x.numel() != in_len(B) or y.numel() != out_len(B):
                raise ValueError(f"buffer sizes do not match bandwidth {B}")
        return ((ctypes.c_void_p * n)(*[t.data_ptr() for t in inputs]),
                (ctypes.c_void_p * n)(*[t.data_ptr() for t in outputs]))

    def idsoft(self, coeffs, grids, stream=None) -> None:
        """iDSOFT of every transform: coeffs[i] (B(4B^2-1)/3) -> grids[i] ((2B)^3)."""
        cp, gp = self._tables(coeffs, grids, "coefficient", "grid", _coef_len, _grid_len)
        _lib.check(self._lib.pfsoft_batch_idsoft(self._h, cp, gp, _stream_handle(stream)))

    def dsoft(self, grids, coeffs, stream=None) -> None:
        """DSOFT of every transform: grids[i] -> coeffs[i]; the grids are not modified."""
        gp, cp = self._tables(grids, coeffs, "grid", "coefficient", _grid_len, _coef_len)
        _lib.check(self._lib.pfsoft_batch_dsoft(self._h, gp, cp, _stream_handle(stream)))

    def status(self) -> None:
        """Raises if a bounded wait in the split-precision kernel ever ran out (synchronises)."""
        _lib.check(self._lib.pfsoft_batch_status(self._h))

    def close(self) -> None:
        if self._h:
            self._lib.pfsoft_batch_destroy(self._h)
            self._h = None

    def __enter__(self) -> "BatchPlan":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _coef_len(B: int) -> int:
    return B * (4 * B * B - 1) // 3


def _grid_len(B: int) -> int:
    return (2 * B) ** 3


def split_supported(B: int) -> bool:
    return bool(_lib.load().pfsoft_split_supported(int(B)))
