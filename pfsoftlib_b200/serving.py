"""Transform server: a persistent request loop with continuous batching (C ABI ``pfsoft_server_*``).

The reference transforms one grid per call (src/fn_dsoft.cpp:76, src/fn_idsoft.cpp:72); here each
such call becomes a request against a server that keeps the data on the device:

    srv = TransformServer(budget_bytes=8 << 30, max_batch=16, streams=4)
    req = srv.dsoft(grid, coeffs)        # device tensors: (2B)^3 complex128 grid, packed coeffs
    req.wait()                           # raises PfsoftError unless the request succeeded
    srv.stats()                          # p50 / p99 latency, transforms/s, batches, arena peak

Requests of equal direction and bandwidth that wait together run as one batch; a batch starts as
soon as a stream and room in the workspace arena (the HBM budget) are free, while earlier
batches are still on the device. With ``split=True`` a batch takes waiting requests of one
direction and any bandwidths up to 256 and runs their Wigner transforms in one split-precision
tensor-core launch (``PFSOFT_SERVER_SPLIT``). A request keeps references to its tensors until it
finishes.
"""
from __future__ import annotations

import ctypes

from . import _lib

DSOFT, IDSOFT = 0, 1
SERVER_SPLIT = 1


class ServerStats(ctypes.Structure):
    _fields_ = [
        ("submitted", ctypes.c_longlong), ("completed", ctypes.c_longlong),
        ("cancelled", ctypes.c_longlong), ("rejected", ctypes.c_longlong),
        ("failed", ctypes.c_longlong), ("batches", ctypes.c_longlong),
        ("mean_batch", ctypes.c_double),
        ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
        ("mean_ms", ctypes.c_double), ("max_ms", ctypes.c_double),
        ("wall_s", ctypes.c_double), ("transforms_per_s", ctypes.c_double),
        ("budget_bytes", ctypes.c_size_t), ("peak_bytes", ctypes.c_size_t),
        ("max_concurrent_batches", ctypes.c_int),
        ("queued", ctypes.c_int), ("running", ctypes.c_int),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


def _bandwidth_of_grid(grid) -> int:
    n = grid.shape[0] if grid.dim() == 3 else round(grid.numel() ** (1 / 3))
    if n % 2 or n ** 3 != grid.numel():
        raise ValueError("grid must hold (2B)^3 complex values")
    return n // 2


class Request:
    """One queued transform. ``wait`` / ``done`` read its final status once."""

    def __init__(self, server: "TransformServer", rid: int, keep: tuple):
        self.server = server
        self.id = rid
        self._keep = keep          # the tensors, alive until the request finished
        self.status: int | None = None

    def _finish(self, rc: int) -> bool:
        if rc == _lib.PFSOFT_EBUSY:
            return False
        self.status = rc
        self._keep = ()
        return True

    def done(self) -> bool:
        if self.status is not None:
            return True
        return self._finish(self.server._lib.pfsoft_server_poll(self.server._h, self.id))

    def wait(self, timeout: float = 60.0) -> None:
        if self.status is None:
            rc = self.server._lib.pfsoft_server_wait(self.server._h, self.id, float(timeout))
            if rc == _lib.PFSOFT_ETIMEOUT:
                raise _lib.PfsoftError(rc, f"request {self.id} still busy after {timeout} s")
            self._finish(rc)
        if self.status != _lib.PFSOFT_OK:
            raise _lib.PfsoftError(self.status, self.server._lib.pfsoft_status_string(self.status).decode())

    def cancel(self) -> bool:
        """True if the request was still queued (it then finishes as cancelled)."""
        return self.server._lib.pfsoft_server_cancel(self.server._h, self.id) == _lib.PFSOFT_OK


class TransformServer:
    def __init__(self, budget_bytes: int = 160 << 30, max_batch: int = 16, streams: int = 4, split: bool = False):
        self._lib = _lib.load()
        self._h = None
        h = ctypes.c_void_p()
        _lib.check(self._lib.pfsoft_server_create_ex(int(budget_bytes), int(max_batch), int(streams),
                                                     SERVER_SPLIT if split else 0, ctypes.byref(h)))
        self._h = h
        self.split = bool(split)

    # -- requests --------------------------------------------------------------------------
    def submit(self, direction: int, B: int, inp, out, stream=None) -> Request:
        """Queue DSOFT (direction 0: grid -> coefficients) or iDSOFT (1). ``stream`` defaults to
        torch's current stream: the request waits for the work queued there before it runs."""
        import torch

        for t in (inp, out):
            if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.complex128 and t.is_contiguous()):
                raise TypeError("requests take contiguous complex128 CUDA tensors")
        if stream is None:
            stream = torch.cuda.current_stream(inp.device)
        sp = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
        rid = ctypes.c_longlong()
        _lib.check(self._lib.pfsoft_server_submit(self._h, int(direction), int(B), inp.data_ptr(), out.data_ptr(),
                                                  sp, ctypes.byref(rid)))
        return Request(self, rid.value, (inp, out))

    def dsoft(self, grid, coeffs, stream=None) -> Request:
        B = _bandwidth_of_grid(grid)
        if coeffs.numel() != B * (4 * B * B - 1) // 3:
            raise ValueError("coefficient buffer does not match the grid's bandwidth")
        return self.submit(DSOFT, B, grid, coeffs, stream)

    def idsoft(self, coeffs, grid, stream=None) -> Request:
        B = _bandwidth_of_grid(grid)
        if coeffs.numel() != B * (4 * B * B - 1) // 3:
            raise ValueError("coefficient buffer does not match the grid's bandwidth")
        return self.submit(IDSOFT, B, coeffs, grid, stream)

    # -- control ---------------------------------------------------------------------------
    def pause(self) -> None:
        _lib.check(self._lib.pfsoft_server_pause(self._h, 1))

    def resume(self) -> None:
        _lib.check(self._lib.pfsoft_server_pause(self._h, 0))

    def drain(self, timeout: float = 60.0) -> None:
        _lib.check(self._lib.pfsoft_server_drain(self._h, float(timeout)))

    def stats(self) -> dict:
        st = ServerStats()
        _lib.check(self._lib.pfsoft_server_get_stats(self._h, ctypes.byref(st)))
        return st.as_dict()

    def reset_stats(self) -> None:
        _lib.check(self._lib.pfsoft_server_reset_stats(self._h))

    def close(self) -> None:
        if self._h:
            self._lib.pfsoft_server_destroy(self._h)
            self._h = None

    def __enter__(self) -> "TransformServer":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
