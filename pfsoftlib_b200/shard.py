"""One SO(3) transform sharded over the ranks of a process group (C ABI ``pfsoft_shard_*``).

    dist.init_process_group("nccl")                 # one process per GPU
    st = ShardedTransform(B=256)
    first, count = st.layers                        # this rank's beta layers of the (2B)^3 grid
    coeffs = st.dsoft(grid[first:first + count])    # every rank gets all B(4B^2-1)/3 coefficients
    slab = st.idsoft(coeffs)                        # this rank's layers of the inverse

Rank r runs the layer-wise FFT passes on its slab of beta layers and the DWT of its share of the
order classes; one all-to-all between the two stages moves the FFT bins to the ranks whose classes
need them (``torch.distributed.all_to_all_single``: NCCL over NVLink), and an all-reduce sums the
per-rank coefficient vectors (each rank writes zeros outside its classes). ``ShardPlan`` is the
plan of one rank with the step functions; the host-only queries (layers, counts, bins, copy runs)
work without a GPU.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

FORWARD, INVERSE = 0, 1
SCATTER, PACK, UNPACK = 0, 1, 2


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _stream_handle(stream):
    import torch

    if stream is None:
        stream = torch.cuda.current_stream()
    return stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)


def _check(t, n, what):
    import torch

    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.complex128 and t.is_contiguous()):
        raise TypeError(f"{what} must be a contiguous complex128 CUDA tensor")
    if t.numel() != n:
        raise ValueError(f"{what} has {t.numel()} values, expected {n}")


class ShardPlan:
    """Plan of rank ``rank`` of ``nranks`` for bandwidth-B transforms."""

    def __init__(self, B: int, nranks: int, rank: int):
        self._lib = _lib.load()
        self.B, self.N, self.nranks, self.rank = int(B), 2 * int(B), int(nranks), int(rank)
        h = ctypes.c_void_p()
        _lib.check(self._lib.pfsoft_shard_create(self.B, self.nranks, self.rank, ctypes.byref(h)))
        self._h = h

    # ---- host-only queries ----------------------------------------------------------------
    def layers_of(self, r: int) -> tuple[int, int]:
        first, count = ctypes.c_int(), ctypes.c_int()
        _lib.check(self._lib.pfsoft_shard_layers(self._h, r, ctypes.byref(first), ctypes.byref(count)))
        return first.value, count.value

    @property
    def layers(self) -> tuple[int, int]:
        return self.layers_of(self.rank)

    def classes(self, r: int) -> np.ndarray:
        n = self._lib.pfsoft_shard_classes(self._h, r, None, 0)
        out = np.zeros(n, dtype=np.int32)
        self._lib.pfsoft_shard_classes(self._h, r, out.ctypes.data, n)
        return out

    def bins(self, r: int) -> np.ndarray:
        n = self._lib.pfsoft_shard_bins(self._h, r, None, 0)
        out = np.zeros(n, dtype=np.int32)
        self._lib.pfsoft_shard_bins(self._h, r, out.ctypes.data, n)
        return out

    def counts(self, direction: int) -> tuple[list, list]:
        """Complex values this rank sends to and receives from each rank in an exchange."""
        send = np.zeros(self.nranks, dtype=np.int64)
        recv = np.zeros(self.nranks, dtype=np.int64)
        _lib.check(self._lib.pfsoft_shard_counts(self._h, direction, send.ctypes.data, recv.ctypes.data))
        return send.tolist(), recv.tolist()

    def runs(self, direction: int, step: int) -> dict:
        """Copy runs of an exchange step: run i copies len[i] values from src + src_off[i] to
        buffer slot[i] + dst_off[i]."""
        n = self._lib.pfsoft_shard_runs(self._h, direction, step, None, None, None, None, 0)
        if n < 0:
            raise ValueError("bad direction or step")
        out = {"src_off": np.zeros(n, np.int64), "dst_off": np.zeros(n, np.int64),
               "slot": np.zeros(n, np.int32), "len": np.zeros(n, np.int32)}
        self._lib.pfsoft_shard_runs(self._h, direction, step, out["src_off"].ctypes.data, out["dst_off"].ctypes.data,
                                    out["slot"].ctypes.data, out["len"].ctypes.data, n)
        return out

    def slab_elems(self, r: int | None = None) -> int:
        return self.layers_of(self.rank if r is None else r)[1] * self.N * self.N

    def spectrum_elems(self) -> int:
        return self.N ** 3

    def coef_elems(self) -> int:
        return self.B * (4 * self.B * self.B - 1) // 3

    # ---- device steps (stream ordered) --------------------------------------------------------
    def fft_forward(self, slab_grid, slab_spectrum, stream=None) -> None:
        _check(slab_grid, self.slab_elems(), "slab grid")
        _check(slab_spectrum, self.slab_elems(), "slab spectrum")
        _lib.check(self._lib.pfsoft_shard_fft_forward(self._h, _ptr(slab_grid), _ptr(slab_spectrum),
                                                      _stream_handle(stream)))

    def fft_inverse(self, slab_spectrum, slab_grid, stream=None) -> None:
        _check(slab_grid, self.slab_elems(), "slab grid")
        _check(slab_spectrum, self.slab_elems(), "slab spectrum")
        _lib.check(self._lib.pfsoft_shard_fft_inverse(self._h, _ptr(slab_spectrum), _ptr(slab_grid),
                                                      _stream_handle(stream)))

    def dwt_forward(self, spectrum, coeffs, stream=None) -> None:
        _check(spectrum, self.spectrum_elems(), "spectrum")
        _check(coeffs, self.coef_elems(), "coefficients")
        _lib.check(self._lib.pfsoft_shard_dwt_forward(self._h, _ptr(spectrum), _ptr(coeffs), _stream_handle(stream)))

    def dwt_inverse(self, coeffs, spectrum, stream=None) -> None:
        _check(spectrum, self.spectrum_elems(), "spectrum")
        _check(coeffs, self.coef_elems(), "coefficients")
        _lib.check(self._lib.pfsoft_shard_dwt_inverse(self._h, _ptr(coeffs), _ptr(spectrum), _stream_handle(stream)))

    def _side(self, direction: int, source: bool) -> tuple[int, str]:
        """Size and name of the exchange's source (source=True) or destination buffer here."""
        if direction not in (FORWARD, INVERSE):
            raise ValueError("direction must be FORWARD or INVERSE")
        slab = (direction == FORWARD) == source
        return (self.slab_elems(), "slab spectrum") if slab else (self.spectrum_elems(), "spectrum")

    def scatter(self, direction: int, src, dsts, stream=None) -> None:
        """Direct stores into every rank's buffer (dsts: one tensor or device address per rank;
        the spectra in the forward direction, the slab spectra in the inverse)."""
        _check(src, *self._side(direction, True))
        if len(dsts) != self.nranks:
            raise ValueError(f"expected {self.nranks} destination buffers")
        addr = [0 if d is None else (d if isinstance(d, int) else d.data_ptr()) for d in dsts]
        table = (ctypes.c_void_p * self.nranks)(*addr)
        _lib.check(self._lib.pfsoft_shard_scatter(self._h, direction, _ptr(src), table, _stream_handle(stream)))

    def pack(self, direction: int, src, send, stream=None) -> None:
        _check(src, *self._side(direction, True))
        _check(send, sum(self.counts(direction)[0]), "send buffer")
        _lib.check(self._lib.pfsoft_shard_pack(self._h, direction, _ptr(src), _ptr(send), _stream_handle(stream)))

    def unpack(self, direction: int, recv, dst, stream=None) -> None:
        _check(recv, sum(self.counts(direction)[1]), "receive buffer")
        _check(dst, *self._side(direction, False))
        _lib.check(self._lib.pfsoft_shard_unpack(self._h, direction, _ptr(recv), _ptr(dst), _stream_handle(stream)))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.pfsoft_shard_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _as_real(t):
    import torch

    return torch.view_as_real(t).reshape(-1) if t.is_complex() else t


class ShardedTransform:
    """DSOFT / iDSOFT of one bandwidth-B transform over all ranks of ``group``.

    ``engine`` is the step implementation (a ShardPlan by default); buffers live on ``device``
    (the current CUDA device by default). Every rank must call dsoft / idsoft in the same order.
    """

    def __init__(self, B: int, group=None, device=None, engine=None):
        import torch
        import torch.distributed as dist

        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.plan = engine if engine is not None else ShardPlan(B, self.world, self.rank)
        self.B, self.N = self.plan.B, self.plan.N
        self.device = torch.device(device) if device is not None else (
            torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else torch.device("cpu"))
        self.counts = {d: self.plan.counts(d) for d in (FORWARD, INVERSE)}
        self._buf = {}

    @property
    def layers(self) -> tuple[int, int]:
        return self.plan.layers

    def _get(self, name, n):
        import torch

        t = self._buf.get(name)
        if t is None or t.numel() != n:
            t = torch.empty(n, dtype=torch.complex128, device=self.device)
            self._buf[name] = t
        return t

    def _exchange(self, direction, src, dst):
        import torch.distributed as dist

        send_n, recv_n = self.counts[direction]
        send = self._get("send", sum(send_n))
        recv = self._get("recv", sum(recv_n))
        self.plan.pack(direction, src, send)
        # complex values travel as pairs of doubles
        dist.all_to_all_single(_as_real(recv), _as_real(send), [2 * c for c in recv_n], [2 * c for c in send_n],
                               group=self.group)
        self.plan.unpack(direction, recv, dst)

    def dsoft(self, slab_grid, out=None, gather: bool = True):
        """DSOFT of the grid whose layers [first, first + count) this rank holds (slab_grid:
        count * N * N complex values). Returns the whole coefficient vector on every rank, or with
        gather=False this rank's part: its classes' coefficients, zero elsewhere (no collective;
        idsoft accepts it as it is, since each rank reads only its own classes)."""
        import torch.distributed as dist

        slab_spec = self._get("slab_spectrum", self.plan.slab_elems())
        spectrum = self._get("spectrum", self.plan.spectrum_elems())
        coeffs = out if out is not None else self._get_out(self.plan.coef_elems())
        self.plan.fft_forward(slab_grid.reshape(-1), slab_spec)
        self._exchange(FORWARD, slab_spec, spectrum)
        self.plan.dwt_forward(spectrum, coeffs)
        if gather:
            dist.all_reduce(_as_real(coeffs), group=self.group)
        return coeffs

    def idsoft(self, coeffs, out=None):
        """iDSOFT of a coefficient vector: the whole vector, or this rank's part of it (only the
        rank's own classes are read). Returns this rank's layers [first, first + count) of the
        grid as a (count, N, N) tensor."""
        nk = self.layers[1]
        slab_spec = self._get("slab_spectrum", self.plan.slab_elems())
        spectrum = self._get("spectrum", self.plan.spectrum_elems())
        slab = out if out is not None else self._get_out(nk * self.N * self.N)
        self.plan.dwt_inverse(coeffs.reshape(-1), spectrum)
        self._exchange(INVERSE, spectrum, slab_spec)
        self.plan.fft_inverse(slab_spec, slab.reshape(-1))
        return slab.reshape(nk, self.N, self.N)

    def _get_out(self, n):
        import torch

        return torch.empty(n, dtype=torch.complex128, device=self.device)
