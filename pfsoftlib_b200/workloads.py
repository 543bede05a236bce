"""Runs one execution of a named workload through the C ABI (used for profiling and as a usage
example). ``python -m pfsoftlib_b200.workloads <name> [reps]``:

  single-<B>      IDSOFT then DSOFT of one transform at bandwidth B (PCG64-seeded inputs)
  batch-<B>x<T>   a batch plan of T transforms at bandwidth B, IDSOFT then DSOFT
  mixed           256 transforms, B uniform over {32,48,64,96,128} (seed 2), batched
  <name>-split    a batch or mixed workload through the split-precision tensor-core DWT
  <name>-fusedfft any of the above with both FFT passes of a direction in one launch
                  (pfsoft_tune_fft_fused), restored to the default afterwards
  shard-<B>x<P>   IDSOFT then DSOFT of one transform sharded over P ranks, the ranks run one after
                  another on this GPU (the all-to-all as device copies between their buffers)
  slab-<B>x<P>    the forward and inverse FFT passes of rank 0's layer slab of a P-rank plan
"""
from __future__ import annotations

import ctypes
import sys

import numpy as np


def _coeffs(lib, B, seed, torch, s):
    c = torch.empty(B * (4 * B * B - 1) // 3, dtype=torch.complex128, device="cuda")
    assert lib.pfsoft_cuda_random_coeffs(c.data_ptr(), B, seed, 1, 1.0, s) == 0
    return c


def run(name: str, reps: int = 1) -> float:
    import torch

    from . import load

    lib = load()
    if name.endswith("-fusedfft"):
        assert lib.pfsoft_tune_fft_fused(0, 1) == 0
        try:
            return run(name[: -len("-fusedfft")], reps)
        finally:
            lib.pfsoft_tune_fft_fused(0, 0)
    s = torch.cuda.current_stream().cuda_stream
    if name.startswith("single-"):
        B = int(name.split("-")[1])
        N = 2 * B
        c = _coeffs(lib, B, 1, torch, s)
        g = torch.empty((N, N, N), dtype=torch.complex128, device="cuda")
        f = torch.empty_like(c)
        for _ in range(reps):
            assert lib.pfsoft_cuda_idsoft(c.data_ptr(), B, g.data_ptr(), None, 0, s) == 0
            assert lib.pfsoft_cuda_dsoft(g.data_ptr(), B, f.data_ptr(), None, 0, s) == 0
        torch.cuda.synchronize()
        return (f - c).abs().max().item()
    split = name.endswith("-split")
    if split:
        name = name[: -len("-split")]
    if name.startswith("batch-") or name == "mixed":
        if name == "mixed":
            bws = [int(b) for b in np.random.default_rng(2).choice((32, 48, 64, 96, 128), size=256)]
        else:
            B, T = (int(x) for x in name.split("-")[1].split("x"))
            bws = [B] * T
        cs = [_coeffs(lib, B, 2000 + i, torch, s) for i, B in enumerate(bws)]
        gs = [torch.empty((2 * B,) * 3, dtype=torch.complex128, device="cuda") for B in bws]
        fs = [torch.empty_like(c) for c in cs]
        plan = ctypes.c_void_p()
        arr = (ctypes.c_int * len(bws))(*bws)
        assert lib.pfsoft_batch_create(arr, len(bws), 0, 1 | (2 if split else 0), ctypes.byref(plan)) == 0
        cp = (ctypes.c_void_p * len(bws))(*[t.data_ptr() for t in cs])
        gp = (ctypes.c_void_p * len(bws))(*[t.data_ptr() for t in gs])
        fp = (ctypes.c_void_p * len(bws))(*[t.data_ptr() for t in fs])
        for _ in range(reps):
            assert lib.pfsoft_batch_idsoft(plan, cp, gp, s) == 0
            assert lib.pfsoft_batch_dsoft(plan, gp, fp, s) == 0
        torch.cuda.synchronize()
        lib.pfsoft_batch_destroy(plan)
        return max((f - c).abs().max().item() for f, c in zip(fs, cs))
    if name.startswith("shard-") or name.startswith("slab-"):
        return _sharded(name, reps, lib, torch, s)
    raise ValueError(f"unknown workload {name}")


def _sharded(name, reps, lib, torch, s):
    from .shard import FORWARD, INVERSE, ShardPlan

    B, P = (int(x) for x in name.split("-")[1].split("x"))
    N = 2 * B
    cplx = dict(dtype=torch.complex128, device="cuda")
    if name.startswith("slab-"):
        plan = ShardPlan(B, P, 0)
        nk = plan.layers[1]
        g = torch.randn(nk * N * N, **cplx)
        spec, back = torch.empty_like(g), torch.empty_like(g)
        for _ in range(reps):
            plan.fft_forward(g, spec)
            plan.fft_inverse(spec, back)
        torch.cuda.synchronize()
        return 0.0   # the Nyquist bins are dropped on the way back: no round-trip identity
    plans = [ShardPlan(B, P, r) for r in range(P)]
    c = _coeffs(lib, B, 1, torch, s)
    f = torch.empty_like(c)
    spectra = [torch.empty(N ** 3, **cplx) for _ in range(P)]
    slabs = [torch.empty(p.slab_elems(), **cplx) for p in plans]
    grids = [torch.empty(p.slab_elems(), **cplx) for p in plans]

    def exchange(direction, srcs, dsts):
        sends = []
        for p in range(P):
            sends.append(torch.empty(sum(plans[p].counts(direction)[0]), **cplx))
            plans[p].pack(direction, srcs[p], sends[p])
        for q in range(P):
            recv = torch.empty(sum(plans[q].counts(direction)[1]), **cplx)
            ro = np.concatenate([[0], np.cumsum(plans[q].counts(direction)[1])])
            for p in range(P):
                so = np.concatenate([[0], np.cumsum(plans[p].counts(direction)[0])])
                recv[ro[p]:ro[p + 1]] = sends[p][so[q]:so[q + 1]]
            plans[q].unpack(direction, recv, dsts[q])

    for _ in range(reps):
        for q in range(P):
            plans[q].dwt_inverse(c, spectra[q])
        exchange(INVERSE, spectra, slabs)
        for p in range(P):
            plans[p].fft_inverse(slabs[p], grids[p])
            plans[p].fft_forward(grids[p], slabs[p])
        exchange(FORWARD, slabs, spectra)
        f.zero_()
        part = torch.empty_like(c)
        for q in range(P):
            plans[q].dwt_forward(spectra[q], part)
            f += part
    torch.cuda.synchronize()
    return (f - c).abs().max().item()


if __name__ == "__main__":
    err = run(sys.argv[1], int(sys.argv[2]) if len(sys.argv) > 2 else 1)
    print(f"{sys.argv[1]}: round-trip max abs {err:.3e}")
