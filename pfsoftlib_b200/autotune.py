"""Project autotuner for the batched engine.

For a multiset of bandwidths it times candidate schedules on the device with CUDA events and
caches the winners in a JSON table keyed by GPU name and the sorted bandwidth counts:

  tune_batch  transforms per CTA of the fused FP64 DWT launch (1, 2, 4), i.e. how many
              transforms share one on-chip Wigner recurrence;
  tune_plan   per bandwidth: the FFT stage as one fused launch or two passes
              (pfsoft_tune_fft_fused), and the DWT of a PFSOFT_BATCH_SPLIT plan on the
              split-precision kernel or the FP64 kernels (pfsoft_tune_split_bandwidth); the
              choices are applied to the library and returned.

``choose`` is the pure decision rule (tested on CPU); the tune_* functions do the timing.
"""
from __future__ import annotations

import ctypes
import json
import os
from collections import Counter

CANDIDATES = (1, 2, 4)


def cache_path() -> str:
    d = os.environ.get("PFSOFT_B200_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "pfsoft_b200"))
    return os.path.join(d, "autotune.json")


def key_for(gpu: str, bandwidths) -> str:
    c = Counter(int(b) for b in bandwidths)
    return gpu + "|" + ",".join(f"{b}x{c[b]}" for b in sorted(c))


def choose(timings: dict) -> int:
    """The fastest candidate; ties go to the smaller value (less register and idle-warp cost)."""
    if not timings:
        raise ValueError("no timings")
    return min(sorted(timings), key=lambda k: (timings[k], k))


def load_cache(path: str | None = None) -> dict:
    path = path or cache_path()
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def store(key: str, value: int, path: str | None = None) -> None:
    path = path or cache_path()
    data = load_cache(path)
    data[key] = value
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path + ".tmp", "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(path + ".tmp", path)
    except OSError:
        pass


def tune_batch(lib, bandwidths, coeffs, grids, back, reps: int = 2, use_cache: bool = True) -> tuple[int, dict]:
    """Time a round trip (IDSOFT then DSOFT) of the batch for each candidate; returns the
    chosen transforms-per-CTA and the timings in ms. Buffers are lists of CUDA tensors."""
    import torch

    gpu = torch.cuda.get_device_name()
    key = key_for(gpu, bandwidths)
    if use_cache:
        cached = load_cache().get(key)
        if cached in CANDIDATES:
            return cached, {}
    arr = (ctypes.c_int * len(bandwidths))(*[int(b) for b in bandwidths])
    cp = (ctypes.c_void_p * len(coeffs))(*[t.data_ptr() for t in coeffs])
    gp = (ctypes.c_void_p * len(grids))(*[t.data_ptr() for t in grids])
    bp = (ctypes.c_void_p * len(back))(*[t.data_ptr() for t in back])
    s = torch.cuda.current_stream().cuda_stream
    timings = {}
    for tpc in CANDIDATES:
        plan = ctypes.c_void_p()
        if lib.pfsoft_batch_create(arr, len(bandwidths), tpc, 0, ctypes.byref(plan)) != 0:
            continue
        try:
            lib.pfsoft_batch_idsoft(plan, cp, gp, s)
            lib.pfsoft_batch_dsoft(plan, gp, bp, s)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                lib.pfsoft_batch_idsoft(plan, cp, gp, s)
                lib.pfsoft_batch_dsoft(plan, gp, bp, s)
            e1.record()
            torch.cuda.synchronize()
            timings[tpc] = e0.elapsed_time(e1) / reps
        finally:
            lib.pfsoft_batch_destroy(plan)
    best = choose(timings)
    store(key, best)
    return best, timings


def _time_ms(fn, reps: int) -> float:
    import torch

    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def apply(lib, plan: dict) -> None:
    """Sets the library's per-bandwidth knobs from a plan returned by tune_plan."""
    for b, on in plan.get("fft_fused", {}).items():
        lib.pfsoft_tune_fft_fused(int(b), int(bool(on)))
    for b, on in plan.get("split", {}).items():
        lib.pfsoft_tune_split_bandwidth(int(b), int(bool(on)))


def tune_plan(lib, bandwidths, coeffs, grids, back, reps: int = 2, use_cache: bool = True) -> dict:
    """Per distinct bandwidth of the mix: (1) the FFT stage fused or as two passes, timed on a
    single-transform round trip; (2) the DWT of a split plan on the split kernel or the FP64
    kernels, timed on a batch plan of that bandwidth's transforms (FFT choice applied). Applies the
    winners (apply) and returns {"fft_fused": {B: bool}, "split": {B: bool}, "ms": {...}}.
    Buffers are lists of CUDA tensors in the order of `bandwidths`."""
    import torch

    gpu = torch.cuda.get_device_name()
    key = "plan|" + key_for(gpu, bandwidths)
    if use_cache:
        cached = load_cache().get(key)
        if isinstance(cached, dict) and "fft_fused" in cached and "split" in cached:
            apply(lib, cached)
            return cached
    s = torch.cuda.current_stream().cuda_stream
    out = {"fft_fused": {}, "split": {}, "ms": {"fft": {}, "dwt": {}}}
    for b in sorted(set(int(x) for x in bandwidths)):
        idx = [i for i, x in enumerate(bandwidths) if int(x) == b]
        i0 = idx[0]
        ws = torch.empty(lib.pfsoft_workspace_bytes(b) // 8, dtype=torch.float64, device="cuda")

        def single():
            lib.pfsoft_cuda_idsoft(coeffs[i0].data_ptr(), b, grids[i0].data_ptr(), ws.data_ptr(), ws.numel() * 8, s)
            lib.pfsoft_cuda_dsoft(grids[i0].data_ptr(), b, back[i0].data_ptr(), ws.data_ptr(), ws.numel() * 8, s)

        t = {}
        for on in (1, 0):
            lib.pfsoft_tune_fft_fused(b, on)
            t[on] = _time_ms(single, reps)
        fused = t[1] <= t[0]
        lib.pfsoft_tune_fft_fused(b, int(fused))
        out["fft_fused"][str(b)] = fused
        out["ms"]["fft"][str(b)] = {"fused": t[1], "two_passes": t[0]}
        del ws
        arr = (ctypes.c_int * len(idx))(*[b] * len(idx))
        cp = (ctypes.c_void_p * len(idx))(*[coeffs[i].data_ptr() for i in idx])
        gp = (ctypes.c_void_p * len(idx))(*[grids[i].data_ptr() for i in idx])
        bp = (ctypes.c_void_p * len(idx))(*[back[i].data_ptr() for i in idx])
        d = {}
        for flags in (0, 2):
            lib.pfsoft_tune_split_bandwidth(b, 1)
            plan = ctypes.c_void_p()
            if lib.pfsoft_batch_create(arr, len(idx), 0, flags | 1, ctypes.byref(plan)) != 0:
                continue
            try:
                d[flags] = _time_ms(lambda: (lib.pfsoft_batch_idsoft(plan, cp, gp, s),
                                             lib.pfsoft_batch_dsoft(plan, gp, bp, s)), reps)
            finally:
                lib.pfsoft_batch_destroy(plan)
        split = 2 in d and (0 not in d or d[2] <= d[0])
        lib.pfsoft_tune_split_bandwidth(b, int(split))
        out["split"][str(b)] = split
        out["ms"]["dwt"][str(b)] = {"split": d.get(2), "fp64": d.get(0), "transforms": len(idx)}
    store(key, out)
    return out
