"""Project autotuner for the batched engine.

For a multiset of bandwidths it times each candidate schedule -- transforms per CTA in the
fused DWT launch (1, 2, 4), i.e. how many transforms share one on-chip Wigner recurrence -- on
the device with CUDA events, and caches the winner in a JSON table keyed by GPU name and the
sorted bandwidth counts. ``choose`` is the pure decision rule (tested on CPU); ``tune_batch``
does the timing.
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
