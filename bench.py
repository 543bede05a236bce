"""Benchmark: DSOFT + iDSOFT transforms/s at bandwidth B = 128 (one B200 per rank).

One step = one iDSOFT (2,796,160 coefficients -> 256^3 complex128 grid) followed by one DSOFT
of that grid (the single-transform workload at B = 128), i.e. 2 transforms per step, on the FP64
drop-in path. Inputs are seeded synthetic coefficients: uniform phase, magnitude
(1+l)^-1 |N(0,1)|, PCG64 seed 1.

  value     transforms/s with everything resident in HBM, device time (CUDA events) over the
            K timed steps, max over ranks; every buffer (268 MB grid) exceeds the 126 MB L2.
  e2e       the same metric through the host-facing C ABI (pfsoft_idsoft_host /
            pfsoft_dsoft_host) from pinned host memory, copies inside the timed region;
            e2e_pageable the same from pageable memory (what the C++ drop-in header hands over).
  roofline  the dominant stage, timed with CUDA events per stage inside the timed region.
  cpu_baseline  the reference's own CPU DSOFT/IDSOFT (compiled from its sources with a project
            FFT in FFTW's place) on a bounded sample, rank 0 at N = 1 only.
At N = 1 the line also carries the other workloads in compact form (skip with --no-extras):
  mixed     256 transforms of uneven bandwidth: plain FP64 loop, FP64 batch, split-precision
            batch, split-precision server (saturated), with errors against FP64 and the oracle.
  b256      8 transforms at B = 256: FP64 batch against the split-precision batch, errors against
            FP64 and the reference CPU DSOFT.
  serving   Poisson arrivals, bandwidths log-uniform over the integers 16..256: p50 / p99 latency
            and transforms/s of the split-precision server and of the plain per-request FP64 path.

--impl reference times the reference CPU implementation alone on the host cores.
Multi-GPU (torchrun): every rank runs its own transforms (independent replicas, weak scaling);
no collective touches the data path.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

B = 128
N = 2 * B
METRIC = "DSOFT+iDSOFT transforms/s at B=128"
UNIT = "transforms/s"
TRANSFORMS_PER_STEP = 2
GRID_BYTES = N ** 3 * 16
COEF_COUNT = B * (4 * B * B - 1) // 3
COEF_BYTES = COEF_COUNT * 16
FP64_PEAK_TFLOPS = 37.0   # mma.sync m8n8k4 f64 measured on B200 (DFMA 33.5), pfsoftlib_b200/peaks

# algorithmic work per transform:
#   each FFT pass reads and writes the grid once: 32 N^3 bytes
#   each DWT does 8 B^2 (4B^2-1)/3 useful FP64 flops
FFT_PASS_BYTES = 2 * GRID_BYTES
DWT_FLOPS = 8 * B * B * (4 * B * B - 1) / 3


def workload_config() -> dict:
    return {
        "workload": "single transform at B=128: iDSOFT of 2,796,160 complex128 coefficients to a "
                    "256^3 complex128 grid, then DSOFT of that grid",
        "B": B,
        "grid": "256x256x256 complex128 (268 MB)",
        "coefficients": COEF_COUNT,
        "transforms_per_step": TRANSFORMS_PER_STEP,
        "inputs": "seeded synthetic (PCG64 seed 1): uniform phase, |f| = (1+l)^-1 |N(0,1)|",
        "l2": "inputs larger than L2: 268 MB grid and workspace, 45 MB coefficients",
    }


def measured_peaks() -> dict:
    """HBM copy bandwidth of this pool's B200s from MEASURED_PEAKS.json (written next to this
    file by the machine's operators), else the pool's earlier fallback figure."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured (MEASURED_PEAKS.json hbm_gbs)"}
    except (OSError, ValueError, KeyError, TypeError):
        return {"hbm_gbs": 6650.0, "source": "fallback 6.65 TB/s (MEASURED_PEAKS.json absent)"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="pfsoft", choices=["pfsoft", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="single", choices=["single", "mixed", "serve", "b256", "shard"],
                    help="single: the B=128 headline; mixed: 256 transforms of uneven bandwidth, batched "
                         "(FP64 and split precision) and served vs plain loop; serve: Poisson sweep of the server; "
                         "b256: 64 transforms at B=256 in groups of 8; shard: one B=256 transform sharded over "
                         "the ranks (strong scaling)")
    ap.add_argument("--rates", default="50,100,200,500,1000,2000", help="serve: offered requests/s")
    ap.add_argument("--seconds", type=float, default=5.2,
                    help="serve: arrival window per rate (5.2 s over the default rates: ~20,000 requests per arm)")
    ap.add_argument("--budget-gb", type=float, default=160.0, help="serve: HBM budget of the server's arena")
    ap.add_argument("--no-extras", action="store_true", help="single: skip the mixed / b256 / serving sections")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ----------------------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active," \
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.f = None

    def start(self):
        try:
            self.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        self.f.close()
        os.unlink(self.f.name)
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
                power.append(float(r[3]))
                for i, nm in enumerate(names):
                    if r[5 + i].strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "power_w_max": max(power) if power else None, "samples": len(sm), "reasons": sorted(reasons)}


# ----------------------------------------------------------------------------- reference arm

def cpu_reference_sample(steps: int, warmup: int, coeffs) -> dict:
    """Times the reference CPU DSOFT/IDSOFT (all host threads) at B = 128."""
    from oracle import oracle as orc

    if orc.Reference.available():
        ref = orc.Reference()
        kind = "reference"
        threads = ref.max_threads()
        timer = orc.ReferenceTimer(ref, B, coeffs)
        for _ in range(warmup):
            timer.idsoft(threads)
            timer.dsoft(threads)
        t = 0.0
        for _ in range(steps):
            t += timer.idsoft(threads)
            t += timer.dsoft(threads)
        timer.close()
        sample = (f"{steps} x (IDSOFT + DSOFT) at B=128 after {warmup} warm-up, reference sources "
                  f"compiled -O3 -fopenmp with the project FFT in FFTW's slot; timing as "
                  f"benchmark/benchmark_dsoft_for.cpp (by-value grid copy included)")
    else:
        ora = orc.Oracle()
        kind = "port"
        threads = 1
        t0 = time.perf_counter()
        g = ora.idsoft(coeffs, B)
        ora.dsoft(g)
        t = time.perf_counter() - t0
        steps = 1
        sample = "1 x (IDSOFT + DSOFT) at B=128 through the long-double C restatement (oracle/), one thread"
    return {"value": TRANSFORMS_PER_STEP * steps / t, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": sample, "seconds": t, "steps": steps}


def run_reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle import oracle as orc

    coeffs = orc.coeffs_decaying(B, seed=1, power=1.0, normal_mag=True)
    # each step is one IDSOFT + DSOFT at B = 128 (~0.65 s on 16 cores): at most 100 steps and
    # 10 warm-up steps keep the arm within a few minutes
    steps = max(1, min(args.steps, 100))
    warm = max(0, min(args.warmup, 10))
    cb = cpu_reference_sample(steps, warm, coeffs)
    line = {
        "impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus,
        "steps": cb["steps"], "warmup": warm, "ms_per_step": 1e3 * cb["seconds"] / cb["steps"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(),
        "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference's DWT accumulates in long double (x87); its FFT slot holds the project FFT",
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- GPU workloads

MIXED_BANDS = (32, 48, 64, 96, 128)
SPLIT, NO_GRAPH = 2, 1


def _dev_coeffs(lib, B, seed, kind, power, s):
    import torch
    c = torch.empty(B * (4 * B * B - 1) // 3, dtype=torch.complex128, device="cuda")
    assert lib.pfsoft_cuda_random_coeffs(c.data_ptr(), B, int(seed), kind, float(power), s) == 0
    return c


def _rel(a, b) -> float:
    import torch
    return (torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)).item()


def _timed(fn, steps, warmup):
    """Device milliseconds per call of fn (CUDA events on torch's current stream)."""
    import torch
    for _ in range(max(1, warmup)):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def pinned_copy_floor(nbytes: int, steps: int) -> dict:
    """What the host link gives with no transform: per step `nbytes` host-to-device and `nbytes`
    device-to-host, each one cudaMemcpyAsync on its own stream so the two directions overlap,
    pinned host memory; wall clock over `steps` steps, in the headline's unit (2 transforms a step)."""
    import torch
    hin = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    hout = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    din = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    dout = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()

    def step():
        with torch.cuda.stream(s1):
            din.copy_(hin, non_blocking=True)
        with torch.cuda.stream(s2):
            hout.copy_(dout, non_blocking=True)

    step()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    torch.cuda.synchronize()
    sec = time.perf_counter() - t0
    del hin, hout, din, dout
    return {"value": TRANSFORMS_PER_STEP * steps / sec, "unit": UNIT, "steps": steps,
            "gb_per_s_each_way": nbytes * steps / sec / 1e9,
            "what": f"{nbytes} bytes host-to-device and {nbytes} device-to-host per step, two streams, pinned"}


def dropin_cpp_timing(bandwidth: int, steps: int) -> dict:
    """Transforms/s of the C++ drop-in header's FourierTransforms::IDSOFT + DSOFT on the header's own
    pageable containers (tests/cpp/dropin_timing.cpp, compiled here against the library)."""
    try:
        import shutil
        import pfsoftlib_b200
        pfsoftlib_b200.load()
        libdir = os.path.join(ROOT, "pfsoftlib_b200")
        cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
        with tempfile.TemporaryDirectory() as td:
            exe = os.path.join(td, "dropin_timing")
            subprocess.run([cxx, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                            os.path.join(ROOT, "tests", "cpp", "dropin_timing.cpp"), "-o", exe,
                            "-L", libdir, "-lpfsoft_b200", f"-Wl,-rpath,{libdir}"],
                           check=True, capture_output=True, text=True, timeout=300)
            r = subprocess.run([exe, str(bandwidth), str(steps), "1"], capture_output=True, text=True,
                               timeout=600)
        out = json.loads(r.stdout.strip().splitlines()[-1])
        if r.returncode != 0:
            out["error"] = f"exit {r.returncode}"
        return {"value": out["transforms_per_s"], "unit": UNIT, "steps": steps,
                "max_abs_err": out["max_abs_err"], "ok": r.returncode == 0,
                "api": "pfsoft::FourierTransforms::IDSOFT + DSOFT (include/pfsoft_b200/pfsoft.hpp) on "
                       "grid3D / DSOFTFourierCoefficients storage (pageable new[])"}
    except Exception as exc:   # reported, the headline line still prints
        return {"error": f"{type(exc).__name__}: {exc}"[:300]}


class _Plan:
    """A batch plan over device tensors (pfsoft_batch_*)."""

    def __init__(self, lib, bws, flags, tpc=0):
        import ctypes
        self.lib, self.n = lib, len(bws)
        self.h = ctypes.c_void_p()
        arr = (ctypes.c_int * len(bws))(*bws)
        assert lib.pfsoft_batch_create(arr, len(bws), tpc, flags, ctypes.byref(self.h)) == 0, lib.pfsoft_last_error()

    def _ptrs(self, ts):
        import ctypes
        return (ctypes.c_void_p * self.n)(*[t.data_ptr() for t in ts])

    def idsoft(self, coeffs, grids, s):
        assert self.lib.pfsoft_batch_idsoft(self.h, self._ptrs(coeffs), self._ptrs(grids), s) == 0

    def dsoft(self, grids, coeffs, s):
        assert self.lib.pfsoft_batch_dsoft(self.h, self._ptrs(grids), self._ptrs(coeffs), s) == 0

    def status(self):
        return self.lib.pfsoft_batch_status(self.h)

    def close(self):
        if self.h:
            self.lib.pfsoft_batch_destroy(self.h)
            self.h = None


def mixed_section(lib, steps: int, warmup: int, tune: bool = False) -> dict:
    """256 independent transforms, bandwidths uniform over {32,48,64,96,128} (PCG64 seed 2),
    |f| = (1+l)^-1.5 with uniform phase (device generator, seed 2000 + i). One step = IDSOFT then
    DSOFT of every transform, for: the plain loop over the single-transform entry points (FP64),
    the FP64 batch plan (one fused DWT launch per direction, CUDA graph), the split-precision batch
    plan (one tcgen05 launch per direction), and the split-precision server, saturated (all 512
    requests submitted at once). Errors: split against FP64 for every transform, and the first
    B = 32 transform's split results against the long-double oracle."""
    import numpy as np
    import torch

    from oracle import oracle as orc
    from pfsoftlib_b200 import autotune
    from pfsoftlib_b200.serving import TransformServer

    s = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(2)
    bws = [int(b) for b in rng.choice(MIXED_BANDS, size=256)]
    coeffs = [_dev_coeffs(lib, Bi, 2000 + i, 2, 1.5, s) for i, Bi in enumerate(bws)]
    grids = [torch.empty((2 * Bi,) * 3, dtype=torch.complex128, device="cuda") for Bi in bws]
    back = [torch.empty_like(c) for c in coeffs]
    ws = torch.empty(lib.pfsoft_workspace_bytes(max(bws)) // 8, dtype=torch.float64, device="cuda")

    def plain():
        for i, Bi in enumerate(bws):
            assert lib.pfsoft_cuda_idsoft(coeffs[i].data_ptr(), Bi, grids[i].data_ptr(), ws.data_ptr(), ws.numel() * 8, s) == 0
            assert lib.pfsoft_cuda_dsoft(grids[i].data_ptr(), Bi, back[i].data_ptr(), ws.data_ptr(), ws.numel() * 8, s) == 0

    ms_plain = _timed(plain, steps, warmup)
    g64 = [g.clone() for g in grids]
    c64 = [b.clone() for b in back]
    del ws
    tpc, tune_ms = 0, None
    if tune:
        tpc, tune_ms = autotune.tune_batch(lib, bws, coeffs, grids, back, use_cache=False)
    p64 = _Plan(lib, bws, 0, tpc)
    ms_batch = _timed(lambda: (p64.idsoft(coeffs, grids, s), p64.dsoft(grids, back, s)), steps, warmup)
    batch_vs = max(_rel(back[i], c64[i]) for i in range(len(bws)))
    p64.close()
    psp = _Plan(lib, bws, SPLIT)
    ms_split = _timed(lambda: (psp.idsoft(coeffs, grids, s), psp.dsoft(grids, back, s)), steps, warmup)
    split_status = psp.status()
    psp.close()
    torch.cuda.synchronize()
    split_grid_vs = max(_rel(grids[i], g64[i]) for i in range(len(bws)))
    split_coef_vs = max(_rel(back[i], c64[i]) for i in range(len(bws)))
    split_rt = max(_rel(back[i], coeffs[i]) for i in range(len(bws)))
    # the autotuned plan: per bandwidth, the FFT stage fused or not and the DWT split or FP64
    tuned = autotune.tune_plan(lib, bws, coeffs, grids, back, use_cache=False)
    ptu = _Plan(lib, bws, SPLIT)
    ms_tuned = _timed(lambda: (ptu.idsoft(coeffs, grids, s), ptu.dsoft(grids, back, s)), steps, warmup)
    ptu.close()
    torch.cuda.synchronize()
    tuned_vs = max(_rel(back[i], c64[i]) for i in range(len(bws)))
    lib.pfsoft_tune_fft_fused(0, 0)        # back to the defaults for what follows
    lib.pfsoft_tune_split_bandwidth(0, 1)
    # the oracle on the first B = 32 transform (long double, all on the host)
    i32 = bws.index(32)
    ora = orc.Oracle()
    c_h = coeffs[i32].cpu().numpy()
    g_h = grids[i32].cpu().numpy()
    oracle_grid = orc.rel_l2(g_h, ora.idsoft(c_h, 32))
    oracle_coef = orc.rel_l2(back[i32].cpu().numpy(), ora.dsoft(g_h))
    # the split-precision server, saturated: all 512 requests at once, fresh outputs
    out_g = [torch.empty_like(g) for g in grids]
    out_c = [torch.empty_like(c) for c in coeffs]
    jobs = [(1, i) for i in range(len(bws))] + [(0, i) for i in range(len(bws))]
    order = np.random.default_rng(3).permutation(len(jobs))
    torch.cuda.synchronize()
    with TransformServer(budget_bytes=48 << 30, max_batch=16, streams=4, split=True) as srv:
        def submit(j):
            d, i = jobs[j]
            return srv.idsoft(coeffs[i], out_g[i]) if d == 1 else srv.dsoft(g64[i], out_c[i])
        for r in [submit(j) for j in order[:64]]:    # warm-up
            r.wait(300)
        srv.reset_stats()
        for r in [submit(j) for j in order]:
            r.wait(300)
        sat = srv.stats()
    served_vs = max(max(_rel(out_c[i], c64[i]), _rel(out_g[i], g64[i])) for i in range(len(bws)))
    n = 2 * len(bws)
    tps = lambda ms: n / (ms / 1e3)
    return {
        "workload": "256 transforms, B uniform over {32,48,64,96,128} (seed 2), |f|=(1+l)^-1.5; "
                    "one step = IDSOFT + DSOFT of all",
        "bandwidth_counts": {str(b): bws.count(b) for b in MIXED_BANDS},
        "plain_loop": {"value": tps(ms_plain), "ms_per_step": ms_plain},
        "fp64_batch": {"value": tps(ms_batch), "ms_per_step": ms_batch, "speedup_vs_plain_loop": ms_plain / ms_batch,
                       "rel_l2_vs_plain_max": batch_vs, "transforms_per_cta": tpc or "default", "autotune_ms": tune_ms},
        "split_batch": {"value": tps(ms_split), "ms_per_step": ms_split, "speedup_vs_plain_loop": ms_plain / ms_split,
                        "status": split_status},
        "tuned_batch": {"value": tps(ms_tuned), "ms_per_step": ms_tuned, "speedup_vs_plain_loop": ms_plain / ms_tuned,
                        "rel_l2_vs_fp64_max": tuned_vs, "autotune": tuned},
        "split_served": {"value": sat["transforms_per_s"], "speedup_vs_plain_loop": sat["transforms_per_s"] / tps(ms_plain),
                         "p50_ms": sat["p50_ms"], "p99_ms": sat["p99_ms"], "mean_batch": sat["mean_batch"],
                         "max_concurrent_batches": sat["max_concurrent_batches"],
                         "timing": "host clock, first submit -> last completion, 512 requests submitted at once"},
        "accuracy": {"split_grid_rel_l2_vs_fp64_max": split_grid_vs, "split_coef_rel_l2_vs_fp64_max": split_coef_vs,
                     "split_round_trip_rel_l2_max": split_rt, "served_rel_l2_vs_fp64_max": served_vs,
                     "split_vs_oracle_B32": {"grid_rel_l2": oracle_grid, "coef_rel_l2": oracle_coef}},
        "steps": steps, "warmup": max(1, warmup),
    }


def run_mixed(args):
    import torch

    import pfsoftlib_b200

    lib = pfsoftlib_b200.load()
    torch.cuda.set_device(0)
    steps = max(1, min(args.steps, 5))
    clocks = ClockSampler(0)
    clocks.start()
    sec = mixed_section(lib, steps, args.warmup, tune=True)
    clk = clocks.stop()
    line = {
        "metric": "DSOFT+iDSOFT transforms/s, 256 transforms of uneven bandwidth (split-precision batch)",
        "value": sec["split_batch"]["value"], "unit": "transforms/s", "n_gpus": 1, "steps": steps,
        "warmup": max(1, args.warmup), "ms_per_step": sec["split_batch"]["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 data; s8 digit products, exact s32 sums, f64 combine",
        "data": "synthetic (device generator)",
        "config": {"workload": sec["workload"], "l2": "working set ~45 GB, far above L2"},
        "mixed": sec, "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def b256_section(lib, groups: int = 1, check_reference: bool = True) -> dict:
    """Transforms at B = 256 (|f| = (1+l)^-2 with uniform phase, device generator, seed 3 + i) in
    groups of 8 through one batch plan: IDSOFT (8 grids of 2.15 GB) then DSOFT of those grids, FP64
    plan (per-transform FP64 DWT above B = 128) against the split-precision plan (one tcgen05 launch
    per direction). Errors: split against FP64, the split round trip, and the last group's first
    split DSOFT against the compiled reference's CPU DSOFT of the same grid (all host threads)."""
    import torch

    from oracle import oracle as orc

    s = torch.cuda.current_stream().cuda_stream
    Bb, G = 256, 8
    coeffs = [torch.empty(Bb * (4 * Bb * Bb - 1) // 3, dtype=torch.complex128, device="cuda") for _ in range(G)]
    grids = [torch.empty((2 * Bb,) * 3, dtype=torch.complex128, device="cuda") for _ in range(G)]
    back = [torch.empty_like(c) for c in coeffs]
    ms = {}
    worst = {"split_grid_rel_l2_vs_fp64_max": 0.0, "split_coef_rel_l2_vs_fp64_max": 0.0, "split_round_trip_rel_l2_max": 0.0,
             "fp64_round_trip_rel_l2_max": 0.0}
    plans = {"fp64": _Plan(lib, [Bb] * G, 0), "split": _Plan(lib, [Bb] * G, SPLIT)}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    status = 0
    for g0 in range(0, G * (groups + 1), G):   # the first group is the warm-up
        for i in range(G):
            assert lib.pfsoft_cuda_random_coeffs(coeffs[i].data_ptr(), Bb, 3 + g0 + i, 2, 2.0, s) == 0
        res = {}
        for name, p in plans.items():
            torch.cuda.synchronize()
            e0.record()
            p.idsoft(coeffs, grids, s)
            p.dsoft(grids, back, s)
            e1.record()
            torch.cuda.synchronize()
            if g0 > 0:
                ms[name] = ms.get(name, 0.0) + e0.elapsed_time(e1)
            if name == "fp64":
                res["g"] = [g.clone() for g in grids]
                res["c"] = [b.clone() for b in back]
                worst["fp64_round_trip_rel_l2_max"] = max(worst["fp64_round_trip_rel_l2_max"],
                                                          max(_rel(back[i], coeffs[i]) for i in range(G)))
        status |= plans["split"].status()
        for i in range(G):
            worst["split_grid_rel_l2_vs_fp64_max"] = max(worst["split_grid_rel_l2_vs_fp64_max"], _rel(grids[i], res["g"][i]))
            worst["split_coef_rel_l2_vs_fp64_max"] = max(worst["split_coef_rel_l2_vs_fp64_max"], _rel(back[i], res["c"][i]))
            worst["split_round_trip_rel_l2_max"] = max(worst["split_round_trip_rel_l2_max"], _rel(back[i], coeffs[i]))
        del res
    for p in plans.values():
        p.close()
    acc = dict(worst)
    if check_reference and orc.Reference.available():
        ref = orc.Reference()
        g_h = grids[0].cpu().numpy()
        t0 = time.perf_counter()
        f_ref = ref.dsoft(g_h, ref.max_threads())
        acc["split_vs_reference_dsoft"] = {"rel_l2": orc.rel_l2(back[0].cpu().numpy(), f_ref),
                                           "max_abs": orc.max_abs(back[0].cpu().numpy(), f_ref),
                                           "reference_s": time.perf_counter() - t0, "threads": ref.max_threads()}
        del g_h, f_ref
    n = 2 * G * groups
    return {
        "workload": f"{G * groups} transforms at B=256 (seed 3+i, |f|=(1+l)^-2) in groups of 8 through one batch "
                    f"plan; IDSOFT + DSOFT of each",
        "fp64": {"value": n / (ms["fp64"] / 1e3), "ms": ms["fp64"]},
        "split": {"value": n / (ms["split"] / 1e3), "ms": ms["split"], "speedup_vs_fp64": ms["fp64"] / ms["split"],
                  "status": status},
        "accuracy": acc,
    }


def run_b256(args):
    import torch

    import pfsoftlib_b200

    lib = pfsoftlib_b200.load()
    torch.cuda.set_device(0)
    clocks = ClockSampler(0)
    clocks.start()
    sec = b256_section(lib, groups=8)
    clk = clocks.stop()
    line = {
        "metric": "DSOFT+iDSOFT transforms/s, 64 transforms at B=256 (split precision)", "value": sec["split"]["value"],
        "unit": "transforms/s", "n_gpus": 1, "steps": 1, "warmup": 1, "ms_per_step": sec["split"]["ms"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 data; s8 digit products, exact s32 sums, f64 combine", "data": "synthetic (device generator)",
        "config": {"workload": sec["workload"], "grid": "512^3 complex128 (2.15 GB) each", "l2": "far above L2"},
        "b256": sec, "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def _log_uniform_bandwidths(rng, n, lo=16, hi=256):
    """Integers lo..hi with P(B) proportional to log((B+1)/B) (a continuous log-uniform variate on
    [lo, hi+1) rounded down)."""
    import numpy as np
    return np.minimum(hi, np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi + 1), size=n)))).astype(int)


def serving_section(lib, rates, seconds: float, budget_gb: float, seed: int = 4) -> dict:
    """Poisson arrivals at each offered rate for `seconds`: requests 50/50 DSOFT / iDSOFT, bandwidth
    log-uniform over the integers 16..256 (PCG64 `seed`). Inputs stay on the device: one seeded
    B = 256 coefficient set (|f| = (1+l)^-1.5, uniform phase) and its grid; a request at bandwidth B
    reads the leading B(4B^2-1)/3 coefficients (a complete coefficient set of bandwidth B, the packed
    layout being degree-major) or the leading (2B)^3 grid values. Outputs go to pools of buffers,
    a request waiting for its buffer's previous user. Two forms, one after the other:
      split_served  TransformServer(split=True): batches of one direction and any bandwidths,
                    split-precision DWT in one launch per batch, up to 4 batches in flight;
                    latency from the scheduled arrival to the completion seen by polling (a
                    request whose output buffer is still in use waits, and that wait counts);
                    server_p50/p99 are the server's own figures from submission;
      plain         the single-transform FP64 entry points, one request at a time in arrival order
                    on one stream (latency from arrival to the completion event on the device).
    Tables of every bandwidth are built in a warm-up pass first (the server builds a bandwidth's
    tables at submission, outside the latency it reports)."""
    import numpy as np
    import torch

    from pfsoftlib_b200.serving import TransformServer

    s = torch.cuda.current_stream().cuda_stream
    BM = 256
    coef_in = _dev_coeffs(lib, BM, 4000, 2, 1.5, s)
    grid_in = torch.empty((2 * BM,) * 3, dtype=torch.complex128, device="cuda")
    assert lib.pfsoft_cuda_idsoft(coef_in.data_ptr(), BM, grid_in.data_ptr(), None, 0, s) == 0
    pool_g, pool_c = 12, 64
    out_g = [torch.empty((2 * BM) ** 3, dtype=torch.complex128, device="cuda") for _ in range(pool_g)]
    out_c = [torch.empty_like(coef_in) for _ in range(pool_c)]
    ws = torch.empty(lib.pfsoft_workspace_bytes(BM) // 8, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ncoef = lambda b: b * (4 * b * b - 1) // 3

    def views(d, b, k):
        if d == 0:   # DSOFT: grid in, coefficients out
            return grid_in.view(-1)[: (2 * b) ** 3], out_c[k % pool_c][: ncoef(b)]
        return coef_in[: ncoef(b)], out_g[k % pool_g][: (2 * b) ** 3]

    rng = np.random.default_rng(seed)
    plan = []
    for rate in rates:
        n = max(20, int(rate * seconds))
        plan.append((rate, _log_uniform_bandwidths(rng, n), rng.integers(0, 2, size=n), rng.exponential(1.0 / rate, size=n)))

    free, _ = torch.cuda.mem_get_info()
    budget = int(min(budget_gb * (1 << 30), free - (6 << 30)))
    out = {"budget_bytes": budget, "requests_per_rate": [len(p[1]) for p in plan], "split_served": [], "plain": []}
    with TransformServer(budget_bytes=budget, max_batch=16, streams=4, split=True) as srv:
        # warm-up: every bandwidth once per direction (tables, first launches); its statistics are
        # the cold-start figures
        t0 = time.perf_counter()
        warm = []
        for b in range(16, BM + 1):
            for d in (0, 1):
                i, o = views(d, b, b)
                warm.append(srv.submit(d, b, i, o))
        for r in warm:
            r.wait(600)
        st = srv.stats()
        out["cold_start"] = {"requests": len(warm), "seconds": time.perf_counter() - t0, "p50_ms": st["p50_ms"],
                             "p99_ms": st["p99_ms"], "note": "all 482 submitted at once with no tables built"}
        for rate, Bs, dirs, gaps in plan:
            srv.reset_stats()
            last = {}
            t0 = time.perf_counter()
            due = t0 + np.cumsum(gaps)
            pending = []   # (request, scheduled arrival) not yet seen complete
            lat = []       # completion - scheduled arrival, ms (host clock, polled)
            first_arrival, last_done = due[0], due[0]

            def poll():
                nonlocal last_done
                now = time.perf_counter()
                keep = []
                for r, t_arr in pending:
                    if r.done():
                        lat.append(1e3 * (now - t_arr))
                        last_done = now
                    else:
                        keep.append((r, t_arr))
                pending[:] = keep

            for k in range(len(Bs)):
                b, d = int(Bs[k]), int(dirs[k])
                slot = (d, k % (pool_c if d == 0 else pool_g))
                # the output buffer's previous request must be done; the wait counts in this
                # request's latency (measured from its scheduled arrival)
                while slot in last and not last[slot].done():
                    poll()
                while time.perf_counter() < due[k]:
                    poll()
                i, o = views(d, b, k)
                r = srv.submit(d, b, i, o)
                last[slot] = r
                pending.append((r, due[k]))
            while pending:
                poll()
            st = srv.stats()
            lat_a = np.array(lat)
            out["split_served"].append({"offered_per_s": rate, "transforms_per_s": len(Bs) / (last_done - first_arrival),
                                        "p50_ms": float(np.percentile(lat_a, 50, method="higher")),
                                        "p99_ms": float(np.percentile(lat_a, 99, method="higher")),
                                        "mean_ms": float(lat_a.mean()), "max_ms": float(lat_a.max()),
                                        "server_p50_ms": st["p50_ms"], "server_p99_ms": st["p99_ms"],
                                        "mean_batch": st["mean_batch"],
                                        "max_concurrent_batches": st["max_concurrent_batches"],
                                        "peak_bytes": st["peak_bytes"], "failed": st["failed"]})
    # the plain per-request FP64 path: one stream, arrival order
    stream = torch.cuda.current_stream()
    for rate, Bs, dirs, gaps in plan:
        n = len(Bs)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(n)]
        start = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        start.record(stream)
        arrive = t0 + np.cumsum(gaps)
        for k in range(n):
            b, d = int(Bs[k]), int(dirs[k])
            while time.perf_counter() < arrive[k]:
                pass
            i, o = views(d, b, k)
            f = lib.pfsoft_cuda_dsoft if d == 0 else lib.pfsoft_cuda_idsoft
            assert f(i.data_ptr(), b, o.data_ptr(), ws.data_ptr(), ws.numel() * 8, s) == 0
            ev[k].record(stream)
        torch.cuda.synchronize()
        done_ms = np.array([start.elapsed_time(e) for e in ev])
        lat = done_ms - 1e3 * (arrive - t0)
        span = done_ms[-1] - 1e3 * (arrive[0] - t0)
        out["plain"].append({"offered_per_s": rate, "transforms_per_s": n / (span / 1e3),
                             "p50_ms": float(np.percentile(lat, 50, method="higher")),
                             "p99_ms": float(np.percentile(lat, 99, method="higher")),
                             "mean_ms": float(lat.mean()), "max_ms": float(lat.max())})
    return out


def run_serve_sweep(args):
    import torch

    import pfsoftlib_b200

    lib = pfsoftlib_b200.load()
    torch.cuda.set_device(0)
    rates = [float(r) for r in args.rates.split(",") if r]
    clocks = ClockSampler(0)
    clocks.start()
    sec = serving_section(lib, rates, args.seconds, args.budget_gb)
    clk = clocks.stop()
    best = max(x["transforms_per_s"] for x in sec["split_served"])
    line = {
        "metric": "served DSOFT/iDSOFT transforms/s under Poisson arrivals, split precision (best over the sweep)",
        "value": best, "unit": "transforms/s", "n_gpus": 1, "steps": len(rates), "warmup": 1, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 data; s8 digit products, exact s32 sums, f64 combine",
        "data": "synthetic (device generator)",
        "config": {"workload": "requests 50/50 DSOFT/iDSOFT, B log-uniform over the integers 16..256 (seed 4), "
                               "Poisson arrivals", "rates": rates, "seconds_per_rate": args.seconds,
                   "max_batch": 16, "streams": 4},
        "serving": sec, "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def run_shard(args):
    """One transform at B = 256 sharded over the N ranks (strong scaling): rank r holds layers
    [first, first + count) of the 512^3 grid and a balanced share of the order classes; an NCCL
    all-to-all moves the FFT bins between the stages (pfsoftlib_b200.shard.ShardedTransform).
    One step = iDSOFT of the coefficients to the ranks' slabs, then DSOFT of the slabs back, the
    coefficients distributed by order class between the two (each rank holds its classes). The
    round trip is checked once with the coefficients gathered (all-reduce) before the timing.
    Timing: barrier + synchronize on both sides of the K steps, max over ranks."""
    import datetime
    import socket

    import torch
    import torch.distributed as dist

    import pfsoftlib_b200
    from pfsoftlib_b200.shard import ShardedTransform

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    lib = pfsoftlib_b200.load()
    if "MASTER_ADDR" in os.environ:
        dist.init_process_group("nccl", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    else:
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            port = sk.getsockname()[1]
        dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                                timeout=datetime.timedelta(seconds=120))
    B = 256
    s = torch.cuda.current_stream().cuda_stream
    coeffs = torch.empty(B * (4 * B * B - 1) // 3, dtype=torch.complex128, device="cuda")
    assert lib.pfsoft_cuda_random_coeffs(coeffs.data_ptr(), B, 1, 1, 1.0, s) == 0
    st = ShardedTransform(B)
    first, count = st.layers
    slab = torch.empty((count, 2 * B, 2 * B), dtype=torch.complex128, device="cuda")
    back = torch.empty_like(coeffs)

    part = torch.empty_like(coeffs)

    def step():
        # coefficients stay distributed by order class between the directions (gather=False)
        st.idsoft(part, out=slab)
        st.dsoft(slab, out=part, gather=False)

    st.idsoft(coeffs, out=slab)
    st.dsoft(slab, out=back)   # gathered once: the round-trip check
    torch.cuda.synchronize()
    err = (torch.linalg.vector_norm(back - coeffs) / torch.linalg.vector_norm(coeffs)).item()
    part.copy_(back)
    for _ in range(max(args.warmup, 1)):
        step()
    steps = max(1, min(args.steps, 20))
    clocks = ClockSampler(local) if rank == 0 else None
    if clocks:
        clocks.start()
    dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    dist.barrier()
    ms = torch.tensor([e0.elapsed_time(e1) / steps], dtype=torch.float64, device="cuda")
    dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    clk = clocks.stop() if clocks else None
    if rank == 0:
        line = {
            "metric": "sharded DSOFT+iDSOFT transforms/s of one B=256 transform", "value": 2 / (ms.item() / 1e3),
            "unit": "transforms/s", "n_gpus": world, "steps": steps, "warmup": max(args.warmup, 1),
            "ms_per_step": ms.item(), "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (device generator, seed 1)",
            "config": {"workload": "one transform at B=256 sharded over the ranks: layer slabs for the FFT, "
                                   "order classes for the DWT, NCCL all-to-all between; coefficients "
                                   "distributed by order class", "B": B, "parallelism": f"shard{world}",
                       "l2": "inputs far above L2 (512^3 complex128 grid: 2.15 GB)"},
            "accuracy": {"round_trip_rel_l2": err},
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    del st
    dist.destroy_process_group()



def main():
    args = parse()
    if args.impl == "reference":
        run_reference_arm(args)
        return
    if args.workload == "mixed":
        run_mixed(args)
        return
    if args.workload == "serve":
        run_serve_sweep(args)
        return
    if args.workload == "b256":
        run_b256(args)
        return
    if args.workload == "shard":
        run_shard(args)
        return

    import numpy as np
    import torch

    import pfsoftlib_b200
    from oracle import oracle as orc

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    lib = pfsoftlib_b200.load()
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream

    coeffs_h = orc.coeffs_decaying(B, seed=1, power=1.0, normal_mag=True)
    c = torch.from_numpy(coeffs_h).cuda()
    f = torch.empty_like(c)
    g = torch.empty((N, N, N), dtype=torch.complex128, device="cuda")
    ws = torch.empty(lib.pfsoft_workspace_bytes(B) // 8, dtype=torch.float64, device="cuda")
    wp, wb = ws.data_ptr(), ws.numel() * 8

    def step():
        rc = lib.pfsoft_cuda_idsoft(c.data_ptr(), B, g.data_ptr(), wp, wb, sp)
        rc |= lib.pfsoft_cuda_dsoft(g.data_ptr(), B, f.data_ptr(), wp, wb, sp)
        if rc:
            raise RuntimeError(lib.pfsoft_last_error().decode())

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(max(3, args.warmup)):
        step()
    barrier()

    # ---- timed region (device time) with per-stage events. The clock sampler runs from
    # here; extra untimed steps keep the GPU loaded for >= 0.6 s before the timed region so
    # that the 200 ms sampler sees the load even when the timed region itself is short.
    clocks = ClockSampler(local)
    clocks.start()
    t_load = time.perf_counter()
    while time.perf_counter() - t_load < 0.6:
        step()
        torch.cuda.synchronize()
    lib.pfsoft_profile_read(None, None, 0)
    lib.pfsoft_profile_enable(1)
    launches0 = lib.pfsoft_launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    barrier()
    launches = lib.pfsoft_launch_count() - launches0
    lib.pfsoft_profile_enable(0)
    nst = 16
    st_ms = np.zeros(nst)
    st_cnt = np.zeros(nst, dtype=np.int64)
    nstages = lib.pfsoft_profile_read(st_ms.ctypes.data, st_cnt.ctypes.data, nst)
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    if dist is not None:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = TRANSFORMS_PER_STEP * args.steps * world / (ms / 1e3)

    # ---- accuracy of the timed results (round trip at B = 128)
    f_h = f.cpu().numpy()
    acc = {"round_trip_rel_l2": orc.rel_l2(f_h, coeffs_h), "round_trip_max_abs": orc.max_abs(f_h, coeffs_h),
           "round_trip_rel_l2_max_bound": 1e-13}

    # ---- per-stage roofline
    peaks = measured_peaks()
    hbm = peaks["hbm_gbs"]
    stages = {}
    for i in range(nstages):
        name = lib.pfsoft_profile_stage_name(i).decode()
        if st_cnt[i] == 0:
            continue
        per = st_ms[i] / st_cnt[i]
        if name.startswith("fft"):
            achieved = FFT_PASS_BYTES / (per / 1e3) / 1e9
            stages[name] = {"bound": "hbm", "ms_per_launch": per, "launches": int(st_cnt[i]),
                            "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm}
        elif name.startswith("dwt"):
            achieved = DWT_FLOPS / (per / 1e3) / 1e12
            stages[name] = {"bound": "tensor", "ms_per_launch": per, "launches": int(st_cnt[i]),
                            "achieved": achieved, "peak": FP64_PEAK_TFLOPS, "unit": "TFLOP/s",
                            "frac": achieved / FP64_PEAK_TFLOPS}
        else:
            stages[name] = {"ms_per_launch": per, "launches": int(st_cnt[i])}
    dominant = max((k for k in stages if "frac" in stages[k]), key=lambda k: stages[k]["ms_per_launch"] * stages[k]["launches"])
    d = stages[dominant]
    # DRAM bytes per launch (read + write) of these kernels at B = 128, from one ncu capture of the
    # same launches (dram__bytes_read.sum + dram__bytes_write.sum)
    traffic = {"dwt_forward": 277.00e6 + 39.89e6, "dwt_inverse": 55.02e6 + 206.65e6,
               "fft_forward_gamma": 268.51e6 + 217.40e6, "fft_forward_alpha": 268.50e6 + 206.99e6,
               "fft_inverse_alpha": 268.51e6 + 206.85e6, "fft_inverse_gamma": 268.51e6 + 217.70e6}
    roofline = {"kernel": dominant, "bound": d["bound"], "achieved": d["achieved"], "peak": d["peak"],
                "unit": d["unit"], "frac": d["frac"], "traffic": traffic.get(dominant),
                "peak_source": ("measured FP64 MMA peak (own micro-benchmark; MEASURED_PEAKS.json has no FP64 entry)"
                                if d["bound"] == "tensor" else peaks["source"])}

    # ---- end to end through the host-facing C ABI (pinned host buffers)
    ch = torch.from_numpy(coeffs_h).pin_memory()
    gh = torch.empty((N, N, N), dtype=torch.complex128).pin_memory()
    fh = torch.empty_like(ch).pin_memory()
    e2e_steps = max(2, min(args.steps, 10))

    def host_step():
        rc = lib.pfsoft_idsoft_host(ch.data_ptr(), B, gh.data_ptr())
        rc |= lib.pfsoft_dsoft_host(gh.data_ptr(), B, fh.data_ptr())
        if rc:
            raise RuntimeError(lib.pfsoft_last_error().decode())

    host_step()
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        host_step()
    t_seq = time.perf_counter() - t0
    # concurrent: one host thread runs the iDSOFTs, another the DSOFTs (of a grid already on the
    # host), so that each step's device-to-host grid copy overlaps the other call's host-to-device
    # grid copy (the PCIe link is full duplex; each call has its own staging buffers and stream)
    import threading

    gin = gh.clone().pin_memory()
    gout = torch.empty_like(gh).pin_memory()
    fout = torch.empty_like(fh).pin_memory()
    errs = []
    start = threading.Barrier(2)

    def worker(fn):
        try:
            start.wait()   # both threads leave together: no thread-start skew inside the timed span
            for _ in range(e2e_steps):
                if fn():
                    raise RuntimeError(lib.pfsoft_last_error().decode())
        except Exception as exc:   # surfaced below
            errs.append(exc)

    inv = lambda: lib.pfsoft_idsoft_host(ch.data_ptr(), B, gout.data_ptr())
    fwd = lambda: lib.pfsoft_dsoft_host(gin.data_ptr(), B, fout.data_ptr())
    inv()
    fwd()
    barrier()
    t0 = time.perf_counter()
    th = [threading.Thread(target=worker, args=(f,)) for f in (inv, fwd)]
    for x in th:
        x.start()
    for x in th:
        x.join()
    t_e2e = time.perf_counter() - t0
    if errs:
        raise errs[0]
    if dist is not None:
        t = torch.tensor([t_e2e, t_seq], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_e2e, t_seq = float(t[0].item()), float(t[1].item())
    e2e = {"value": TRANSFORMS_PER_STEP * e2e_steps * world / t_e2e, "unit": UNIT,
           "h2d_bytes_per_step": COEF_BYTES + GRID_BYTES, "d2h_bytes_per_step": GRID_BYTES + COEF_BYTES,
           "api": "pfsoft_idsoft_host and pfsoft_dsoft_host (include/pfsoft_b200.h) from two host threads, one "
                  "call of each in flight, pinned host buffers",
           "steps": e2e_steps}
    e2e_sequential = {"value": TRANSFORMS_PER_STEP * e2e_steps * world / t_seq, "unit": UNIT, "steps": e2e_steps,
                      "api": "pfsoft_idsoft_host then pfsoft_dsoft_host of its grid, one thread, pinned host buffers"}
    fout_check = orc.rel_l2(fout.numpy(), coeffs_h)
    del gin, gout, fout
    # the same on pageable host memory (what the C++ drop-in header passes: grid3D's new[] storage)
    chp = coeffs_h.copy()
    ghp = np.empty((N, N, N), dtype=np.complex128)
    fhp = np.empty_like(chp)

    def host_step_pageable():
        rc = lib.pfsoft_idsoft_host(chp.ctypes.data, B, ghp.ctypes.data)
        rc |= lib.pfsoft_dsoft_host(ghp.ctypes.data, B, fhp.ctypes.data)
        if rc:
            raise RuntimeError(lib.pfsoft_last_error().decode())

    host_step_pageable()
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        host_step_pageable()
    t_pg = time.perf_counter() - t0
    acc["host_round_trip_rel_l2"] = fout_check
    e2e_pageable = {"value": TRANSFORMS_PER_STEP * e2e_steps / t_pg, "unit": UNIT, "steps": e2e_steps,
                    "h2d_bytes_per_step": COEF_BYTES + GRID_BYTES, "d2h_bytes_per_step": GRID_BYTES + COEF_BYTES,
                    "api": "pfsoft_idsoft_host + pfsoft_dsoft_host on pageable numpy buffers"}
    del chp, ghp, fhp
    # the copy floor of e2e: the same bytes moved by plain pinned copies, host-to-device and
    # device-to-host on two streams at once (what the link gives with no transform at all)
    copy_floor = pinned_copy_floor(COEF_BYTES + GRID_BYTES, e2e_steps)
    e2e["copy_floor"] = copy_floor
    e2e["frac_of_copy_floor"] = e2e["value"] / copy_floor["value"]
    # the C++ drop-in itself: FourierTransforms::IDSOFT / DSOFT of pfsoft_b200/pfsoft.hpp on its
    # own containers (pageable new[] storage), a compiled program timed by its own clock
    e2e_dropin = dropin_cpp_timing(B, e2e_steps) if rank == 0 else None

    # ---- CPU baseline (rank 0, N = 1 only)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_reference_sample(1, 0, coeffs_h)
        cpu = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
        # parity of the GPU DSOFT against the reference DSOFT of the same grid
        if cb["kind"] == "reference":
            ref = orc.Reference()
            g_h = g.cpu().numpy()
            f_ref = ref.dsoft(g_h, ref.max_threads())
            acc["vs_reference_dsoft_rel_l2"] = orc.rel_l2(f_h, f_ref)
            acc["vs_reference_dsoft_max_abs"] = orc.max_abs(f_h, f_ref)

    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(),
        "e2e": e2e, "e2e_sequential": e2e_sequential, "e2e_pageable": e2e_pageable, "e2e_dropin_cpp": e2e_dropin,
        "gpu_launches": int(launches), "roofline": roofline,
        "stages": stages, "cpu_baseline": cpu, "accuracy": acc, "clocks": clk,
        "parallelism": f"replicas x{world} (independent transforms per GPU, no collective)",
    }
    # the other workloads, compact (N = 1 only): each section catches its own failure so that the
    # headline line is still printed
    if world == 1 and not args.no_extras:
        del c, f, g, ws, ch, gh, fh
        torch.cuda.empty_cache()
        extras_clock = ClockSampler(local)
        extras_clock.start()
        t_x = time.perf_counter()
        for key, fn in (("mixed", lambda: mixed_section(lib, 2, 1)),
                        ("b256", lambda: b256_section(lib, groups=1)),
                        ("serving", lambda: serving_section(lib, [100.0, 500.0, 1500.0], 1.5, 160.0))):
            t_s = time.perf_counter()
            try:
                line[key] = fn()
            except Exception as exc:   # reported, not hidden: the key carries the failure
                line[key] = {"error": f"{type(exc).__name__}: {exc}"}
            line[key]["section_s"] = time.perf_counter() - t_s
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
        line["extras_clocks"] = extras_clock.stop()
        line["extras_s"] = time.perf_counter() - t_x
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
