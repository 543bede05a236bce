"""Benchmark: DSOFT + iDSOFT transforms/s at bandwidth B = 128 (one B200 per rank).

One step = one iDSOFT (2,796,160 coefficients -> 256^3 complex128 grid) followed by one DSOFT
of that grid (the single-transform workload at B = 128), i.e. 2 transforms per step. Inputs are
seeded synthetic coefficients: uniform phase, magnitude (1+l)^-1 |N(0,1)|, PCG64 seed 1.

  value     transforms/s with everything resident in HBM, device time (CUDA events) over the
            K timed steps, max over ranks; every buffer (268 MB grid) exceeds the 126 MB L2.
  e2e       the same metric through the host-facing C ABI (pfsoft_idsoft_host /
            pfsoft_dsoft_host) from pinned host memory, copies inside the timed region.
  roofline  the dominant stage, timed with CUDA events per stage inside the timed region.
  cpu_baseline  the reference's own CPU DSOFT/IDSOFT (compiled from its sources with a project
            FFT in FFTW's place) on a bounded sample, rank 0 at N = 1 only.

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


def workload_config(l2_note: str) -> dict:
    return {
        "workload": "single transform at B=128: iDSOFT of 2,796,160 complex128 coefficients to a "
                    "256^3 complex128 grid, then DSOFT of that grid",
        "B": B,
        "grid": "256x256x256 complex128 (268 MB)",
        "coefficients": COEF_COUNT,
        "transforms_per_step": TRANSFORMS_PER_STEP,
        "inputs": "seeded synthetic (PCG64 seed 1): uniform phase, |f| = (1+l)^-1 |N(0,1)|",
        "l2": l2_note,
    }


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
                    help="serve: arrival window per rate (5.2 s over the default rates: ~20,000 requests)")
    ap.add_argument("--budget-gb", type=float, default=160.0, help="serve: HBM budget of the server's arena")
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
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        g = ora.idsoft(coeffs, B)
        ora.dsoft(g)
        t = time.perf_counter() - t0
        steps = 1
        sample = "1 x (IDSOFT + DSOFT) at B=128 through the long-double C restatement (oracle/)"
    return {"value": TRANSFORMS_PER_STEP * steps / t, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": sample, "seconds": t}


def run_reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle import oracle as orc

    coeffs = orc.coeffs_decaying(B, seed=1, power=1.0, normal_mag=True)
    steps = max(1, min(args.steps, 20))
    warm = 1 if args.warmup > 0 else 0
    cb = cpu_reference_sample(steps, warm, coeffs)
    line = {
        "impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "warmup": warm, "ms_per_step": 1e3 * cb["seconds"] / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 (long double DWT accumulation)", "data": "synthetic",
        "config": workload_config("host memory"),
        "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- GPU arm

MIXED_BANDS = (32, 48, 64, 96, 128)


def run_served(lib, bws, coeffs, grids, plain_back, ms_plain, seed=3):
    """The mixed workload as requests to the transform server (pfsoft_server_*): 256 iDSOFT
    requests (coefficients -> fresh grids) and 256 DSOFT requests (the plain loop's grids ->
    fresh coefficients), independent, submitted in a shuffled order.
      saturated  all 512 submitted at once; transforms/s = 512 / (first submit -> last result)
      open_loop  Poisson arrivals at 60% of the saturated rate; p50 / p99 submit -> result
    Results are checked against the plain loop's (same kernels: equal)."""
    import numpy as np
    import torch

    from pfsoftlib_b200.serving import TransformServer

    rng = np.random.default_rng(seed)
    n = len(bws)
    out_g = [torch.empty_like(g) for g in grids]
    out_c = [torch.empty_like(c) for c in coeffs]
    jobs = [(1, i) for i in range(n)] + [(0, i) for i in range(n)]
    order = rng.permutation(len(jobs))
    torch.cuda.synchronize()

    def submit(srv, j):
        d, i = jobs[j]
        if d == 1:
            return srv.idsoft(coeffs[i], out_g[i])
        return srv.dsoft(grids[i], out_c[i])

    with TransformServer(budget_bytes=48 << 30, max_batch=16, streams=4) as srv:
        reqs = [submit(srv, j) for j in order[:64]]          # warm-up: tables, item lists
        for r in reqs:
            r.wait()
        srv.reset_stats()
        reqs = [submit(srv, j) for j in order]
        for r in reqs:
            r.wait()
        sat = srv.stats()
        rate = 0.6 * sat["transforms_per_s"]
        srv.reset_stats()
        gaps = rng.exponential(1.0 / rate, size=len(jobs))
        t0 = time.perf_counter()
        due = t0 + np.cumsum(gaps)
        reqs = []
        for k, j in enumerate(order):
            while time.perf_counter() < due[k]:
                pass
            reqs.append(submit(srv, j))
        for r in reqs:
            r.wait()
        ol = srv.stats()
    worst = 0.0
    for i in range(n):
        worst = max(worst, torch.linalg.vector_norm(out_c[i] - plain_back[i]).item()
                    / torch.linalg.vector_norm(plain_back[i]).item())
    keep = ("transforms_per_s", "p50_ms", "p99_ms", "mean_ms", "max_ms", "batches", "mean_batch",
            "max_concurrent_batches", "peak_bytes")
    plain_tps = 2 * n / (ms_plain / 1e3)
    return {
        "server": {"budget_bytes": 48 << 30, "max_batch": 16, "streams": 4},
        "saturated": {k: sat[k] for k in keep},
        "open_loop": dict({k: ol[k] for k in keep}, offered_per_s=rate),
        "speedup_vs_plain_loop": sat["transforms_per_s"] / plain_tps,
        "served_vs_plain_rel_l2_max": worst,
        "timing": "host clock, submit -> completion callback on the server's stream",
    }


def run_mixed(args):
    """256 independent transforms, bandwidths uniform over {32,48,64,96,128} (PCG64 seed 2),
    |f| = (1+l)^-1.5 with uniform phase (device generator, seed 2000 + i). One step = IDSOFT then
    DSOFT of every transform. Batched engine (one plan, one fused DWT launch per direction, CUDA
    graph, autotuned) against looping the single-transform entry points over the same inputs."""
    import ctypes

    import numpy as np
    import torch

    import pfsoftlib_b200
    from pfsoftlib_b200 import autotune

    lib = pfsoftlib_b200.load()
    torch.cuda.set_device(0)
    s = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(2)
    bws = [int(b) for b in rng.choice(MIXED_BANDS, size=256)]
    coeffs, grids, back = [], [], []
    for i, B in enumerate(bws):
        c = torch.empty(B * (4 * B * B - 1) // 3, dtype=torch.complex128, device="cuda")
        assert lib.pfsoft_cuda_random_coeffs(c.data_ptr(), B, 2000 + i, 2, 1.5, s) == 0
        coeffs.append(c)
        grids.append(torch.empty((2 * B,) * 3, dtype=torch.complex128, device="cuda"))
        back.append(torch.empty_like(c))
    tpc, timings = autotune.tune_batch(lib, bws, coeffs, grids, back, use_cache=False)
    plan = ctypes.c_void_p()
    arr = (ctypes.c_int * len(bws))(*bws)
    assert lib.pfsoft_batch_create(arr, len(bws), tpc, 0, ctypes.byref(plan)) == 0, lib.pfsoft_last_error()
    cp = (ctypes.c_void_p * len(bws))(*[t.data_ptr() for t in coeffs])
    gp = (ctypes.c_void_p * len(bws))(*[t.data_ptr() for t in grids])
    bp = (ctypes.c_void_p * len(bws))(*[t.data_ptr() for t in back])

    def batched():
        assert lib.pfsoft_batch_idsoft(plan, cp, gp, s) == 0
        assert lib.pfsoft_batch_dsoft(plan, gp, bp, s) == 0

    ws = torch.empty(lib.pfsoft_workspace_bytes(max(bws)) // 8, dtype=torch.float64, device="cuda")

    def plain():
        for i, B in enumerate(bws):
            assert lib.pfsoft_cuda_idsoft(coeffs[i].data_ptr(), B, grids[i].data_ptr(), ws.data_ptr(), ws.numel() * 8, s) == 0
            assert lib.pfsoft_cuda_dsoft(grids[i].data_ptr(), B, back[i].data_ptr(), ws.data_ptr(), ws.numel() * 8, s) == 0

    def timed(fn, steps):
        for _ in range(max(1, args.warmup)):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    steps = max(1, min(args.steps, 5))
    clocks = ClockSampler(0)
    clocks.start()
    ms_plain = timed(plain, steps)
    plain_back = [b.clone() for b in back]
    ms_batch = timed(batched, steps)
    clk = clocks.stop()
    # accuracy: round trip of the batched engine, and batched vs plain on the same inputs
    worst_rt, worst_vs = 0.0, 0.0
    for i in range(len(bws)):
        d = (back[i] - coeffs[i]).abs().max().item()
        worst_rt = max(worst_rt, d)
        nrm = torch.linalg.vector_norm(plain_back[i]).item()
        worst_vs = max(worst_vs, torch.linalg.vector_norm(back[i] - plain_back[i]).item() / nrm)
    lib.pfsoft_batch_destroy(plan)
    # the same batch with the split-precision tensor-core DWT
    plan_s = ctypes.c_void_p()
    assert lib.pfsoft_batch_create(arr, len(bws), tpc, 2, ctypes.byref(plan_s)) == 0, lib.pfsoft_last_error()

    def split():
        assert lib.pfsoft_batch_idsoft(plan_s, cp, gp, s) == 0
        assert lib.pfsoft_batch_dsoft(plan_s, gp, bp, s) == 0

    ms_split = timed(split, steps)
    split_status = lib.pfsoft_batch_status(plan_s)
    lib.pfsoft_batch_destroy(plan_s)
    split_vs, split_rt = 0.0, 0.0
    for i in range(len(bws)):
        split_vs = max(split_vs, (torch.linalg.vector_norm(back[i] - plain_back[i]) / torch.linalg.vector_norm(plain_back[i])).item())
        split_rt = max(split_rt, (torch.linalg.vector_norm(back[i] - coeffs[i]) / torch.linalg.vector_norm(coeffs[i])).item())
    served = run_served(lib, bws, coeffs, grids, plain_back, ms_plain)
    n = 2 * len(bws)
    line = {
        "metric": "DSOFT+iDSOFT transforms/s, 256 transforms of uneven bandwidth", "value": n / (ms_batch / 1e3),
        "unit": "transforms/s", "n_gpus": 1, "steps": steps, "warmup": max(1, args.warmup),
        "ms_per_step": ms_batch, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (device generator)",
        "config": {"workload": "256 transforms, B uniform over {32,48,64,96,128} (seed 2), |f|=(1+l)^-1.5, "
                               "one step = IDSOFT + DSOFT of all", "bandwidth_counts": {str(b): bws.count(b) for b in MIXED_BANDS},
                   "l2": "working set ~45 GB, far above L2"},
        "plain_loop": {"value": n / (ms_plain / 1e3), "ms_per_step": ms_plain},
        "speedup_vs_plain_loop": ms_plain / ms_batch,
        "split_precision": {"value": n / (ms_split / 1e3), "ms_per_step": ms_split,
                            "speedup_vs_plain_loop": ms_plain / ms_split, "rel_l2_vs_fp64_max": split_vs,
                            "round_trip_rel_l2_max": split_rt, "status": split_status,
                            "note": "DWT as bf16 digit-plane products on tcgen05, FP32 accumulation, FP64 sum"},
        "served": served,
        "autotune": {"transforms_per_cta": tpc, "round_trip_ms": timings},
        "accuracy": {"round_trip_max_abs": worst_rt, "batched_vs_plain_rel_l2_max": worst_vs},
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def run_b256(args):
    """64 transforms at B = 256 (|f| = (1+l)^-2 with uniform phase, device generator, seed 3 + i),
    streamed through one batch plan in groups of 8: per group the coefficients are generated, then
    IDSOFT (8 grids of 2.15 GB) and DSOFT of those grids. One step = all 64 IDSOFT + DSOFT; the
    generation is outside the timed region. Accuracy: round trip of every transform, and the first
    grid of the last group against the compiled reference's CPU DSOFT (all host threads) when it is
    built."""
    import ctypes

    import torch

    import pfsoftlib_b200

    lib = pfsoftlib_b200.load()
    torch.cuda.set_device(0)
    s = torch.cuda.current_stream().cuda_stream
    B, G, T = 256, 8, 64
    n = B * (4 * B * B - 1) // 3
    coeffs = [torch.empty(n, dtype=torch.complex128, device="cuda") for _ in range(G)]
    grids = [torch.empty((2 * B,) * 3, dtype=torch.complex128, device="cuda") for _ in range(G)]
    back = [torch.empty_like(c) for c in coeffs]
    plan = ctypes.c_void_p()
    assert lib.pfsoft_batch_create((ctypes.c_int * G)(*[B] * G), G, 0, 0, ctypes.byref(plan)) == 0, lib.pfsoft_last_error()
    cp = (ctypes.c_void_p * G)(*[t.data_ptr() for t in coeffs])
    gp = (ctypes.c_void_p * G)(*[t.data_ptr() for t in grids])
    bp = (ctypes.c_void_p * G)(*[t.data_ptr() for t in back])
    worst = [0.0]

    def group(g0, check):
        for i in range(G):
            assert lib.pfsoft_cuda_random_coeffs(coeffs[i].data_ptr(), B, 3 + g0 + i, 2, 2.0, s) == 0
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        assert lib.pfsoft_batch_idsoft(plan, cp, gp, s) == 0
        assert lib.pfsoft_batch_dsoft(plan, gp, bp, s) == 0
        e1.record()
        torch.cuda.synchronize()
        if check:
            for c, b in zip(coeffs, back):
                worst[0] = max(worst[0], (torch.linalg.vector_norm(b - c) / torch.linalg.vector_norm(c)).item())
        return e0.elapsed_time(e1)

    group(0, False)   # warm-up: tables, plan graph
    steps = max(1, min(args.steps, 2))
    clocks = ClockSampler(0)
    clocks.start()
    ms = 0.0
    for _ in range(steps):
        for g0 in range(0, T, G):
            ms += group(g0, True)
    clk = clocks.stop()
    lib.pfsoft_batch_destroy(plan)
    ms /= steps
    acc = {"round_trip_rel_l2_max": worst[0]}
    # checker: the compiled reference's CPU DSOFT of the last group's first grid, all host threads
    from oracle import oracle as orc
    if orc.Reference.available():
        ref = orc.Reference()
        g_h = grids[0].cpu().numpy()
        t0 = time.perf_counter()
        f_ref = ref.dsoft(g_h, ref.max_threads())
        acc["vs_reference_dsoft_rel_l2"] = orc.rel_l2(back[0].cpu().numpy(), f_ref)
        acc["vs_reference_dsoft_max_abs"] = orc.max_abs(back[0].cpu().numpy(), f_ref)
        acc["reference_dsoft_s"] = time.perf_counter() - t0
        acc["reference_threads"] = ref.max_threads()
        del g_h, f_ref
    line = {
        "metric": "DSOFT+iDSOFT transforms/s, 64 transforms at B=256", "value": 2 * T / (ms / 1e3),
        "unit": "transforms/s", "n_gpus": 1, "steps": steps, "warmup": 1, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (device generator)",
        "config": {"workload": "64 transforms at B=256 (seed 3+i, |f|=(1+l)^-2), groups of 8 through one "
                               "batch plan; one step = IDSOFT + DSOFT of all 64",
                   "grid": "512^3 complex128 (2.15 GB) each", "l2": "far above L2"},
        "accuracy": acc,
        "split_precision": "not run: the split-precision DWT covers B = 16..128 (K <= 256 keeps its "
                           "leading digit-plane sums exact in FP32)",
        "clocks": clk,
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


SERVE_BANDS = (16, 24, 32, 48, 64, 96, 128, 192, 256)   # log-spaced: equal weights = log-uniform


def run_serve_sweep(args):
    """Serving under Poisson arrivals: requests 50/50 DSOFT / iDSOFT, bandwidth log-uniform over
    16..256 (on the log-spaced grid SERVE_BANDS, PCG64 seed 4), offered at each rate of --rates for
    --seconds. Inputs per bandwidth are generated once on the device; each request writes one of
    four output buffers of its (bandwidth, direction), and waits for that buffer's previous request
    before reusing it. Per rate: achieved transforms/s and p50 / p99 latency (submit -> result,
    host clock at the server's completion callback)."""
    import numpy as np
    import torch

    import pfsoftlib_b200
    from pfsoftlib_b200.serving import TransformServer

    lib = pfsoftlib_b200.load()
    torch.cuda.set_device(0)
    s = torch.cuda.current_stream().cuda_stream
    pool = 4
    ins, outs = {}, {}
    for B in SERVE_BANDS:
        c = torch.empty(B * (4 * B * B - 1) // 3, dtype=torch.complex128, device="cuda")
        assert lib.pfsoft_cuda_random_coeffs(c.data_ptr(), B, 4000 + B, 2, 1.5, s) == 0
        g = torch.empty((2 * B,) * 3, dtype=torch.complex128, device="cuda")
        assert lib.pfsoft_cuda_idsoft(c.data_ptr(), B, g.data_ptr(), None, 0, s) == 0
        ins[B] = (g, c)                     # direction 0 reads the grid, 1 the coefficients
        outs[B] = ([torch.empty_like(c) for _ in range(pool)], [torch.empty_like(g) for _ in range(pool)])
    torch.cuda.synchronize()
    rng = np.random.default_rng(4)
    rates = [float(r) for r in args.rates.split(",") if r]
    sweep = []
    # the arena is one allocation of the whole budget: cap it by what the device has left after
    # the request buffers above (4 GiB kept back for tables, staging and the CUDA context)
    free, _ = torch.cuda.mem_get_info()
    budget = min(int(args.budget_gb * (1 << 30)), free - (4 << 30))
    with TransformServer(budget_bytes=budget, max_batch=16, streams=4) as srv:
        # warm-up: tables and item lists of every bandwidth and direction
        warm = [srv.submit(d, B, ins[B][d], outs[B][d][0]) for B in SERVE_BANDS for d in (0, 1)]
        for r in warm:
            r.wait(300)
        for rate in rates:
            n = max(20, int(rate * args.seconds))
            Bs = rng.choice(SERVE_BANDS, size=n)
            dirs = rng.integers(0, 2, size=n)
            gaps = rng.exponential(1.0 / rate, size=n)
            slot = {}
            last = {}
            srv.reset_stats()
            t0 = time.perf_counter()
            due = t0 + np.cumsum(gaps)
            reqs = []
            for i in range(n):
                B, d = int(Bs[i]), int(dirs[i])
                k = slot.get((B, d), 0)
                slot[(B, d)] = (k + 1) % pool
                prev = last.get((B, d, k))
                if prev is not None:
                    prev.wait(300)                 # the output buffer is free again
                while time.perf_counter() < due[i]:
                    pass
                r = srv.submit(d, B, ins[B][d], outs[B][d][k])
                last[(B, d, k)] = r
                reqs.append(r)
            for r in reqs:
                r.wait(300)
            st = srv.stats()
            sweep.append({"offered_per_s": rate, "requests": n, "transforms_per_s": st["transforms_per_s"],
                          "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"],
                          "max_ms": st["max_ms"], "mean_batch": st["mean_batch"],
                          "max_concurrent_batches": st["max_concurrent_batches"], "peak_bytes": st["peak_bytes"]})
            print(json.dumps({"rate": rate, **sweep[-1]}), file=sys.stderr, flush=True)
    best = max(x["transforms_per_s"] for x in sweep)
    line = {
        "metric": "served DSOFT/iDSOFT transforms/s under Poisson arrivals (best over the sweep)", "value": best,
        "unit": "transforms/s", "n_gpus": 1, "steps": len(rates), "warmup": 1, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (device generator)",
        "config": {"workload": "requests 50/50 DSOFT/iDSOFT, B log-uniform over 16..256 on "
                               f"{list(SERVE_BANDS)} (seed 4), Poisson arrivals", "rates": rates,
                   "seconds_per_rate": args.seconds, "budget_bytes": budget, "max_batch": 16, "streams": 4,
                   "output_buffers_per_bandwidth_and_direction": pool},
        "sweep": sweep,
    }
    print(json.dumps(line), flush=True)


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
    acc = {"round_trip_rel_l2": orc.rel_l2(f_h, coeffs_h), "round_trip_max_abs": orc.max_abs(f_h, coeffs_h)}

    # ---- per-stage roofline
    stages = {}
    for i in range(nstages):
        name = lib.pfsoft_profile_stage_name(i).decode()
        if st_cnt[i] == 0:
            continue
        per = st_ms[i] / st_cnt[i]
        if name.startswith("fft"):
            achieved = FFT_PASS_BYTES / (per / 1e3) / 1e9
            stages[name] = {"bound": "hbm", "ms_per_launch": per, "launches": int(st_cnt[i]),
                            "achieved": achieved, "peak": 6551.7, "unit": "GB/s", "frac": achieved / 6551.7}
        elif name.startswith("dwt"):
            achieved = DWT_FLOPS / (per / 1e3) / 1e12
            stages[name] = {"bound": "tensor", "ms_per_launch": per, "launches": int(st_cnt[i]),
                            "achieved": achieved, "peak": FP64_PEAK_TFLOPS, "unit": "TFLOP/s",
                            "frac": achieved / FP64_PEAK_TFLOPS}
        else:
            stages[name] = {"ms_per_launch": per, "launches": int(st_cnt[i])}
    dominant = max((k for k in stages if "frac" in stages[k]), key=lambda k: stages[k]["ms_per_launch"] * stages[k]["launches"])
    d = stages[dominant]
    # DRAM bytes per launch (read + write) from one ncu capture of the same kernels at B = 128,
    # profiles/dwt_single_b128.md and profiles/fft_pass_b128.md
    traffic = {"dwt_forward": 268.37e6 + 43.51e6, "dwt_inverse": 46.44e6 + 208.20e6,
               "fft_forward_gamma": 268.5e6 + 221.6e6, "fft_inverse_alpha": 268.5e6 + 214.7e6,
               "fft_inverse_gamma": 268.5e6 + 219.7e6}
    roofline = {"kernel": dominant, "bound": d["bound"], "achieved": d["achieved"], "peak": d["peak"],
                "unit": d["unit"], "frac": d["frac"], "traffic": traffic.get(dominant),
                "peak_source": ("measured FP64 MMA peak (own micro-benchmark; MEASURED_PEAKS.json has no FP64 entry)"
                                if d["bound"] == "tensor" else "measured copy bandwidth, MEASURED_PEAKS.json hbm_gbs")}

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
    t_e2e = time.perf_counter() - t0
    if dist is not None:
        t = torch.tensor([t_e2e], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_e2e = float(t.item())
    e2e = {"value": TRANSFORMS_PER_STEP * e2e_steps * world / t_e2e, "unit": UNIT,
           "h2d_bytes_per_step": COEF_BYTES + GRID_BYTES, "d2h_bytes_per_step": GRID_BYTES + COEF_BYTES,
           "api": "pfsoft_idsoft_host + pfsoft_dsoft_host (include/pfsoft_b200.h), pinned host buffers", "steps": e2e_steps}

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
        "config": workload_config("inputs larger than L2: 268 MB grid and workspace, 45 MB coefficients"),
        "e2e": e2e, "gpu_launches": int(launches), "roofline": roofline, "stages": stages,
        "cpu_baseline": cpu, "accuracy": acc, "clocks": clk,
        "parallelism": f"replicas x{world} (independent transforms per GPU, no collective)",
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
