"""Transform server (pfsoft_server_*, pfsoftlib_b200.serving).

CPU: the host policy -- workspace arena, batch forming, admission by HBM footprint, backfill and
aging, cancellation, and a simulated serving run -- compiled from serving.hpp on its own.
GPU: each result is the same alone and in a mix of bandwidths and directions, requests that
arrive while others run are admitted as memory frees up and overlap on the device, requests
larger than the budget are rejected, queued requests can be cancelled, and inputs produced on
another stream are waited for.
"""
import ctypes
import os
import shutil
import subprocess
import threading
import time

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "pfsoftlib_b200", "csrc")

REL_TOL = 1e-13   # served vs plain per-transform path (identical kernels: equal in practice)


def _cxx():
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")


def test_policy(tmp_path):
    exe = str(tmp_path / "serving_policy")
    subprocess.run([_cxx(), "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", CSRC,
                    os.path.join(ROOT, "tests", "cpp", "serving_policy.cpp"), "-o", exe],
                   check=True, capture_output=True, text=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == "ok"


def test_stats_layout_matches_header():
    """ServerStats mirrors struct pfsoft_server_stats field for field."""
    from pfsoftlib_b200.serving import ServerStats

    src = open(os.path.join(ROOT, "include", "pfsoft_b200.h")).read()
    body = src[src.index("typedef struct pfsoft_server_stats {"):]
    body = body[:body.index("} pfsoft_server_stats;")]
    names = []
    for line in body.splitlines()[1:]:
        decl = line.split("/*")[0].strip().rstrip(";")
        if not decl:
            continue
        names += [p for p in decl.replace(",", " ").split() if p not in ("long", "double", "int", "size_t")]
    assert names == [f for f, _ in ServerStats._fields_]


# ---------------------------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------------------------

def _coeffs(lib, torch, B, seed):
    c = torch.empty(B * (4 * B * B - 1) // 3, dtype=torch.complex128, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    assert lib.pfsoft_cuda_random_coeffs(c.data_ptr(), B, seed, 1, 1.0, s) == 0
    return c


def _plain(lib, torch, direction, B, inp):
    s = torch.cuda.current_stream().cuda_stream
    if direction == 0:
        out = torch.empty(B * (4 * B * B - 1) // 3, dtype=torch.complex128, device="cuda")
        assert lib.pfsoft_cuda_dsoft(inp.data_ptr(), B, out.data_ptr(), None, 0, s) == 0
    else:
        out = torch.empty((2 * B,) * 3, dtype=torch.complex128, device="cuda")
        assert lib.pfsoft_cuda_idsoft(inp.data_ptr(), B, out.data_ptr(), None, 0, s) == 0
    return out


def _rel(a, b):
    return ((a - b).abs().pow(2).sum().sqrt() / b.abs().pow(2).sum().sqrt()).item()


def _mix(lib, torch, n=28, seed=5):
    """n requests: bandwidths over {1, 2, 3, 5, 8, 16, 24, 32, 48, 64}, both directions, plain results."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        B = int(rng.choice((1, 2, 3, 5, 8, 16, 24, 32, 48, 64)))
        direction = int(rng.integers(0, 2))
        c = _coeffs(lib, torch, B, 100 + i)
        inp = c if direction == 1 else _plain(lib, torch, 1, B, c)
        out.append((direction, B, inp, _plain(lib, torch, direction, B, inp)))
    torch.cuda.synchronize()
    return out


def _out_like(torch, direction, B):
    if direction == 0:
        return torch.full((B * (4 * B * B - 1) // 3,), float("nan"), dtype=torch.complex128, device="cuda")
    return torch.full((2 * B,) * 3, float("nan"), dtype=torch.complex128, device="cuda")


@pytest.mark.gpu
def test_same_alone_and_in_mix(lib):
    import torch

    from pfsoftlib_b200.serving import TransformServer

    mix = _mix(lib, torch)
    with TransformServer(budget_bytes=2 << 30, max_batch=8, streams=4) as srv:
        alone = []
        for direction, B, inp, _ in mix:
            o = _out_like(torch, direction, B)
            srv.submit(direction, B, inp, o).wait()
            alone.append(o)
        st = srv.stats()
        assert st["batches"] == len(mix) and st["completed"] == len(mix)
        # all at once: equal (direction, B) requests share batches
        srv.pause()
        together, reqs = [], []
        for direction, B, inp, _ in mix:
            o = _out_like(torch, direction, B)
            reqs.append(srv.submit(direction, B, inp, o))
            together.append(o)
        srv.resume()
        for r in reqs:
            r.wait()
        st = srv.stats()
        assert st["batches"] < 2 * len(mix)          # some requests were batched together
        assert st["mean_batch"] > 1.0
    for (direction, B, inp, ref), a, t in zip(mix, alone, together):
        assert torch.equal(a, t), f"B={B} dir={direction}: result differs alone vs in the mix"
        assert _rel(a, ref) <= REL_TOL, f"B={B} dir={direction}: served vs plain {_rel(a, ref):.2e}"


@pytest.mark.gpu
def test_split_server_mixed_bandwidths(lib, oracle):
    """Split mode: requests of one direction and different bandwidths share a batch and one
    split-precision launch. Each result is bitwise the same alone and in the mix, within 1e-11
    (relative L2) of the plain FP64 path, and the small ones match the long-double oracle."""
    import torch

    from oracle import oracle as orc
    from pfsoftlib_b200.serving import TransformServer

    tol = 1e-11
    mix = _mix(lib, torch, n=24, seed=9)
    with TransformServer(budget_bytes=2 << 30, max_batch=8, streams=3, split=True) as srv:
        alone = []
        for direction, B, inp, _ in mix:
            o = _out_like(torch, direction, B)
            srv.submit(direction, B, inp, o).wait()
            alone.append(o)
        srv.pause()
        srv.reset_stats()
        together, reqs = [], []
        for direction, B, inp, _ in mix:
            o = _out_like(torch, direction, B)
            reqs.append(srv.submit(direction, B, inp, o))
            together.append(o)
        srv.resume()
        for r in reqs:
            r.wait()
        st = srv.stats()
        assert st["mean_batch"] > 2.0, st              # mixed bandwidths batched together
        assert st["failed"] == 0
    for (direction, B, inp, ref), a, t in zip(mix, alone, together):
        assert torch.equal(a, t), f"B={B} dir={direction}: result differs alone vs in the mix"
        assert _rel(a, ref) <= tol, f"B={B} dir={direction}: split served vs FP64 {_rel(a, ref):.2e}"
        if B <= 16:
            x = inp.cpu().numpy()
            want = oracle.dsoft(x) if direction == 0 else oracle.idsoft(x, B)
            assert orc.rel_l2(a.cpu().numpy().reshape(want.shape), want) <= tol, f"B={B} dir={direction} vs oracle"


@pytest.mark.gpu
def test_split_server_rejects_large_bandwidth(lib):
    import torch

    from pfsoftlib_b200 import _lib
    from pfsoftlib_b200.serving import TransformServer

    with TransformServer(budget_bytes=1 << 30, max_batch=4, streams=1, split=True) as srv:
        c = torch.empty(257 * (4 * 257 * 257 - 1) // 3, dtype=torch.complex128, device="cuda")
        g = torch.empty(514 ** 3, dtype=torch.complex128, device="cuda")
        with pytest.raises(_lib.PfsoftError) as e:
            srv.submit(1, 257, c, g)
        assert e.value.status == _lib.PFSOFT_EINVAL


@pytest.mark.gpu
def test_continuous_admission_under_budget(lib):
    """Budget for 3 spectra at B=32: 40 requests arriving from another thread while batches run
    all finish, the arena never exceeds the budget, and batches overlap on the device."""
    import torch

    from pfsoftlib_b200.serving import TransformServer

    B = 32
    ws = lib.pfsoft_workspace_bytes(B)
    cs = [_coeffs(lib, torch, B, 500 + i) for i in range(40)]
    refs = [_plain(lib, torch, 1, B, c) for c in cs]
    torch.cuda.synchronize()
    outs = [_out_like(torch, 1, B) for _ in cs]
    with TransformServer(budget_bytes=3 * ws, max_batch=2, streams=4) as srv:
        reqs = [None] * len(cs)

        def producer():
            for i, (c, o) in enumerate(zip(cs, outs)):
                reqs[i] = srv.idsoft(c, o)
                if i % 5 == 4:
                    time.sleep(0.002)

        th = threading.Thread(target=producer)
        th.start()
        th.join()
        for r in reqs:
            r.wait()
        st = srv.stats()
    assert st["completed"] == len(cs) and st["failed"] == 0
    assert st["peak_bytes"] <= 3 * ws
    assert st["max_concurrent_batches"] >= 2
    assert st["p99_ms"] >= st["p50_ms"] > 0
    for o, r in zip(outs, refs):
        assert torch.equal(o, r)


@pytest.mark.gpu
def test_reject_cancel_and_errors(lib):
    import torch

    from pfsoftlib_b200 import PfsoftError, _lib
    from pfsoftlib_b200.serving import TransformServer

    with TransformServer(budget_bytes=lib.pfsoft_workspace_bytes(16), max_batch=4, streams=2) as srv:
        c32 = _coeffs(lib, torch, 32, 1)
        g32 = _out_like(torch, 1, 32)
        with pytest.raises(PfsoftError) as e:          # larger than the whole budget: rejected
            srv.idsoft(c32, g32)
        assert e.value.status == _lib.PFSOFT_ENOMEM
        srv.pause()
        cs = [_coeffs(lib, torch, 16, 10 + i) for i in range(3)]
        gs = [_out_like(torch, 1, 16) for _ in cs]
        reqs = [srv.idsoft(c, g) for c, g in zip(cs, gs)]
        assert not reqs[1].done()
        assert reqs[1].cancel()
        srv.resume()
        reqs[0].wait()
        reqs[2].wait()
        with pytest.raises(PfsoftError) as e:
            reqs[1].wait()
        assert e.value.status == _lib.PFSOFT_ECANCELED
        assert not reqs[0].cancel()                     # already finished
        st = srv.stats()
        assert st["rejected"] == 1 and st["cancelled"] == 1 and st["completed"] == 2
        assert torch.isnan(gs[1]).all()                 # the cancelled request never ran
        rid = ctypes.c_longlong()
        assert lib.pfsoft_server_submit(srv._h, 2, 16, cs[0].data_ptr(), gs[0].data_ptr(), None,
                                        ctypes.byref(rid)) == _lib.PFSOFT_EINVAL
        assert lib.pfsoft_server_submit(srv._h, 0, 0, cs[0].data_ptr(), gs[0].data_ptr(), None,
                                        ctypes.byref(rid)) == _lib.PFSOFT_EINVAL
        assert lib.pfsoft_server_poll(srv._h, 123456) == _lib.PFSOFT_EINVAL


@pytest.mark.gpu
def test_waits_for_the_producing_stream(lib):
    """Coefficients generated on a side stream behind a long kernel are read only after it."""
    import torch

    from pfsoftlib_b200.serving import TransformServer

    B = 24
    ref_c = _coeffs(lib, torch, B, 77)
    ref = _plain(lib, torch, 1, B, ref_c)
    torch.cuda.synchronize()
    side = torch.cuda.Stream()
    c = torch.zeros_like(ref_c)
    g = _out_like(torch, 1, B)
    big = torch.empty(1 << 27, device="cuda")
    with TransformServer(budget_bytes=1 << 30, max_batch=4, streams=2) as srv:
        with torch.cuda.stream(side):
            for _ in range(20):
                big.mul_(1.0001)                       # keeps the side stream busy
            assert lib.pfsoft_cuda_random_coeffs(c.data_ptr(), B, 77, 1, 1.0, side.cuda_stream) == 0
            req = srv.idsoft(c, g, stream=side)
        req.wait()
    assert torch.equal(g, ref)


@pytest.mark.gpu
def test_large_bandwidth_requests(lib):
    """B = 160 runs the per-transform DWT kernels inside a served batch."""
    import torch

    from pfsoftlib_b200.serving import TransformServer

    B = 160
    c = [_coeffs(lib, torch, B, 900 + i) for i in range(2)]
    refs = [_plain(lib, torch, 1, B, x) for x in c]
    torch.cuda.synchronize()
    outs = [_out_like(torch, 1, B) for _ in c]
    with TransformServer(budget_bytes=3 * lib.pfsoft_workspace_bytes(B), max_batch=2, streams=2) as srv:
        srv.pause()
        reqs = [srv.idsoft(x, o) for x, o in zip(c, outs)]
        srv.resume()
        for r in reqs:
            r.wait()
        assert srv.stats()["batches"] == 1
    for o, r in zip(outs, refs):
        assert torch.equal(o, r)
