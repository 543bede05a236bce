"""One transform sharded over several ranks (pfsoftlib_b200/shard.py, C ABI pfsoft_shard_*).

CPU: the plan's own checks (tests/cpp/shard_plan.cpp), the host-only queries, and the
orchestration of ShardedTransform over gloo with 2 and 3 ranks, whose steps run on the CPU
(FFTs by numpy, the DWT replaced by copying each owned bin's beta column, the exchange by the
plan's own copy runs), against numpy's transform of the whole grid.
GPU: every rank of a P-rank plan emulated in turn on one GPU (no kernel waits on another rank's;
the exchange is a copy between the ranks' buffers on the same device), both exchange modes,
against the unsharded transform; and ShardedTransform end to end over a one-rank NCCL group.
"""
import ctypes
import os
import shutil
import socket
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "pfsoftlib_b200", "csrc")


def _cxx():
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")


def _cuda_include():
    for d in (os.environ.get("CUDA_HOME", ""), "/usr/local/cuda"):
        if d and os.path.exists(os.path.join(d, "include", "cuda_runtime.h")):
            return os.path.join(d, "include")
    pytest.skip("cuda_runtime.h not found")


def test_plan_program(tmp_path):
    exe = str(tmp_path / "shard_plan")
    subprocess.run([_cxx(), "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", CSRC, "-I", _cuda_include(),
                    os.path.join(ROOT, "tests", "cpp", "shard_plan.cpp"), "-o", exe],
                   check=True, capture_output=True, text=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == "ok"


def test_host_queries(lib):
    from pfsoftlib_b200.shard import FORWARD, INVERSE, PACK, SCATTER, UNPACK, ShardPlan

    B, P = 12, 3
    plans = [ShardPlan(B, P, r) for r in range(P)]
    N = 2 * B
    assert [p.layers for p in plans] == [(0, 8), (8, 8), (16, 8)]
    # the exchange is consistent: what p sends to q is what q receives from p
    for d in (FORWARD, INVERSE):
        for p in range(P):
            for q in range(P):
                assert plans[p].counts(d)[0][q] == plans[q].counts(d)[1][p]
    bins = np.concatenate([plans[0].bins(r) for r in range(P)])
    assert len(np.unique(bins)) == len(bins) == (N - 1) ** 2
    assert sum(len(plans[0].classes(r)) for r in range(P)) == B * (B + 1) // 2
    r = plans[1].runs(FORWARD, SCATTER)
    assert len(r["len"]) == (N - 1) ** 2 and set(r["len"].tolist()) == {8}
    assert set(r["slot"].tolist()) == {0, 1, 2}
    assert plans[1].runs(INVERSE, UNPACK)["len"].sum() == (N - 1) ** 2 * 8
    assert plans[1].runs(FORWARD, PACK)["slot"].max() == 0
    with pytest.raises(ValueError):
        plans[0].runs(2, 0)
    from pfsoftlib_b200 import PfsoftError

    for bad in ((0, 2, 0), (8, 0, 0), (8, 2, 2), (8, 65, 0)):
        with pytest.raises(PfsoftError):
            ShardPlan(*bad)


# ---- gloo: the orchestration with CPU steps ----------------------------------------------------

class CpuSteps:
    """ShardPlan's step interface on CPU tensors; the exchange uses the plan's copy runs. With
    real=False the DWT is replaced by copying the owned bins' beta columns (the 'coefficients' are
    the (N^3) spectrum itself); with real=True each rank runs the long-double oracle's DWT stage
    on its own order classes (oracle/soft_oracle.c: oracle_dwt_forward / oracle_dwt_inverse)."""

    def __init__(self, B, nranks, rank, real=False):
        from pfsoftlib_b200.shard import ShardPlan

        self.p = ShardPlan(B, nranks, rank)
        self.B, self.N, self.nranks, self.rank = B, 2 * B, nranks, rank
        self.own = self.p.bins(rank)
        self.run = {(d, s): self.p.runs(d, s) for d in (0, 1) for s in (0, 1, 2)}
        self.real = real
        if real:
            from oracle.oracle import Oracle

            self.oracle = Oracle()
            self.cls = self.p.classes(rank)

    layers = property(lambda self: self.p.layers)

    def counts(self, d):
        return self.p.counts(d)

    def slab_elems(self):
        return self.p.slab_elems()

    def spectrum_elems(self):
        return self.N ** 3

    def coef_elems(self):
        return self.B * (4 * self.B * self.B - 1) // 3 if self.real else self.N ** 3

    def _copy(self, d, step, src, dst):
        r = self.run[(d, step)]
        s, t = src.numpy(), dst.numpy()
        for so, do, n in zip(r["src_off"], r["dst_off"], r["len"]):
            t[do:do + n] = s[so:so + n]

    def pack(self, d, src, send):
        self._copy(d, 1, src, send)

    def unpack(self, d, recv, dst):
        self._copy(d, 2, recv, dst)

    def fft_forward(self, g, s):
        nk, N = self.layers[1], self.N
        if nk:
            F = np.fft.fft2(g.numpy().reshape(nk, N, N), axes=(1, 2))   # [layer][alpha f][gamma f]
            s.numpy()[:] = F.transpose(2, 1, 0).reshape(-1)

    def fft_inverse(self, s, g):
        nk, N, B = self.layers[1], self.N, self.B
        if nk:
            S = s.numpy().reshape(N, N, nk).copy()
            S[B] = 0
            S[:, B] = 0
            g.numpy()[:] = np.fft.ifft2(S.transpose(2, 1, 0), axes=(1, 2)).reshape(-1)

    def dwt_forward(self, spec, coeffs):
        N = self.N
        if self.real:
            c = coeffs.numpy()
            c[:] = 0
            self.oracle.dwt_forward(spec.numpy(), self.B, self.cls, out=c)
            return
        c = coeffs.numpy().reshape(N * N, N)
        c[:] = 0
        c[self.own] = spec.numpy().reshape(N * N, N)[self.own]

    def dwt_inverse(self, coeffs, spec):
        N = self.N
        if self.real:
            self.oracle.dwt_inverse(coeffs.numpy(), self.B, self.cls, out=spec.numpy())
            return
        spec.numpy().reshape(N * N, N)[self.own] = coeffs.numpy().reshape(N * N, N)[self.own]


def _spectrum(grid, B):
    """Full beta-innermost spectrum [gamma f][alpha f][layer] with the Nyquist bins zeroed."""
    S = np.fft.fft2(grid, axes=(1, 2)).transpose(2, 1, 0).copy()
    S[B] = 0
    S[:, B] = 0
    return S


def _gloo_rank(rank, world, port, B, errq):
    import torch
    import torch.distributed as dist

    from pfsoftlib_b200.shard import ShardedTransform

    try:
        os.environ["MASTER_ADDR"], os.environ["MASTER_PORT"] = "127.0.0.1", str(port)
        dist.init_process_group("gloo", rank=rank, world_size=world)
        N = 2 * B
        rng = np.random.default_rng(7)
        grid = rng.standard_normal((N, N, N)) + 1j * rng.standard_normal((N, N, N))
        st = ShardedTransform(B, device="cpu", engine=CpuSteps(B, world, rank))
        first, count = st.layers
        out = st.dsoft(torch.from_numpy(grid[first:first + count].copy()))
        ref = _spectrum(grid, B)
        assert np.array_equal(out.numpy().reshape(N, N, N), ref), "forward"
        # inverse of an arbitrary spectrum
        S2 = rng.standard_normal((N, N, N)) + 1j * rng.standard_normal((N, N, N))
        slab = st.idsoft(torch.from_numpy(S2.reshape(-1).copy()))
        S2[B] = 0
        S2[:, B] = 0
        g2 = np.fft.ifft2(S2.transpose(2, 1, 0), axes=(1, 2))
        assert np.allclose(slab.numpy(), g2[first:first + count], rtol=0, atol=1e-13), "inverse"
        # coefficients left distributed by class: each rank's part feeds its own inverse
        part = st.dsoft(torch.from_numpy(grid[first:first + count].copy()), gather=False)
        own = np.zeros(N * N, bool)
        own[st.plan.own] = True
        assert not part.numpy().reshape(N * N, N)[~own].any(), "partial vector outside own bins"
        slab = st.idsoft(part)
        g3 = np.fft.ifft2(ref.transpose(2, 1, 0), axes=(1, 2))
        assert np.allclose(slab.numpy(), g3[first:first + count], rtol=0, atol=1e-12), "distributed round trip"
        dist.barrier()
        dist.destroy_process_group()
    except BaseException as e:   # reported to the parent
        errq.put(f"rank {rank}: {type(e).__name__}: {e}")
        raise


def _gloo_rank_oracle(rank, world, port, B, errq):
    """Each rank runs the oracle's DWT on its own classes: the assembled coefficients (all-reduce)
    against the oracle's DSOFT of the whole grid, and each rank's inverse slab against the
    oracle's IDSOFT, both within 1e-13 relative L2."""
    import torch
    import torch.distributed as dist

    from oracle import oracle as orc
    from pfsoftlib_b200.shard import ShardedTransform

    try:
        os.environ["MASTER_ADDR"], os.environ["MASTER_PORT"] = "127.0.0.1", str(port)
        dist.init_process_group("gloo", rank=rank, world_size=world)
        ora = orc.Oracle()
        c = orc.coeffs_uniform(B, seed=31)
        grid = ora.idsoft(c, B)
        st = ShardedTransform(B, device="cpu", engine=CpuSteps(B, world, rank, real=True))
        first, count = st.layers
        f = st.dsoft(torch.from_numpy(grid[first:first + count].copy()))
        assert orc.rel_l2(f.numpy(), ora.dsoft(grid)) <= 1e-13, "forward vs oracle"
        assert orc.rel_l2(f.numpy(), c) <= 1e-13, "round trip"
        slab = st.idsoft(torch.from_numpy(c.copy()))
        assert orc.rel_l2(slab.numpy().reshape(count, 2 * B, 2 * B), grid[first:first + count]) <= 1e-13, "inverse"
        dist.barrier()
        dist.destroy_process_group()
    except BaseException as e:   # reported to the parent
        errq.put(f"rank {rank}: {type(e).__name__}: {e}")
        raise


@pytest.mark.parametrize("world,B,target", [(2, 8, "copy"), (3, 5, "copy"), (2, 6, "oracle"), (3, 7, "oracle")])
def test_sharded_transform_gloo(world, B, target):
    import torch.multiprocessing as mp

    from pfsoftlib_b200 import _lib

    _lib.load()   # build once before the ranks start
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    errq = ctx.Queue()
    fn = _gloo_rank if target == "copy" else _gloo_rank_oracle
    procs = [ctx.Process(target=fn, args=(r, world, port, B, errq)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(240)
    alive = [p for p in procs if p.is_alive()]
    for p in alive:
        p.kill()
    errs = []
    while not errq.empty():
        errs.append(errq.get())
    assert not alive and not errs and all(p.exitcode == 0 for p in procs), errs


# ---- GPU ----------------------------------------------------------------------------------------

def _single(lib, fn, src, B):
    import torch

    s = torch.cuda.current_stream().cuda_stream
    if fn == "idsoft":
        out = torch.empty((2 * B,) * 3, dtype=torch.complex128, device="cuda")
        assert lib.pfsoft_cuda_idsoft(src.data_ptr(), B, out.data_ptr(), None, 0, s) == 0, lib.pfsoft_last_error()
    else:
        out = torch.empty(B * (4 * B * B - 1) // 3, dtype=torch.complex128, device="cuda")
        assert lib.pfsoft_cuda_dsoft(src.data_ptr(), B, out.data_ptr(), None, 0, s) == 0, lib.pfsoft_last_error()
    return out


def _emulate(B, P, mode):
    """Forward and inverse of one transform with P plans run one after another on this GPU."""
    import torch

    from pfsoftlib_b200.shard import FORWARD, INVERSE, ShardPlan

    N = 2 * B
    plans = [ShardPlan(B, P, r) for r in range(P)]
    nan = complex(np.nan, np.nan)
    cplx = dict(dtype=torch.complex128, device="cuda")

    def exchange(direction, srcs, dsts):
        if mode == "scatter":
            for p in range(P):
                plans[p].scatter(direction, srcs[p], dsts)
            return
        sends, recvs = [], []
        for p in range(P):
            sn, rn = plans[p].counts(direction)
            sends.append(torch.full((sum(sn),), nan, **cplx))
            recvs.append(torch.full((sum(rn),), nan, **cplx))
            plans[p].pack(direction, srcs[p], sends[p])
        for q in range(P):   # the all-to-all: q's part from p is p's part for q
            roff = np.concatenate([[0], np.cumsum(plans[q].counts(direction)[1])])
            for p in range(P):
                soff = np.concatenate([[0], np.cumsum(plans[p].counts(direction)[0])])
                recvs[q][roff[p]:roff[p + 1]] = sends[p][soff[q]:soff[q + 1]]
        for q in range(P):
            plans[q].unpack(direction, recvs[q], dsts[q])

    g = torch.randn((N, N, N), **cplx)
    slabs, specs = [], []
    for p in range(P):
        first, count = plans[p].layers
        slabs.append(g[first:first + count].reshape(-1).contiguous())
        specs.append(torch.full((count * N * N,), nan, **cplx))
        plans[p].fft_forward(slabs[p], specs[p])
    full = [torch.full((N ** 3,), nan, **cplx) for _ in range(P)]   # NaN where a rank owns nothing
    exchange(FORWARD, specs, full)
    coef = torch.zeros(plans[0].coef_elems(), **cplx)
    for q in range(P):
        c = torch.full_like(coef, nan)
        plans[q].dwt_forward(full[q], c)
        coef += c
    # inverse of the result
    for q in range(P):
        full[q].fill_(nan)
        plans[q].dwt_inverse(coef, full[q])
    outs = []
    for p in range(P):
        specs[p].fill_(nan)
    exchange(INVERSE, full, specs)
    for p in range(P):
        first, count = plans[p].layers
        o = torch.full((count * N * N,), nan, **cplx)
        plans[p].fft_inverse(specs[p], o)
        outs.append(o.reshape(count, N, N))
    torch.cuda.synchronize()
    return g, coef, torch.cat(outs)


@pytest.mark.gpu
@pytest.mark.parametrize("B,P,mode", [(8, 2, "scatter"), (8, 3, "pack"), (5, 4, "scatter"), (33, 3, "pack"),
                                      (64, 8, "scatter"), (64, 5, "pack"), (128, 4, "scatter"), (2, 8, "pack"),
                                      (256, 3, "scatter")])
def test_emulated_ranks_match_single_gpu(lib, B, P, mode):
    g, coef, back = _emulate(B, P, mode)
    ref = _single(lib, "dsoft", g, B)
    gref = _single(lib, "idsoft", ref, B)
    import torch

    torch.cuda.synchronize()
    # the same kernels over the same values: equal up to the summation of exact zeros
    assert torch.isfinite(coef).all() and torch.isfinite(back).all()
    assert torch.equal(coef, ref), (coef - ref).abs().max().item()
    assert torch.equal(back, gref), (back - gref).abs().max().item()


@pytest.mark.gpu
@pytest.mark.parametrize("B,P,mode", [(8, 3, "scatter"), (13, 4, "pack")])
def test_emulated_ranks_match_oracle(lib, oracle, B, P, mode):
    """The sharded forward and inverse against the long-double oracle's DSOFT / IDSOFT."""
    from oracle import oracle as orc

    g, coef, back = _emulate(B, P, mode)
    g_h = g.cpu().numpy()
    f_ref = oracle.dsoft(g_h)
    assert orc.rel_l2(coef.cpu().numpy(), f_ref) <= 1e-13
    assert orc.rel_l2(back.cpu().numpy(), oracle.idsoft(coef.cpu().numpy(), B)) <= 1e-13


@pytest.mark.gpu
def test_sharded_transform_one_rank_nccl(lib):
    """ShardedTransform end to end through NCCL (a one-rank group: the collectives run, the
    exchange is a self-copy) against the unsharded transform."""
    import torch
    import torch.distributed as dist

    from pfsoftlib_b200.shard import ShardedTransform

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        B = 48
        N = 2 * B
        g = torch.randn((N, N, N), dtype=torch.complex128, device="cuda")
        st = ShardedTransform(B)
        assert st.layers == (0, N)
        coef = st.dsoft(g)
        back = st.idsoft(coef)
        torch.cuda.synchronize()
        ref = _single(lib, "dsoft", g, B)
        assert torch.equal(coef, ref)
        assert torch.equal(back, _single(lib, "idsoft", ref, B))
    finally:
        dist.destroy_process_group()
