"""GPU test of pfsoft_cuda_dsoft_noalloc, the DSOFT entry point for callers that cannot
allocate device memory (a framework-owned, capped memory pool; a hard per-process memory limit;
a loop that must not take cudaMalloc's locks or cudaFree's device synchronisation). It keeps its
scratch in a device array the library holds from load to exit, which limits it to B <= 32.

Checked through the C ABI: two calls in a row (different bandwidths, so the second rebuilds the
tables in the shared array) each agree with pfsoft_cuda_dsoft within the parity tolerance used
by the other GPU tests; bandwidths beyond the limit are rejected with PFSOFT_EINVAL. This file
sorts last so a run that stops at the first failure has run everything else first."""
import numpy as np
import pytest

from oracle import oracle as orc

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

REL_TOL = 1e-13
ABS_TOL = 1e-12


def _grid(B, seed):
    rng = np.random.default_rng(seed)
    N = 2 * B
    return rng.uniform(-1, 1, (N, N, N)) + 1j * rng.uniform(-1, 1, (N, N, N))


def _dsoft(lib, fn, grid, B):
    g = torch.from_numpy(grid).cuda()
    out = torch.full((orc.coef_count(B),), complex(np.nan, np.nan), dtype=torch.complex128, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    if fn == "noalloc":
        rc = lib.pfsoft_cuda_dsoft_noalloc(g.data_ptr(), B, out.data_ptr(), s)
    else:
        rc = lib.pfsoft_cuda_dsoft(g.data_ptr(), B, out.data_ptr(), None, 0, s)
    assert rc == 0, lib.pfsoft_last_error()
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_matches_dsoft_on_two_calls_in_a_row(lib):
    for B, seed in ((32, 1), (16, 2)):
        grid = _grid(B, seed)
        got = _dsoft(lib, "noalloc", grid, B)
        ref = _dsoft(lib, "dsoft", grid, B)
        assert np.isfinite(got).all()
        assert orc.rel_l2(got, ref) <= REL_TOL
        assert orc.max_abs(got, ref) <= ABS_TOL


def test_noalloc_bandwidth_sequence(lib):
    """Each call changes the bandwidth (small and odd FFT lengths: generic and direct-radix plans,
    a leading radix-1 stage; tables rebuilt from smaller to larger and back)."""
    for i, B in enumerate((1, 3, 5, 31, 32, 8)):
        grid = _grid(B, 40 + i)
        got = _dsoft(lib, "noalloc", grid, B)
        ref = _dsoft(lib, "dsoft", grid, B)
        assert orc.rel_l2(got, ref) <= REL_TOL, B
        assert orc.max_abs(got, ref) <= ABS_TOL, B


def test_noalloc_graph_replay_then_eager(lib):
    """A call captured into a CUDA graph at B = 32, an eager call at B = 16, the graph replayed,
    then another eager call at B = 16: every result matches pfsoft_cuda_dsoft (the replay rewrites
    the shared tables, so later calls rebuild theirs)."""
    g32, g16 = _grid(32, 5), _grid(16, 6)
    ref32, ref16 = _dsoft(lib, "dsoft", g32, 32), _dsoft(lib, "dsoft", g16, 16)
    d32 = torch.from_numpy(g32).cuda()
    o32 = torch.empty(orc.coef_count(32), dtype=torch.complex128, device="cuda")
    _dsoft(lib, "noalloc", g32, 32)   # first call on the device: symbol address, outside the capture
    side = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.stream(side):
        with torch.cuda.graph(graph, stream=side):
            assert lib.pfsoft_cuda_dsoft_noalloc(d32.data_ptr(), 32, o32.data_ptr(), side.cuda_stream) == 0
    assert orc.rel_l2(_dsoft(lib, "noalloc", g16, 16), ref16) <= REL_TOL
    o32.fill_(complex(np.nan, np.nan))
    graph.replay()
    torch.cuda.synchronize()
    assert orc.rel_l2(o32.cpu().numpy(), ref32) <= REL_TOL
    assert orc.rel_l2(_dsoft(lib, "noalloc", g16, 16), ref16) <= REL_TOL


def test_noalloc_repeat_same_bandwidth(lib):
    grid = _grid(32, 3)
    a = _dsoft(lib, "noalloc", grid, 32)
    b = _dsoft(lib, "noalloc", grid, 32)
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("B", [0, 33, 128])
def test_noalloc_rejects_sizes_beyond_the_limit(lib, B):
    assert lib.pfsoft_cuda_dsoft_noalloc(16, B, 16, None) == 1   # PFSOFT_EINVAL
    assert b"bandwidth must be in [1, 32]" in lib.pfsoft_last_error()
