"""Device coefficient generator (pfsoft_cuda_random_coeffs) against a numpy restatement of its
definition: SplitMix64 (Steele, Lea, Flood, OOPSLA 2014) on the counter, value i of the packed
vector a function of (seed, i) only, filling the storage of the reference's rand(fc)
(include/PFSOFTlib_headers/random.hpp:80-117) with a reproducible stream.

kind 0 (uniform re, im) is bit-exact; kinds 1 and 2 go through pow / log / sqrt / sincospi, which
the device and numpy round differently in the last bits, so they are compared to 1e-13 relative,
and their distributions are checked (magnitude law per degree, uniform phase)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(x):
    x = np.asarray(x, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = x + np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def unit(x):
    return (x >> np.uint64(11)).astype(np.float64) * 2.0 ** -53


def degrees(n):
    l = np.zeros(n, dtype=np.int64)
    B = 1
    while B * (4 * B * B - 1) // 3 < n:
        B += 1
    for d in range(B):
        lo, hi = d * (4 * d * d - 1) // 3, (d + 1) * (4 * (d + 1) ** 2 - 1) // 3
        l[lo:min(hi, n)] = d
    return l


def restated(B, seed, kind, power):
    n = B * (4 * B * B - 1) // 3
    i = np.arange(n, dtype=np.uint64)
    base = splitmix64(np.uint64(seed))
    r0 = splitmix64(base ^ (np.uint64(2) * i))
    r1 = splitmix64(base ^ (np.uint64(2) * i + np.uint64(1)))
    if kind == 0:
        return (2.0 * unit(r0) - 1.0) + 1j * (2.0 * unit(r1) - 1.0)
    l = degrees(n)
    mag = (1.0 + l) ** (-power)
    if kind == 1:
        r2 = splitmix64(base ^ (np.uint64(0x8000000000000000) | i))
        u = 1.0 - unit(r2)
        mag = mag * np.abs(np.sqrt(-2.0 * np.log(u)) * np.cos(np.pi * 2.0 * unit(r0)))
    ph = np.pi * 2.0 * unit(r1)
    return mag * np.cos(ph) + 1j * mag * np.sin(ph)


def _device(lib, B, seed, kind, power):
    import torch
    c = torch.empty(B * (4 * B * B - 1) // 3, dtype=torch.complex128, device="cuda")
    assert lib.pfsoft_cuda_random_coeffs(c.data_ptr(), B, seed, kind, power, torch.cuda.current_stream().cuda_stream) == 0
    return c.cpu().numpy()


@pytest.mark.parametrize("B,seed", [(1, 0), (7, 3), (32, 12345), (64, 2 ** 63 + 11)])
def test_kind0_bit_exact(lib, B, seed):
    np.testing.assert_array_equal(_device(lib, B, seed, 0, 0.0), restated(B, seed, 0, 0.0))


@pytest.mark.parametrize("kind,power", [(1, 1.0), (2, 1.5), (2, 2.0)])
def test_kinds_1_2_match_definition(lib, kind, power):
    B, seed = 48, 2024
    d = _device(lib, B, seed, kind, power)
    r = restated(B, seed, kind, power)
    assert np.max(np.abs(d - r)) <= 1e-13 * np.max(np.abs(r))


def test_distributions(lib):
    B = 96
    # kind 2: |f| exactly (1+l)^-p, phase uniform
    d = _device(lib, B, 7, 2, 1.5)
    l = degrees(d.size)
    np.testing.assert_allclose(np.abs(d), (1.0 + l) ** -1.5, rtol=1e-13)
    ph = np.angle(d)
    hist, _ = np.histogram(ph, bins=16, range=(-np.pi, np.pi))
    assert hist.min() > 0.9 * d.size / 16 and hist.max() < 1.1 * d.size / 16
    # kind 1: |f| (1+l)^p is |N(0,1)|: mean sqrt(2/pi), second moment 1
    d = _device(lib, B, 8, 1, 1.0)
    z = np.abs(d) * (1.0 + degrees(d.size))
    assert abs(z.mean() - np.sqrt(2 / np.pi)) < 0.01 and abs((z * z).mean() - 1.0) < 0.02
    # kind 0: re, im uniform on [-1, 1)
    d = _device(lib, B, 9, 0, 0.0)
    for x in (d.real, d.imag):
        assert x.min() >= -1.0 and x.max() < 1.0 and abs(x.mean()) < 0.01 and abs((x * x).mean() - 1 / 3) < 0.01


def test_seeds_differ_and_repeat(lib):
    a = _device(lib, 16, 1, 0, 0.0)
    assert np.array_equal(a, _device(lib, 16, 1, 0, 0.0))
    assert not np.array_equal(a, _device(lib, 16, 2, 0, 0.0))
    # the packed layout is degree-major: a smaller bandwidth is a prefix of the same stream
    assert np.array_equal(_device(lib, 8, 1, 0, 0.0), a[: 8 * (4 * 64 - 1) // 3])
