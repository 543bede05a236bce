"""CPU tests of the autotuner's decision rule and cache."""
from pfsoftlib_b200 import autotune


def test_choose_fastest_and_break_ties_low():
    assert autotune.choose({1: 3.0, 2: 2.0, 4: 2.5}) == 2
    assert autotune.choose({1: 2.0, 2: 2.0, 4: 2.0}) == 1


def test_key_is_order_free():
    assert autotune.key_for("B200", [32, 64, 32]) == autotune.key_for("B200", [64, 32, 32])


def test_cache_roundtrip(tmp_path):
    p = str(tmp_path / "t.json")
    autotune.store("k", 4, p)
    autotune.store("j", 2, p)
    assert autotune.load_cache(p) == {"k": 4, "j": 2}


class _FakeLib:
    def __init__(self):
        self.calls = []

    def pfsoft_tune_fft_fused(self, b, on):
        self.calls.append(("fft", b, on))
        return 0

    def pfsoft_tune_split_bandwidth(self, b, on):
        self.calls.append(("split", b, on))
        return 0


def test_apply_sets_per_bandwidth_knobs():
    lib = _FakeLib()
    autotune.apply(lib, {"fft_fused": {"64": True, "96": False}, "split": {"128": True}})
    assert ("fft", 64, 1) in lib.calls and ("fft", 96, 0) in lib.calls and ("split", 128, 1) in lib.calls
