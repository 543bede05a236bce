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
