"""The C++ drop-in header (include/pfsoft_b200/pfsoft.hpp): compiles on CPU; on a GPU the
example-style round trip of the reference (examples/example.cpp:44-74) passes through it."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "roundtrip.cpp")
LIBDIR = os.path.join(ROOT, "pfsoftlib_b200")


def _cxx():
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")


def _build(out, src=SRC):
    import pfsoftlib_b200

    pfsoftlib_b200.load()   # builds libpfsoft_b200.so if needed
    cmd = [_cxx(), "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"), src, "-o", out,
           "-L", LIBDIR, "-lpfsoft_b200", f"-Wl,-rpath,{LIBDIR}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)


def test_header_compiles(tmp_path):
    _build(str(tmp_path / "roundtrip"))
    # the drop-in timing program the benchmark runs
    _build(str(tmp_path / "dropin_timing"), os.path.join(ROOT, "tests", "cpp", "dropin_timing.cpp"))


@pytest.mark.gpu
@pytest.mark.parametrize("B", [8, 16, 33])
def test_cpp_round_trip_on_gpu(tmp_path, B):
    exe = str(tmp_path / "roundtrip")
    _build(exe)
    r = subprocess.run([exe, str(B), "5"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Correct result:  Yes" in r.stdout
    assert "does not match" in r.stderr
