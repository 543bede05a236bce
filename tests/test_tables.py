"""CPU check of the per-bandwidth recurrence-coefficient table's layout (tests/cpp/rc_table.cpp):
the closed-form class offsets that the DWT kernels use agree with the running sum over the
classes in their order, for B = 1..512."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "pfsoftlib_b200", "csrc")


def _cuda_include():
    for d in (os.environ.get("CUDA_HOME", ""), "/usr/local/cuda"):
        if d and os.path.exists(os.path.join(d, "include", "cuda_runtime.h")):
            return os.path.join(d, "include")
    pytest.skip("cuda_runtime.h not found")


def test_rc_table_offsets(tmp_path):
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    exe = str(tmp_path / "rc_table")
    subprocess.run([cxx, "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", CSRC, "-I", _cuda_include(),
                    os.path.join(ROOT, "tests", "cpp", "rc_table.cpp"), "-o", exe],
                   check=True, capture_output=True, text=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == "ok"
