"""Text output of the grid and coefficient containers in the reference's format
(grid3D_cx.hpp:429-523, matrix_cx.hpp:545-620, dsoft_fourier_coefficients.cpp:124-137), against
tests/golden/formats_ref.txt, printed by the compiled reference (tests/golden/make_formats.py)."""
import os
import shutil
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = open(os.path.join(ROOT, "tests", "golden", "formats_ref.txt")).read()


def _val(a, b, c, salt):
    h = (a * 131 + b * 31 + c * 7 + salt * 17) % 23
    return (h - 11) * 0.3125 + (0.0 if h % 5 == 0 else 0.001 * h)


def test_cpp_header_prints_like_the_reference(tmp_path):
    import pfsoftlib_b200

    pfsoftlib_b200.load()
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    exe = str(tmp_path / "formats")
    lib = os.path.join(ROOT, "pfsoftlib_b200")
    subprocess.run([cxx, "-std=c++17", "-O1", "-Wall", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "formats.cpp"), "-o", exe, "-L", lib, "-lpfsoft_b200",
                    f"-Wl,-rpath,{lib}"], check=True, capture_output=True, text=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    assert out == REF


def test_python_containers_print_like_the_reference():
    from pfsoftlib_b200 import DSOFTFourierCoefficients, grid3D

    g = grid3D(2)
    for z in range(2):
        for x in range(2):
            for y in range(2):
                g[x, y, z] = complex(_val(x, y, z, 1), _val(x, y, z, 2))
    g[1, 0, 1] = 0j
    g[0, 1, 1] = complex(-0.5, -0.0)
    h = grid3D(2)
    for z in range(2):
        for x in range(2):
            for y in range(2):
                h[x, y, z] = complex(_val(x, y, z, 3), -_val(x, y, z, 4))
    h[0, 0, 0] = complex(12345.678, 1.0)
    h[1, 1, 1] = complex(-42.5, 3.0)
    text = str(g) + str(h)
    h[1, 1, 1] = complex(2.5, -1500.25)
    text += str(h)
    fc = DSOFTFourierCoefficients(3)
    for l in range(3):
        for M in range(-l, l + 1):
            for Mp in range(-l, l + 1):
                fc[l, M, Mp] = complex(_val(l, M + 3, Mp + 3, 5) * (l + 1), _val(l, M + 3, Mp + 3, 6))
    fc[2, -2, 1] = complex(150.0, -0.25)
    text += str(fc)
    assert text == REF[: REF.rindex("0.3333")]
    assert np.isfinite(fc.mem).all()
