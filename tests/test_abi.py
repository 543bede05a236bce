"""CPU tests of the C ABI boundary: the library loads, exports every function declared in
include/pfsoft_b200.h, and rejects bad arguments before touching the GPU."""
import os
import re

import pytest

from pfsoftlib_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(pfsoft_\w+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "pfsoft_cuda_dsoft" in names and "pfsoft_cuda_idsoft" in names
    assert len(names) >= 14


def test_every_declared_symbol_is_exported(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_table_covers_header():
    assert set(declared_functions()) <= set(_lib.SIGNATURES)


def test_sizes(lib):
    assert lib.pfsoft_coef_count(16) == 5456
    assert lib.pfsoft_coef_count(128) == 2796160
    assert lib.pfsoft_grid_bytes(128) == 256 ** 3 * 16
    assert lib.pfsoft_workspace_bytes(128) >= lib.pfsoft_grid_bytes(128)
    assert lib.pfsoft_coef_count(0) == 0


@pytest.mark.parametrize("B", [0, -3, 513])
def test_bad_bandwidth_is_einval(lib, B):
    assert lib.pfsoft_cuda_dsoft(1, B, 1, None, 0, None) == _lib.PFSOFT_EINVAL
    assert lib.pfsoft_cuda_idsoft(1, B, 1, None, 0, None) == _lib.PFSOFT_EINVAL
    assert lib.pfsoft_dsoft_host(1, B, 1) == _lib.PFSOFT_EINVAL
    assert b"bandwidth" in lib.pfsoft_last_error()


def test_null_pointers_are_einval(lib):
    assert lib.pfsoft_cuda_dsoft(None, 8, 1, None, 0, None) == _lib.PFSOFT_EINVAL
    assert lib.pfsoft_cuda_idsoft(1, 8, None, None, 0, None) == _lib.PFSOFT_EINVAL
    assert lib.pfsoft_dsoft_host(None, 8, None) == _lib.PFSOFT_EINVAL


def test_small_workspace_is_einval(lib):
    assert lib.pfsoft_cuda_dsoft(16, 8, 16, 16, 100, None) == _lib.PFSOFT_EINVAL
    assert b"workspace" in lib.pfsoft_last_error()


def test_wigner_orders_checked(lib):
    assert lib.pfsoft_cuda_wigner_d_matrix(8, 8, 0, 0, 16, None) == _lib.PFSOFT_EINVAL
    assert lib.pfsoft_cuda_layer_wise_dft2(0, 4, 4, 16, 1.0, None) == _lib.PFSOFT_EINVAL


def test_status_strings(lib):
    assert lib.pfsoft_status_string(0) == b"ok"
    assert lib.pfsoft_status_string(_lib.PFSOFT_ENOMEM) == b"out of memory"
