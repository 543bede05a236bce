"""CPU tests of the Python mirror of the reference interface (no GPU work is issued)."""
import numpy as np
import pytest

from oracle import oracle as orc
from pfsoftlib_b200 import DSOFTFourierCoefficients, FourierTransforms, coef_count, coef_index, grid3D


def test_coef_index_matches_oracle_layout():
    for l in range(6):
        for M in range(-l, l + 1):
            for Mp in range(-l, l + 1):
                assert coef_index(l, M, Mp) == int(orc.coef_index(l, M, Mp))
    assert coef_count(16) == 5456


def test_coefficient_container_indexing():
    fc = DSOFTFourierCoefficients(4)
    fc[3, -2, 1] = 1 + 2j
    assert fc(3, -2, 1) == 1 + 2j
    assert fc.mem[coef_index(3, -2, 1)] == 1 + 2j
    with pytest.raises(IndexError):
        fc[2, 3, 0] = 1.0
    with pytest.raises(IndexError):
        fc(4, 0, 0)


def test_grid_indexing_matches_reference_layout():
    g = grid3D(4)
    g[1, 2, 3] = 5.0
    # grid3D_cx.hpp:293-303: mem[rows*cols*lay + cols*col + row]
    assert g.mem.reshape(-1)[16 * 3 + 4 * 2 + 1] == 5.0
    assert g(1, 2, 3) == 5.0


def test_dsoft_warns_and_returns_on_bad_shapes(capsys):
    fc = DSOFTFourierCoefficients(4)
    fc.mem[:] = 7
    FourierTransforms.DSOFT(grid3D(8, 8, 6), fc)
    FourierTransforms.DSOFT(grid3D(7), fc)
    FourierTransforms.DSOFT(grid3D(6), fc)
    err = capsys.readouterr().err
    assert "dimensions should be equal" in err
    assert "not even" in err
    assert "does not match" in err
    assert np.all(fc.mem == 7)


def test_idsoft_warns_and_returns_on_bad_shapes(capsys):
    fc = DSOFTFourierCoefficients(3)
    g = grid3D(8)
    g.mem[:] = 3
    FourierTransforms.IDSOFT(fc, g)
    assert "does not match" in capsys.readouterr().err
    assert np.all(g.mem == 3)
