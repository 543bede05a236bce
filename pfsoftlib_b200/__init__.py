"""pfsoftlib_b200 -- a B200-native SO(3) Fourier transform engine (DSOFT / iDSOFT).

The transforms run in hand-written sm_100a CUDA kernels behind a C ABI
(include/pfsoft_b200.h, ``libpfsoft_b200.so``). This package is the Python mirror of
PFSOFTlib's interface for that path: ``grid3D``, ``DSOFTFourierCoefficients``,
``FourierTransforms.DSOFT/IDSOFT`` and the ``DWT`` helpers; ``BatchPlan`` (many transforms in one
execution) and ``serving.TransformServer`` (requests with continuous batching) go beyond it.
"""
from ._lib import PfsoftError, load  # noqa: F401
from .batch import BatchPlan, split_supported  # noqa: F401
from .transforms import (  # noqa: F401
    DSOFTFourierCoefficients,
    DWT,
    FourierTransforms,
    coef_count,
    coef_index,
    grid3D,
)

__all__ = ["grid3D", "DSOFTFourierCoefficients", "FourierTransforms", "DWT", "PfsoftError", "load",
           "coef_count", "coef_index", "BatchPlan", "split_supported"]
