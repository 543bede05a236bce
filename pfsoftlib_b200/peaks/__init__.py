"""Measured FP64 peaks of the current GPU (the DWT kernels' roofline denominator).

``python -m pfsoftlib_b200.peaks`` builds fp64_peak.cu with nvcc for sm_100a and runs it."""
