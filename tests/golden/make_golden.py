"""Regenerates the golden fixtures in this folder from the reference itself.

Run in a container that has the reference sources (the oracle Makefile compiles them into
oracle/_ref/libpfsoft_ref.so):

    python tests/golden/make_golden.py [--ref /path/to/PFSOFTlib]

For each bandwidth B in (2, 4, 8, 16) it stores ``ref_B{B}.npz`` with
  coeffs_in   seeded input coefficients (U[-1,1] re/im, PCG64 seed = B, reference fill order)
  grid        the reference IDSOFT of coeffs_in on a fresh (zero) grid, shape (2B,2B,2B)
  coeffs_out  the reference DSOFT of ``grid``
  weights     the reference quadrature weights w_B(j), j < 2B
  wigner_*    reference Wigner d-matrices (weighted and plain) for a few order pairs
All values come from the reference's own code paths (src/fn_idsoft.cpp, src/fn_dsoft.cpp,
include/PFSOFTlib_headers/fn_dwt.hpp); FFTW's two entry points are served by the project FFT
(oracle/fft_standin.cpp) because FFTW is not installed.
"""
import argparse
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as orc  # noqa: E402

PAIRS = [(0, 0), (1, 0), (1, 1), (2, -1), (-3, 2), (3, 3)]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="the reference project's source tree")
    a = ap.parse_args()
    orc.build(a.ref)
    ref = orc.Reference()
    here = os.path.dirname(os.path.abspath(__file__))
    for B in (2, 4, 8, 16):
        c = orc.coeffs_uniform(B, seed=B)
        g = ref.idsoft(c, B, threads=1)
        f = ref.dsoft(g, threads=1)
        extra = {}
        for (M, Mp) in PAIRS:
            if max(abs(M), abs(Mp)) < B:
                extra[f"wigner_{M}_{Mp}"] = ref.wigner_d(B, M, Mp, weighted=False)
                extra[f"wwigner_{M}_{Mp}"] = ref.wigner_d(B, M, Mp, weighted=True)
        np.savez_compressed(os.path.join(here, f"ref_B{B}.npz"), B=B, coeffs_in=c, grid=g,
                            coeffs_out=f, weights=ref.weights(B), **extra)
        print(B, "round-trip max abs", float(np.abs(f - c).max()))


if __name__ == "__main__":
    main()
