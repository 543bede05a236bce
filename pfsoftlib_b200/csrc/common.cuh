// Shared device helpers for the SO(3) Fourier transform kernels (sm_100a).
//
// Data layouts in HBM (N = 2B, all complex values interleaved {re, im} doubles = double2):
//   grid     G[k][c][r]   element (row r, col c, layer k) at (k*N + c)*N + r, exactly the
//                         reference grid3D layout (include/PFSOFTlib_headers/grid3D_cx.hpp:293-303);
//                         r is the gamma index (order M'), c the alpha index (order M), k = beta_k.
//   spectrum X[r][c][k]   the layer-wise 2D DFT with beta innermost: bin (row r, col c) of layer k
//                         at (r*N + c)*N + k. One (r, c) "beta column" is N contiguous values,
//                         which is what the discrete Wigner transform reads and writes.
//   coeffs   packed       degree l at l(4l^2-1)/3, column-major (2l+1)^2 block, negative orders
//                         wrapped to 2l+1+M (src/dsoft_fourier_coefficients.cpp:80-89).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace pfsoft_dev {

__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// multiply by sign*i: sign = -1 gives -i*a, +1 gives i*a
template <int SIGN>
__host__ __device__ __forceinline__ double2 cmul_i(double2 a)
{
    return SIGN < 0 ? make_double2(a.y, -a.x) : make_double2(-a.y, a.x);
}

__host__ __device__ __forceinline__ size_t coef_offset(int l) { return (size_t)l * (4 * (size_t)l * l - 1) / 3; }

// packed index of f^l_{m1,m2}
__host__ __device__ __forceinline__ size_t coef_index(int l, int m1, int m2)
{
    const int L = 2 * l + 1;
    const int i1 = m1 >= 0 ? m1 : L + m1;
    const int i2 = m2 >= 0 ? m2 : L + m2;
    return coef_offset(l) + (size_t)i2 * L + i1;
}

// Order-pair classes (M, M'), M >= M' >= 0, enumerated by M ascending then M' ascending:
// class i has M = floor((sqrt(8i+1)-1)/2), M' = i - M(M+1)/2. Ascending M is descending work
// (B - M degrees), i.e. longest-first order for the schedulers.
__host__ __device__ __forceinline__ void class_orders(int i, int& M, int& Mp)
{
    int m = (int)((sqrtf(8.0f * (float)i + 1.0f) - 1.0f) * 0.5f);   // corrected below: exact for any i
    while (m * (m + 1) / 2 > i) --m;
    while ((m + 1) * (m + 2) / 2 <= i) ++m;
    M = m;
    Mp = i - m * (m + 1) / 2;
}

__host__ __device__ __forceinline__ int num_classes(int B) { return B * (B + 1) / 2; }

// The coefficients served by one Wigner matrix d_{M,M'} (the reference's 8-fold symmetry,
// src/fn_dsoft.cpp:137-283): up to 8 distinct (m1, m2). For each:
//   FFT bin       row = m2 mod N, col = m1 mod N
//   beta reversal rev = (m1 < 0) xor (m2 < 0)     (d read at pi - beta)
//   sign(l)       s0 * (rev ? (-1)^(l-M) : 1),  s0 = -1 * ((-1)^(M-M') if x else 1),
//                 x = (m1 < 0) if |m1| == M else (m2 > 0)
struct PairCase {
    int m1, m2;
    int row, col;
    int rev;
    double s0;
};

// Number of distinct coefficients class (M, M') serves: 1 for (0,0), 4 when M' = 0 or M' = M,
// otherwise 8.
__host__ __device__ __forceinline__ int class_case_count(int M, int Mp)
{
    return M == 0 ? 1 : ((Mp == 0 || Mp == M) ? 4 : 8);
}

// Case c (< class_case_count) of class (M, M'). The eight orientations, in this order, are
//   (M,M') (M',M) (-M,-M') (-M',-M) (M',-M) (M,-M') (-M',M) (-M,M');
// for M' = 0 the first four are distinct, for M' = M the even ones.
__host__ __device__ __forceinline__ PairCase class_case(int M, int Mp, int c, int N)
{
    const int e = (Mp == M && M > 0) ? 2 * c : c;
    int m1, m2;
    switch (e) {
        case 0: m1 = M; m2 = Mp; break;
        case 1: m1 = Mp; m2 = M; break;
        case 2: m1 = -M; m2 = -Mp; break;
        case 3: m1 = -Mp; m2 = -M; break;
        case 4: m1 = Mp; m2 = -M; break;
        case 5: m1 = M; m2 = -Mp; break;
        case 6: m1 = -Mp; m2 = M; break;
        default: m1 = -M; m2 = Mp; break;
    }
    PairCase p;
    p.m1 = m1;
    p.m2 = m2;
    p.row = m2 >= 0 ? m2 : N + m2;
    p.col = m1 >= 0 ? m1 : N + m1;
    p.rev = (m1 < 0) != (m2 < 0);
    const int a1 = m1 < 0 ? -m1 : m1;
    const bool x = (a1 == M) ? (m1 < 0) : (m2 > 0);
    p.s0 = (x && ((M - Mp) & 1)) ? 1.0 : -1.0;
    return p;
}

}  // namespace pfsoft_dev
