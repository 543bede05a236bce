// Test infrastructure (oracle): a project-written FFT that stands in for FFTW 3.3.4 behind
// the two C symbols the reference declares in include/PFSOFTlib_headers/fftw_wrapper.hpp:31-32.
// FFTW is a third-party dependency of the reference (README.md:9; located by
// cmake_aux/PFSOFTlib_FindFFTW.cmake:34-35). It is not vendored and not installed in this
// image, so the compiled reference links this file instead of src/fftw_wrapper.cpp.
//
// Semantics kept from src/fftw_wrapper.cpp:47-173:
//   * every layer of `lays` is an independent, in-place, UNNORMALISED 2D DFT of size
//     cols x rows, rows being the contiguous (fastest) index (fftw_plan_dft_2d(cols, rows, ..));
//   * DFT2 uses exp(-2*pi*i*jk/n) (FFTW_FORWARD), IDFT2 uses exp(+2*pi*i*jk/n) (FFTW_BACKWARD);
//   * layers run in an OpenMP parallel loop with `threads` threads (fftw_wrapper.cpp:70,134).
// Algorithm: mixed-radix Stockham autosort (radices 4, 2, 3, 5 and a direct DFT for any other
// prime), twiddles evaluated in long double and rounded once. The column pass treats each
// row of the layer as one vector element, so every access is contiguous.
// Accuracy is pinned against numpy.fft (pocketfft) in tests/test_oracle.py.

#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

typedef std::complex<double> cplx;

struct Stage {
    int radix;
    int ns;                       // product of the radices of the previous stages
    std::vector<cplx> twiddle;    // twiddle[k*radix + r] = w^(r*k), w = exp(sign*2*pi*i/(ns*radix))
    std::vector<cplx> roots;      // roots[q*radix + r] = exp(sign*2*pi*i*r*q/radix)
};

struct Plan {
    int n = 0;
    int sign = -1;
    std::vector<Stage> stages;
};

std::vector<int> factorize(int n)
{
    std::vector<int> r;
    while (n % 4 == 0) { r.push_back(4); n /= 4; }
    while (n % 2 == 0) { r.push_back(2); n /= 2; }
    for (int p = 3; n > 1; p += 2) {
        while (n % p == 0) { r.push_back(p); n /= p; }
    }
    return r;
}

cplx unit_root(long long num, long long den, int sign)
{
    // exp(sign * 2*pi*i * num/den), evaluated in long double
    const long double two_pi = 6.283185307179586476925286766559005768L;
    long long m = num % den;
    if (m < 0) m += den;
    long double a = two_pi * (long double)m / (long double)den;
    return cplx((double)cosl(a), (double)(sign * sinl(a)));
}

Plan make_plan(int n, int sign)
{
    Plan p;
    p.n = n;
    p.sign = sign;
    int ns = 1;
    for (int R : factorize(n)) {
        Stage s;
        s.radix = R;
        s.ns = ns;
        s.twiddle.resize((size_t)ns * R);
        for (int k = 0; k < ns; ++k)
            for (int r = 0; r < R; ++r)
                s.twiddle[(size_t)k * R + r] = unit_root((long long)r * k, (long long)ns * R, sign);
        s.roots.resize((size_t)R * R);
        for (int q = 0; q < R; ++q)
            for (int r = 0; r < R; ++r)
                s.roots[(size_t)q * R + r] = unit_root((long long)r * q, R, sign);
        p.stages.push_back(s);
        ns *= R;
    }
    return p;
}

// One Stockham stage over n elements, each element being `vec` consecutive complex values.
void stage_apply(const Stage& s, int n, int vec, int sign, const cplx* in, cplx* out, cplx* v)
{
    const int R = s.radix, ns = s.ns, m = n / R;
    for (int j = 0; j < m; ++j) {
        const int k = j % ns;
        const cplx* tw = &s.twiddle[(size_t)k * R];
        const size_t obase = (size_t)(j / ns) * ns * R + k;
        for (int e = 0; e < vec; ++e) {
            for (int r = 0; r < R; ++r) v[r] = in[((size_t)j + (size_t)r * m) * vec + e] * tw[r];
            if (R == 2) {
                cplx a = v[0], b = v[1];
                out[(obase) * vec + e] = a + b;
                out[(obase + ns) * vec + e] = a - b;
            } else if (R == 4) {
                cplx a0 = v[0] + v[2], a1 = v[0] - v[2];
                cplx b0 = v[1] + v[3], b1 = v[1] - v[3];
                // multiply b1 by sign*i
                cplx b1r = (sign < 0) ? cplx(b1.imag(), -b1.real()) : cplx(-b1.imag(), b1.real());
                out[(obase) * vec + e] = a0 + b0;
                out[(obase + ns) * vec + e] = a1 + b1r;
                out[(obase + 2 * (size_t)ns) * vec + e] = a0 - b0;
                out[(obase + 3 * (size_t)ns) * vec + e] = a1 - b1r;
            } else {
                for (int q = 0; q < R; ++q) {
                    cplx acc = v[0];
                    const cplx* rt = &s.roots[(size_t)q * R];
                    for (int r = 1; r < R; ++r) acc += v[r] * rt[r];
                    out[(obase + (size_t)q * ns) * vec + e] = acc;
                }
            }
        }
    }
}

// In-place transform of n elements of `vec` complex values each; tmp holds n*vec values.
void transform(const Plan& p, int vec, cplx* data, cplx* tmp, cplx* v)
{
    cplx* a = data;
    cplx* b = tmp;
    for (const Stage& s : p.stages) {
        stage_apply(s, p.n, vec, p.sign, a, b, v);
        std::swap(a, b);
    }
    if (a != data) std::memcpy(data, a, sizeof(cplx) * (size_t)p.n * vec);
}

void layer_wise(int cols, int rows, int lays, double* arr, int threads, int sign)
{
    Plan prow = make_plan(rows, sign);
    Plan pcol = make_plan(cols, sign);
    int maxr = 1;
    for (const Stage& s : prow.stages) maxr = s.radix > maxr ? s.radix : maxr;
    for (const Stage& s : pcol.stages) maxr = s.radix > maxr ? s.radix : maxr;
    const size_t layer = (size_t)rows * cols;
    if (threads < 1) threads = 1;
#pragma omp parallel num_threads(threads)
    {
        std::vector<cplx> tmp(layer);
        std::vector<cplx> v(maxr);
#pragma omp for schedule(dynamic)
        for (int i = 0; i < lays; ++i) {
            cplx* x = reinterpret_cast<cplx*>(arr) + (size_t)i * layer;
            for (int c = 0; c < cols; ++c) transform(prow, 1, x + (size_t)c * rows, tmp.data(), v.data());
            transform(pcol, rows, x, tmp.data(), v.data());
        }
    }
}

}  // namespace

extern "C" {

void uzl_fftw_layer_wise_DFT2_grid3D(int cols, int rows, int lays, double* arr, int threads)
{
    layer_wise(cols, rows, lays, arr, threads, -1);
}

void uzl_fftw_layer_wise_IDFT2_grid3D(int cols, int rows, int lays, double* arr, int threads)
{
    layer_wise(cols, rows, lays, arr, threads, +1);
}

}
