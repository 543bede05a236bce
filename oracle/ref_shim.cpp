// Test infrastructure (oracle): a C wrapper around the UNMODIFIED reference C++ API, compiled
// together with the reference's own sources into oracle/_ref/libpfsoft_ref.so by
// oracle/Makefile. Nothing here re-implements the reference; every call goes to
//   pfsoft::FourierTransforms::DSOFT   (src/fn_dsoft.cpp:76)
//   pfsoft::FourierTransforms::IDSOFT  (src/fn_idsoft.cpp:72)
//   pfsoft::DWT::quadrature_weights / weighted_wigner_d_matrix / wigner_d_matrix
//                                      (include/PFSOFTlib_headers/fn_dwt.hpp:64,107,239)
// Data cross this boundary in the packed layouts used throughout this project:
//   grid    : N*N*N interleaved complex128, element (row, col, lay) at (lay*N + col)*N + row
//             (grid3D_cx.hpp:293-303), N = 2B;
//   coeffs  : degree l occupies l(4l^2-1)/3 .. (l+1)(4(l+1)^2-1)/3, column-major
//             (2l+1)x(2l+1) with negative orders wrapped to 2l+1+M
//             (dsoft_fourier_coefficients.cpp:80-89, matrix_cx.hpp:481-484).
// The timed entry points (ref_ctx_*) time only the reference call itself, including the
// by-value grid copy that DSOFT makes, as benchmark/benchmark_dsoft_for.cpp:157-186 does.

#include <pfsoft>

#include <chrono>
#include <cstring>

using namespace pfsoft;

namespace {

size_t coef_offset(int l) { return (size_t)l * (4 * (size_t)l * l - 1) / 3; }

struct RefCtx {
    int B;
    grid3D<complex<double> > grid;
    DSOFTFourierCoefficients fc;
    explicit RefCtx(int b) : B(b), grid((size_t)(2 * b)), fc(b) {}
};

void grid_from(grid3D<complex<double> >& g, const double* src)
{
    std::memcpy(const_cast<complex<double>*>(g.mem), src, sizeof(complex<double>) * g.rows * g.cols * g.lays);
}

void grid_to(const grid3D<complex<double> >& g, double* dst)
{
    std::memcpy(dst, g.mem, sizeof(complex<double>) * g.rows * g.cols * g.lays);
}

void coeffs_from(DSOFTFourierCoefficients& fc, const double* src)
{
    for (int l = 0; l < fc.bandwidth; ++l) {
        const int L = 2 * l + 1;
        const double* base = src + 2 * coef_offset(l);
        for (int M = -l; M <= l; ++M)
            for (int Mp = -l; Mp <= l; ++Mp) {
                const size_t i = (size_t)(Mp >= 0 ? Mp : L + Mp) * L + (M >= 0 ? M : L + M);
                fc(l, M, Mp) = complex<double>(base[2 * i], base[2 * i + 1]);
            }
    }
}

void coeffs_to(const DSOFTFourierCoefficients& fc, double* dst)
{
    for (int l = 0; l < fc.bandwidth; ++l) {
        const int L = 2 * l + 1;
        double* base = dst + 2 * coef_offset(l);
        for (int M = -l; M <= l; ++M)
            for (int Mp = -l; Mp <= l; ++Mp) {
                const size_t i = (size_t)(Mp >= 0 ? Mp : L + Mp) * L + (M >= 0 ? M : L + M);
                const complex<double>& v = fc(l, M, Mp);
                base[2 * i] = v.re;
                base[2 * i + 1] = v.im;
            }
    }
}

}  // namespace

extern "C" {

int ref_max_threads(void) { return PFSOFT_MAX_THREADS; }

// DSOFT on a host grid (not modified), result written to packed coefficients.
void ref_dsoft(const double* grid, int B, double* coeffs, int threads)
{
    grid3D<complex<double> > g((size_t)(2 * B));
    grid_from(g, grid);
    DSOFTFourierCoefficients fc(B);
    FourierTransforms::DSOFT(g, fc, threads);
    coeffs_to(fc, coeffs);
}

// IDSOFT from packed coefficients into a FRESH zero-initialised grid (grid3D(2B) zero-fills,
// complex.hpp:117-120), so the Nyquist columns that IDSOFT never writes stay zero.
void ref_idsoft(const double* coeffs, int B, double* grid, int threads)
{
    DSOFTFourierCoefficients fc(B);
    coeffs_from(fc, coeffs);
    grid3D<complex<double> > g((size_t)(2 * B));
    FourierTransforms::IDSOFT(fc, g, threads);
    grid_to(g, grid);
}

// Quadrature weights w_B(j), j < 2B, computed in long double and rounded to double.
void ref_quadrature_weights(int B, double* w)
{
    vector<long double> v(2 * B);
    DWT::quadrature_weights<long double>(v);
    for (int j = 0; j < 2 * B; ++j) w[j] = (double)v[j];
}

// Wigner d-matrix rows l = J..B-1 (J = max(|M|,|M'|)) times 2B columns, written row-major
// out[(l-J)*2B + k], rounded from long double. weighted != 0 folds in the quadrature weights.
void ref_wigner_d_matrix(int B, int M, int Mp, int weighted, double* out)
{
    const int J = std::max(std::abs(M), std::abs(Mp));
    matrix<long double> d(B - J, 2 * B);
    if (weighted) {
        vector<long double> v(2 * B);
        DWT::quadrature_weights<long double>(v);
        DWT::weighted_wigner_d_matrix(d, B, M, Mp, v);
    } else {
        DWT::wigner_d_matrix<long double>(d, B, M, Mp);
    }
    for (int i = 0; i < B - J; ++i)
        for (int k = 0; k < 2 * B; ++k) out[(size_t)i * 2 * B + k] = (double)d(i, k);
}

// Persistent contexts for timing: the containers are built once, each call times only the
// reference transform.
void* ref_ctx_create(int B) { return new RefCtx(B); }
void ref_ctx_destroy(void* c) { delete static_cast<RefCtx*>(c); }
void ref_ctx_set_grid(void* c, const double* g) { grid_from(static_cast<RefCtx*>(c)->grid, g); }
void ref_ctx_get_grid(void* c, double* g) { grid_to(static_cast<RefCtx*>(c)->grid, g); }
void ref_ctx_set_coeffs(void* c, const double* x) { coeffs_from(static_cast<RefCtx*>(c)->fc, x); }
void ref_ctx_get_coeffs(void* c, double* x) { coeffs_to(static_cast<RefCtx*>(c)->fc, x); }

double ref_ctx_dsoft(void* c, int threads)
{
    RefCtx* r = static_cast<RefCtx*>(c);
    auto t0 = std::chrono::steady_clock::now();
    FourierTransforms::DSOFT(r->grid, r->fc, threads);
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

double ref_ctx_idsoft(void* c, int threads)
{
    RefCtx* r = static_cast<RefCtx*>(c);
    auto t0 = std::chrono::steady_clock::now();
    FourierTransforms::IDSOFT(r->fc, r->grid, threads);
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

}
