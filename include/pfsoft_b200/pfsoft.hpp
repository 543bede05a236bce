// pfsoft_b200/pfsoft.hpp -- C++ drop-in for PFSOFTlib's DSOFT / iDSOFT interface.
//
// Re-exposes the reference names used on this path, with the same index semantics and error
// behaviour, and runs every transform on the GPU through the C ABI (pfsoft_b200.h):
//
//   pfsoft::complex<T>                        include/PFSOFTlib_headers/complex.hpp:67-68 ({re, im})
//   pfsoft::grid3D<complex<double>>           include/PFSOFTlib_headers/grid3D_cx.hpp:47-83
//   pfsoft::DSOFTFourierCoefficients          include/PFSOFTlib_headers/dsoft_fourier_coefficients.hpp:50-72
//   pfsoft::FourierTransforms::DSOFT/IDSOFT   include/PFSOFTlib_headers/fn_fourier_transforms.hpp:75-78
//   operator<< of complex, grid3D, DSOFTFourierCoefficients
//                                             complex.hpp:596, grid3D_cx.hpp:429-523,
//                                             src/dsoft_fourier_coefficients.cpp:124-137
//
// Differences a caller can observe: DSOFT takes the sample by const reference (every call site
// of the by-value original still compiles, and the caller's grid is untouched either way);
// IDSOFT also writes the Nyquist bins (row or column order B), which the reference leaves as
// they were -- the values equal the reference's on a fresh grid. `threads` has no effect.
// Coefficient storage is one packed array (data()), degree l at l(4l^2-1)/3.
#ifndef PFSOFT_B200_PFSOFT_HPP
#define PFSOFT_B200_PFSOFT_HPP

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

#include "../pfsoft_b200.h"

namespace pfsoft {

// warn-and-return reporting of the reference (cmake_aux/compiler_config.hpp.in:112-120)
#define PFSOFT_B200_WARN(fn, msg) std::fprintf(stderr, "** [PFSOFTLib warning] %s(): %s **\n", fn, msg)

template <typename T>
struct complex {
    T re, im;
    complex() : re(0), im(0) {}
    complex(const T& r, const T& i) : re(r), im(i) {}
    explicit complex(const T& r) : re(r), im(0) {}
    complex operator+(const complex& o) const { return complex(re + o.re, im + o.im); }
    complex operator-(const complex& o) const { return complex(re - o.re, im - o.im); }
    complex operator*(const complex& o) const { return complex(re * o.re - im * o.im, re * o.im + im * o.re); }
    complex operator*(const T& s) const { return complex(re * s, im * s); }
    complex& operator+=(const complex& o) { re += o.re; im += o.im; return *this; }
    complex& operator*=(const complex& o) { *this = *this * o; return *this; }
    bool operator==(const complex& o) const { return re == o.re && im == o.im; }
    bool operator!=(const complex& o) const { return !(*this == o); }
};

template <typename T>
struct grid3D;

// Complex 3D sample grid; element (row, col, lay) at rows*cols*lay + cols*col + row.
template <typename T>
struct grid3D<complex<T> > {
    size_t rows, cols, lays;
    complex<T>* mem;

    grid3D() : rows(0), cols(0), lays(0), mem(nullptr) {}
    explicit grid3D(size_t rcl) : grid3D(rcl, rcl, rcl) {}
    grid3D(size_t r, size_t c, size_t l) : rows(r), cols(c), lays(l), mem(new complex<T>[r * c * l]) {}
    grid3D(size_t rcl, const complex<T>& initial) : grid3D(rcl) { std::fill(mem, mem + size(), initial); }
    grid3D(const grid3D& o) : grid3D(o.rows, o.cols, o.lays) { std::memcpy(mem, o.mem, sizeof(complex<T>) * size()); }
    grid3D(grid3D&& o) noexcept : rows(o.rows), cols(o.cols), lays(o.lays), mem(o.mem) { o.mem = nullptr; }
    grid3D& operator=(grid3D o)
    {
        std::swap(rows, o.rows);
        std::swap(cols, o.cols);
        std::swap(lays, o.lays);
        std::swap(mem, o.mem);
        return *this;
    }
    ~grid3D() { delete[] mem; }

    size_t size() const { return rows * cols * lays; }
    complex<T>& operator()(size_t row, size_t col, size_t lay) { return mem[rows * cols * lay + cols * col + row]; }
    const complex<T>& operator()(size_t row, size_t col, size_t lay) const { return mem[rows * cols * lay + cols * col + row]; }

    // grid3D_cx.hpp:309-427: in-place unnormalised 2D DFT of every layer, then * scale
    void layer_wise_DFT2(const complex<double>& scale = complex<double>(1, 0), int threads = 1) { layer_wise(scale, false); (void)threads; }
    void layer_wise_IDFT2(const complex<double>& scale = complex<double>(1, 0), int threads = 1) { layer_wise(scale, true); (void)threads; }

  private:
    void layer_wise(const complex<double>& scale, bool inverse)
    {
        static_assert(sizeof(complex<T>) == 2 * sizeof(double), "the GPU path transforms complex<double> grids");
        const double real = scale.im == 0 ? scale.re : 1.0;
        double* d = reinterpret_cast<double*>(mem);
        const int rc = inverse ? pfsoft_layer_wise_idft2_host((int)cols, (int)rows, (int)lays, d, real)
                               : pfsoft_layer_wise_dft2_host((int)cols, (int)rows, (int)lays, d, real);
        if (rc != PFSOFT_OK) {
            PFSOFT_B200_WARN("layer_wise_DFT2", pfsoft_last_error());
            return;
        }
        if (scale.im != 0)
            for (size_t i = 0; i < size(); ++i) mem[i] = mem[i] * complex<T>((T)scale.re, (T)scale.im);
    }
};

// Coefficients f^l_{M,M'}, 0 <= l < B, |M|, |M'| <= l (dsoft_fourier_coefficients.cpp:48-112).
struct DSOFTFourierCoefficients {
    const int bandwidth;

    DSOFTFourierCoefficients() : bandwidth(0) {}
    explicit DSOFTFourierCoefficients(int bandlimit)
        : bandwidth(bandlimit), mem_((size_t)pfsoft_coef_count(bandlimit))
    {
    }

    complex<double>& operator()(int l, int M, int Mp) { return mem_[index(l, M, Mp)]; }
    const complex<double>& operator()(int l, int M, int Mp) const { return mem_[index(l, M, Mp)]; }

    complex<double>* data() { return mem_.data(); }
    const complex<double>* data() const { return mem_.data(); }
    size_t size() const { return mem_.size(); }

  private:
    std::vector<complex<double> > mem_;

    size_t index(int l, int M, int Mp) const
    {
        if (M > l || Mp > l || M < -l || Mp < -l || l < 0 || l >= bandwidth) {
            // dsoft_fourier_coefficients.cpp:82 (pfsoft_cond_e): report and exit
            std::fprintf(stderr, "** [PFSOFTLib error]   operator()(): illegal parameter for DSOFTFourierCoefficients. "
                                 "Condition |M|,|Mp| <= l violated. **\n");
            std::exit(EXIT_FAILURE);
        }
        const size_t L = 2 * (size_t)l + 1;
        const size_t i1 = M >= 0 ? (size_t)M : L + M;
        const size_t i2 = Mp >= 0 ? (size_t)Mp : L + Mp;
        return (size_t)l * (4 * (size_t)l * l - 1) / 3 + i2 * L + i1;
    }
};

// ---- text output, in the reference's format ------------------------------------------------
namespace detail {

// Column layout of the reference's complex grid and matrix printers: width 20 in fixed
// notation; the LAST element (in print order) whose real or imaginary magnitude reaches 10, 100
// or 1000 sets the width to 22, 24 or 28, the last of these in scientific notation.
struct CellFormat {
    int width = 20;
    bool scientific = false;
    void see(double re, double im)
    {
        const double a = std::abs(re), b = std::abs(im);
        if (a >= 10 || b >= 10) {
            width = 22;
            scientific = false;
        }
        if (a >= 100 || b >= 100) {
            width = 24;
            scientific = false;
        }
        if (a >= 1000 || b >= 1000) {
            width = 28;
            scientific = true;
        }
    }
};

// "re + |im|i" with four decimals; a zero imaginary part prints as +0
inline std::string cell_text(double re, double im, bool scientific)
{
    std::ostringstream v;
    if (scientific)
        v << std::scientific;
    else
        v << std::fixed;
    v << std::setprecision(4) << re << (im < 0 ? " - " : " + ") << (im == 0 ? 0.0 : std::abs(im)) << "i";
    return v.str();
}

inline void put_cell(std::ostream& o, const CellFormat& f, double re, double im)
{
    o << std::setfill(' ') << std::right << std::setw(f.width) << cell_text(re, im, f.scientific);
}

}  // namespace detail

// complex.hpp:596: scientific, 4 digits; leaves the stream in fixed notation
template <typename T>
std::ostream& operator<<(std::ostream& o, const complex<T>& c)
{
    const std::ios::fmtflags saved = std::cout.flags();
    o << std::scientific << std::setprecision(4) << std::noshowpos << c.re << (c.im < 0 ? " - " : " + ")
      << (c.im == 0 ? 0 : std::abs(c.im)) << "i";
    std::cout.flags(saved);
    return o << std::fixed;
}

// grid3D_cx.hpp:429-523: a blank line, then per layer "layer[z]" and one row per grid row
template <typename T>
std::ostream& operator<<(std::ostream& o, const grid3D<complex<T> >& g)
{
    const std::ios::fmtflags saved = std::cout.flags();
    o << std::endl;
    detail::CellFormat f;
    for (size_t z = 0; z < g.lays; ++z)
        for (size_t x = 0; x < g.rows; ++x)
            for (size_t y = 0; y < g.cols; ++y) f.see((double)g(x, y, z).re, (double)g(x, y, z).im);
    for (size_t z = 0; z < g.lays; ++z) {
        o << "layer[" << z << "]" << std::endl;
        for (size_t x = 0; x < g.rows; ++x) {
            for (size_t y = 0; y < g.cols; ++y) detail::put_cell(o, f, (double)g(x, y, z).re, (double)g(x, y, z).im);
            o << std::endl;
        }
        o << std::endl;
    }
    std::cout.flags(saved);
    return o;
}

// src/dsoft_fourier_coefficients.cpp:124-137: per degree a title line and the (2l+1)^2 block,
// rows = order M, columns = order M' (0, 1, ..., l, -l, ..., -1), in the matrix format above
inline std::ostream& operator<<(std::ostream& o, const DSOFTFourierCoefficients& fc)
{
    const std::ios::fmtflags saved = std::cout.flags();
    o << std::endl << std::setprecision(4);
    for (int l = 0; l < fc.bandwidth; ++l) {
        o << "DSOFTFourierCoefficients[M_{0,1,2,...,-2,-1} x M'_{0,1,2,...,-2,-1}] ~> [l = " << l << "]" << std::endl;
        const size_t L = 2 * (size_t)l + 1, base = (size_t)l * (4 * (size_t)l * l - 1) / 3;
        const complex<double>* blk = fc.data() + base;   // column-major: (row i, column j) at j L + i
        detail::CellFormat f;
        o << std::endl;
        for (size_t i = 0; i < L; ++i)
            for (size_t j = 0; j < L; ++j) f.see(blk[j * L + i].re, blk[j * L + i].im);
        for (size_t i = 0; i < L; ++i) {
            for (size_t j = 0; j < L; ++j) detail::put_cell(o, f, blk[j * L + i].re, blk[j * L + i].im);
            o << std::endl;
        }
        o << std::endl;
    }
    std::cout.flags(saved);
    return o;
}

namespace FourierTransforms {

// src/fn_dsoft.cpp:76
inline void DSOFT(const grid3D<complex<double> >& sample, DSOFTFourierCoefficients& fc, int threads = 1)
{
    (void)threads;
    if (sample.rows != sample.cols || sample.rows != sample.lays) {
        PFSOFT_B200_WARN("DSOFT", "all DSOFT sample grid dimensions should be equal.");
        return;
    }
    if (sample.rows & 1) {
        PFSOFT_B200_WARN("DSOFT", "DSOFT sample grid dimensions are not even.");
        return;
    }
    const int bandwidth = (int)(sample.cols / 2);
    if (bandwidth != fc.bandwidth) {
        PFSOFT_B200_WARN("DSOFT", "DSOFT Fourier coefficients container bandwidth does not match to sample grid bandwidth.");
        return;
    }
    const int rc = pfsoft_dsoft_host(reinterpret_cast<const double*>(sample.mem), bandwidth, reinterpret_cast<double*>(fc.data()));
    if (rc != PFSOFT_OK) PFSOFT_B200_WARN("DSOFT", pfsoft_last_error());
}

// src/fn_idsoft.cpp:72
inline void IDSOFT(const DSOFTFourierCoefficients& fc, grid3D<complex<double> >& synthesis, int threads = 1)
{
    (void)threads;
    if (synthesis.rows != synthesis.cols || synthesis.rows != synthesis.lays) {
        PFSOFT_B200_WARN("IDSOFT", "all IDSOFT synthesis grid dimensions should be equal.");
        return;
    }
    if (synthesis.rows & 1) {
        PFSOFT_B200_WARN("IDSOFT", "IDSOFT synthesis grid dimensions are not even.");
        return;
    }
    const int bandwidth = (int)(synthesis.cols / 2);
    if (bandwidth != fc.bandwidth) {
        PFSOFT_B200_WARN("IDSOFT", "IDSOFT Fourier coefficients container bandwidth does not match to synthesis grid bandwidth.");
        return;
    }
    const int rc = pfsoft_idsoft_host(reinterpret_cast<const double*>(fc.data()), bandwidth, reinterpret_cast<double*>(synthesis.mem));
    if (rc != PFSOFT_OK) PFSOFT_B200_WARN("IDSOFT", pfsoft_last_error());
}

}  // namespace FourierTransforms

}  // namespace pfsoft

#undef PFSOFT_B200_WARN

#endif  // PFSOFT_B200_PFSOFT_HPP
