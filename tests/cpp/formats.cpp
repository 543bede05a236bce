// Prints grids and coefficient containers with operator<< (grid3D_cx.hpp:429-523,
// dsoft_fourier_coefficients.cpp:124-137). Compiled against the drop-in header by
// tests/test_formats.py, and against the reference by tests/golden/make_formats.py, which
// writes the fixture the test compares with. The values exercise every column-width rule.
#ifdef USE_REFERENCE
#include <pfsoft>
#else
#include <pfsoft_b200/pfsoft.hpp>
#endif
#include <iostream>

using namespace pfsoft;

static double val(int a, int b, int c, int salt)
{
    const int h = (a * 131 + b * 31 + c * 7 + salt * 17) % 23;
    return (h - 11) * 0.3125 + (h % 5 == 0 ? 0.0 : 0.001 * h);
}

int main()
{
    // small values only: width 20, fixed
    grid3D<complex<double> > g(2);
    for (size_t z = 0; z < 2; ++z)
        for (size_t x = 0; x < 2; ++x)
            for (size_t y = 0; y < 2; ++y) g(x, y, z) = complex<double>(val(x, y, z, 1), val(x, y, z, 2));
    g(1, 0, 1) = complex<double>(0.0, 0.0);
    g(0, 1, 1) = complex<double>(-0.5, -0.0);
    std::cout << g;

    // a large value first, a moderate one last: the last one sets the width
    grid3D<complex<double> > h(2);
    for (size_t z = 0; z < 2; ++z)
        for (size_t x = 0; x < 2; ++x)
            for (size_t y = 0; y < 2; ++y) h(x, y, z) = complex<double>(val(x, y, z, 3), -val(x, y, z, 4));
    h(0, 0, 0) = complex<double>(12345.678, 1.0);
    h(1, 1, 1) = complex<double>(-42.5, 3.0);
    std::cout << h;

    // the largest last: scientific
    h(1, 1, 1) = complex<double>(2.5, -1500.25);
    std::cout << h;

    DSOFTFourierCoefficients fc(3);
    for (int l = 0; l < 3; ++l)
        for (int M = -l; M <= l; ++M)
            for (int Mp = -l; Mp <= l; ++Mp) fc(l, M, Mp) = complex<double>(val(l, M + 3, Mp + 3, 5) * (l + 1), val(l, M + 3, Mp + 3, 6));
    fc(2, -2, 1) = complex<double>(150.0, -0.25);
    std::cout << fc;
    std::cout << 1.0 / 3.0 << std::endl;   // stream state left behind
    return 0;
}
