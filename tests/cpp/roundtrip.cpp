// C++ drop-in check: the shape of the reference's examples/example.cpp (random coefficients ->
// IDSOFT -> DSOFT -> every |d re|, |d im| <= 1e-11) written against pfsoft_b200/pfsoft.hpp.
// Coefficients come from a seeded mt19937_64 (the reference seeds from the clock,
// include/PFSOFTlib_headers/random.hpp:90-96) in the reference fill order l -> M -> M'.
// Usage: roundtrip <bandwidth> [seed]; prints "Correct result:  Yes" and exits 0 on success.
#include <pfsoft_b200/pfsoft.hpp>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>

using namespace pfsoft;

int main(int argc, char** argv)
{
    if (argc < 2) {
        std::printf("usage: roundtrip <Bandwidth> [seed]\n");
        return 1;
    }
    const int bandwidth = std::atoi(argv[1]);
    const unsigned long seed = argc > 2 ? std::strtoul(argv[2], nullptr, 10) : 1;

    grid3D<complex<double> > sample(2 * bandwidth);
    DSOFTFourierCoefficients coef(bandwidth);
    DSOFTFourierCoefficients rec_coef(bandwidth);

    std::mt19937_64 e(seed);
    std::uniform_real_distribution<double> d(-1.0, 1.0);
    for (int l = 0; l < bandwidth; ++l)
        for (int M = -l; M <= l; ++M)
            for (int Mp = -l; Mp <= l; ++Mp) {
                coef(l, M, Mp).re = d(e);
                coef(l, M, Mp).im = d(e);
            }

    FourierTransforms::IDSOFT(coef, sample);
    const grid3D<complex<double> > before(sample);
    FourierTransforms::DSOFT(sample, rec_coef);

    bool equal = true;
    double worst = 0.0;
    int cnt = 0;
    for (int m = 0; m < bandwidth; ++m)
        for (int n = -m; n <= m; ++n)
            for (int k = -m; k <= m; ++k) {
                const double dr = std::fabs(coef(m, n, k).re - rec_coef(m, n, k).re);
                const double di = std::fabs(coef(m, n, k).im - rec_coef(m, n, k).im);
                if (dr > 1e-11 || di > 1e-11) equal = false;
                worst = std::fmax(worst, std::fmax(dr, di));
                ++cnt;
            }
    // DSOFT must leave the caller's grid as it was
    for (size_t i = 0; i < sample.size(); ++i)
        if (sample.mem[i] != before.mem[i]) equal = false;

    std::printf("#coefficients:   %d\n", cnt);
    std::printf("Bandbreite:      %d\n", bandwidth);
    std::printf("max abs error:   %.3e\n", worst);
    std::printf("Correct result:  %s\n", equal ? "Yes" : "No");

    // argument checks: a mismatched container warns and leaves it untouched
    DSOFTFourierCoefficients wrong(bandwidth + 1);
    wrong(0, 0, 0) = complex<double>(7.0, 0.0);
    FourierTransforms::DSOFT(sample, wrong);
    if (wrong(0, 0, 0).re != 7.0) equal = false;
    return equal ? 0 : 2;
}
