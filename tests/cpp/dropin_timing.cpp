// Timing of the C++ drop-in path: the calls a reference user makes (FourierTransforms::IDSOFT then
// FourierTransforms::DSOFT of pfsoft_b200/pfsoft.hpp) on the header's own containers, whose
// storage is plain new[] memory (pageable), exactly as the reference's benchmark drivers hold it
// (benchmark/benchmark_dsoft_for.cpp, benchmark/benchmark_idsoft_for.cpp).
// Usage: dropin_timing <bandwidth> <steps> <warmup> [seed]
// Prints one JSON object: transforms per second over the timed steps (each step one IDSOFT and
// one DSOFT), the wall time per step, and the round trip's max abs error.
#include <pfsoft_b200/pfsoft.hpp>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>

using namespace pfsoft;

int main(int argc, char** argv)
{
    if (argc < 4) {
        std::printf("usage: dropin_timing <bandwidth> <steps> <warmup> [seed]\n");
        return 1;
    }
    const int bandwidth = std::atoi(argv[1]);
    const int steps = std::atoi(argv[2]);
    const int warmup = std::atoi(argv[3]);
    const unsigned long seed = argc > 4 ? std::strtoul(argv[4], nullptr, 10) : 1;
    if (bandwidth < 1 || steps < 1 || warmup < 0) return 1;

    grid3D<complex<double> > sample(2 * bandwidth);
    DSOFTFourierCoefficients coef(bandwidth);
    DSOFTFourierCoefficients rec_coef(bandwidth);
    std::mt19937_64 e(seed);
    std::uniform_real_distribution<double> d(-1.0, 1.0);
    for (int l = 0; l < bandwidth; ++l)
        for (int M = -l; M <= l; ++M)
            for (int Mp = -l; Mp <= l; ++Mp) coef(l, M, Mp) = complex<double>(d(e), d(e));

    for (int i = 0; i < warmup; ++i) {
        FourierTransforms::IDSOFT(coef, sample);
        FourierTransforms::DSOFT(sample, rec_coef);
    }
    const auto t0 = std::chrono::steady_clock::now();
    for (int i = 0; i < steps; ++i) {
        FourierTransforms::IDSOFT(coef, sample);
        FourierTransforms::DSOFT(sample, rec_coef);
    }
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

    double worst = 0.0;
    for (int l = 0; l < bandwidth; ++l)
        for (int M = -l; M <= l; ++M)
            for (int Mp = -l; Mp <= l; ++Mp) {
                worst = std::fmax(worst, std::fabs(coef(l, M, Mp).re - rec_coef(l, M, Mp).re));
                worst = std::fmax(worst, std::fabs(coef(l, M, Mp).im - rec_coef(l, M, Mp).im));
            }
    std::printf("{\"transforms_per_s\": %.6g, \"ms_per_step\": %.6g, \"steps\": %d, \"max_abs_err\": %.3e}\n",
                2.0 * steps / sec, 1e3 * sec / steps, steps, worst);
    return worst <= 1e-11 ? 0 : 2;
}
