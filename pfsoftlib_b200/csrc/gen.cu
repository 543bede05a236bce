// Seeded, counter-based coefficient generator on the device (pfsoft_cuda_random_coeffs).
//
// The reference fills coefficients on the host from a clock-seeded mt19937_64
// (include/PFSOFTlib_headers/random.hpp:80-117), which is not reproducible. This generator is
// reproducible and order free: value i of a packed coefficient vector is a pure function of
// (seed, i), built from SplitMix64 (Steele, Lea, Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014) on the counter, so any launch shape gives the same numbers.
//   kind 0  re, im i.i.d. uniform in [-1, 1)
//   kind 1  |f| = (1+l)^-power * |N(0,1)| (Box-Muller), phase uniform in [0, 2 pi)
//   kind 2  |f| = (1+l)^-power, phase uniform in [0, 2 pi)

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/pfsoft_b200.h"
#include "common.cuh"
#include "dwt.cuh"

namespace {

__device__ __forceinline__ uint64_t splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// uniform in [0, 1) with 53 random bits
__device__ __forceinline__ double unit(uint64_t x) { return (double)(x >> 11) * 0x1.0p-53; }

__device__ __forceinline__ int degree_of(long long i)
{
    // largest l with l(4l^2-1)/3 <= i
    int l = (int)cbrt(0.75 * (double)i);
    while (l > 0 && (long long)l * (4LL * l * l - 1) / 3 > i) --l;
    while ((long long)(l + 1) * (4LL * (l + 1) * (l + 1) - 1) / 3 <= i) ++l;
    return l;
}

__global__ void random_coeffs_kernel(double2* out, long long n, uint64_t seed, int kind, double power)
{
    const uint64_t base = splitmix64(seed);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const uint64_t r0 = splitmix64(base ^ (2 * (uint64_t)i));
        const uint64_t r1 = splitmix64(base ^ (2 * (uint64_t)i + 1));
        double2 v;
        if (kind == 0) {
            v = make_double2(2.0 * unit(r0) - 1.0, 2.0 * unit(r1) - 1.0);
        } else {
            const int l = degree_of(i);
            double mag = pow(1.0 + l, -power);
            if (kind == 1) {
                const uint64_t r2 = splitmix64(base ^ (0x8000000000000000ull | (uint64_t)i));
                const double u = 1.0 - unit(r2);   // (0, 1]
                mag *= fabs(sqrt(-2.0 * log(u)) * cospi(2.0 * unit(r0)));
            }
            double s, c;
            sincospi(2.0 * unit(r1), &s, &c);
            v = make_double2(mag * c, mag * s);
        }
        out[i] = v;
    }
}

}  // namespace

extern "C" int pfsoft_cuda_random_coeffs(double* d_coeffs, int B, unsigned long long seed, int kind, double power,
                                         void* stream)
{
    pfsoft_dev::set_last_error("");
    if (B < 1 || B > 512) {
        pfsoft_dev::set_last_error("bandwidth must be in [1, 512]");
        return PFSOFT_EINVAL;
    }
    if (!d_coeffs || kind < 0 || kind > 2) {
        pfsoft_dev::set_last_error("bad output pointer or kind");
        return PFSOFT_EINVAL;
    }
    const long long n = (long long)pfsoft_dev::coef_offset(B);
    int blocks = (int)((n + 255) / 256);
    if (blocks > 8192) blocks = 8192;
    random_coeffs_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(reinterpret_cast<double2*>(d_coeffs), n, seed,
                                                                                kind, power);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        pfsoft_dev::set_last_error(cudaGetErrorString(e));
        return PFSOFT_ECUDA;
    }
    return PFSOFT_OK;
}
