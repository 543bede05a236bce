// Per-bandwidth constant tables, computed on the device in FP64 once per bandwidth.
//
//   cos(beta_k), sin(beta_k/2), cos(beta_k/2)  beta_k = pi(2k+1)/(4B)     fn_dwt.hpp:155-159
//   w_B(j) = 2/B sin(pi(2j+1)/(4B)) sum_{k<B} sin((2j+1)(2k+1)pi/(4B))/(2k+1)   fn_dwt.hpp:62-83
//   normf(M,M') = sqrt((2M+1)/2) prod_{i<M-M'} sqrt((2M-i)/(i+1))              fn_dwt.hpp:117-121
//   twiddle[t] = exp(-2 pi i t/N)
//   rc_cf / rc_f1: the recurrence coefficients c1, f1 f2 and f1 of every class and degree
//       (fn_dwt.hpp:167-199), so that the DWT kernels load them instead of recomputing them
//   pw_sin[p][k], pw_cos[p][k] = sin(beta_k/2)^p, cos(beta_k/2)^p, p < 2B, as an exact binary
//       exponent and a mantissa in [0.5, 1) (exponentiation by squaring, renormalised each
//       product), so that Wigner seeds far below the FP64 range keep full relative precision
// The sine arguments are reduced exactly in integers before sinpi/cospi, and the weight sum
// is compensated (Neumaier), so each entry is within a few ulp of the exact value.

#include "common.cuh"
#include "dwt.cuh"
#include "dwt_common.cuh"

namespace pfsoft_dev {

namespace {

__host__ __device__ inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// x^p as {m, e}: x^p = m 2^e, m in [0.5, 1); x > 0
__device__ double2 ext_pow_tab(double x, int p)
{
    int xe;
    double xm = frexp(x, &xe);
    double rm = 1.0;
    int re = 0;
    while (p) {
        if (p & 1) {
            int t;
            rm = frexp(rm * xm, &t);
            re += xe + t;
        }
        p >>= 1;
        if (p) {
            int t;
            xm = frexp(xm * xm, &t);
            xe = 2 * xe + t;
        }
    }
    int t;
    rm = frexp(rm, &t);
    return make_double2(rm, (double)(re + t));
}

__global__ void powers_kernel(int B, const double* sinh, const double* cosh, double2* pw_sin, double2* pw_cos)
{
    const int N = 2 * B;
    const long long total = (long long)2 * B * N;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int p = (int)(i / N), k = (int)(i - (long long)p * N);
        pw_sin[i] = ext_pow_tab(sinh[k], p);
        pw_cos[i] = ext_pow_tab(cosh[k], p);
    }
}

__global__ void tables_kernel(int B, double* cosb, double* sinh, double* cosh, double* w, double* normf,
                              double2* tw)
{
    const int N = 2 * B;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nthr = gridDim.x * blockDim.x;
    for (int k = tid; k < N; k += nthr) {
        const double x = (double)(2 * k + 1) / (double)(4 * B);
        cosb[k] = cospi(x);
        double s, c;
        sincospi(0.5 * x, &s, &c);
        sinh[k] = s;
        cosh[k] = c;
        // twiddles of the length-N DFT
        double ts, tc;
        sincospi(2.0 * (double)k / (double)N, &ts, &tc);
        tw[k] = make_double2(tc, -ts);
        // weights are symmetric, w(N-1-k) = w(k) (fn_dwt.hpp:80-81): compute k < B, mirror
        if (k >= B) continue;
        // exact integer reduction of (2k+1)(2q+1) modulo 8B (period of sin(pi p/(4B)))
        double sum = 0.0, comp = 0.0;
        const long long a = 2 * k + 1;
        for (int q = 0; q < B; ++q) {
            const long long p = (a * (2 * q + 1)) % (8LL * B);
            const double term = sinpi((double)p / (double)(4 * B)) / (double)(2 * q + 1);
            const double t = sum + term;
            comp += (fabs(sum) >= fabs(term)) ? (sum - t) + term : (term - t) + sum;
            sum = t;
        }
        const double wk = 2.0 / B * sinpi(x) * (sum + comp);
        w[k] = wk;
        w[N - 1 - k] = wk;
    }
    const int ncls = num_classes(B);
    for (int i = tid; i < ncls; i += nthr) {
        int M, Mp;
        class_orders(i, M, Mp);
        double nf = sqrt((2.0 * M + 1.0) / 2.0);
        for (int q = 0; q < M - Mp; ++q) nf *= sqrt((2.0 * M - q) / (q + 1.0));
        normf[i] = nf;
    }
}

// One CTA per order class: c1, f1 f2, f1 of the steps l -> l+1, l = M .. B-1.
__global__ void rc_kernel(int B, double2* rc_cf, double* rc_f1)
{
    int M, Mp;
    class_orders(blockIdx.x, M, Mp);
    const long long base = rc_offset(B, M, Mp);
    for (int l = M + threadIdx.x; l < B; l += blockDim.x) {
        double c1, f1, f2;
        dwtk::rec_coef(l, M, Mp, c1, f1, f2);
        rc_cf[base + (l - M)] = make_double2(c1, f1 * f2);
        rc_f1[base + (l - M)] = f1;
    }
}

}  // namespace

size_t tables_bytes(int B)
{
    const size_t N = 2 * (size_t)B, R = (size_t)rc_entries(B);
    return 4 * align256(N * sizeof(double)) + align256(num_classes(B) * sizeof(double)) +
           align256(N * sizeof(double2)) + 2 * align256(2 * (size_t)B * N * sizeof(double2)) +
           align256(R * sizeof(double2)) + align256(R * sizeof(double));
}

cudaError_t tables_build(int B, void* mem, BandTables* t, cudaStream_t stream)
{
    const size_t N = 2 * (size_t)B;
    char* p = static_cast<char*>(mem);
    t->B = B;
    t->N = (int)N;
    t->block = mem;
    t->cosb = reinterpret_cast<double*>(p);
    p += align256(N * sizeof(double));
    t->sinh = reinterpret_cast<double*>(p);
    p += align256(N * sizeof(double));
    t->cosh = reinterpret_cast<double*>(p);
    p += align256(N * sizeof(double));
    t->w = reinterpret_cast<double*>(p);
    p += align256(N * sizeof(double));
    t->normf = reinterpret_cast<double*>(p);
    p += align256(num_classes(B) * sizeof(double));
    t->twiddle = reinterpret_cast<double2*>(p);
    p += align256(N * sizeof(double2));
    t->pw_sin = reinterpret_cast<double2*>(p);
    p += align256(2 * (size_t)B * N * sizeof(double2));
    t->pw_cos = reinterpret_cast<double2*>(p);
    p += align256(2 * (size_t)B * N * sizeof(double2));
    t->rc_cf = reinterpret_cast<double2*>(p);
    p += align256((size_t)rc_entries(B) * sizeof(double2));
    t->rc_f1 = reinterpret_cast<double*>(p);
    const int threads = 128;
    int blocks = (int)((num_classes(B) + threads - 1) / threads);
    if (blocks < 1) blocks = 1;
    tables_kernel<<<blocks, threads, 0, stream>>>(B, t->cosb, t->sinh, t->cosh, t->w, t->normf, t->twiddle);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const long long total = (long long)2 * B * N;
    int pblocks = (int)((total + 255) / 256);
    if (pblocks > 4096) pblocks = 4096;
    powers_kernel<<<pblocks, 256, 0, stream>>>(B, t->sinh, t->cosh, t->pw_sin, t->pw_cos);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    rc_kernel<<<num_classes(B), 128, 0, stream>>>(B, t->rc_cf, t->rc_f1);
    return cudaGetLastError();
}

}  // namespace pfsoft_dev
