// Per-bandwidth constant tables, computed on the device in FP64 once per bandwidth.
//
//   cos(beta_k), sin(beta_k/2), cos(beta_k/2)  beta_k = pi(2k+1)/(4B)     fn_dwt.hpp:155-159
//   w_B(j) = 2/B sin(pi(2j+1)/(4B)) sum_{k<B} sin((2j+1)(2k+1)pi/(4B))/(2k+1)   fn_dwt.hpp:62-83
//   normf(M,M') = sqrt((2M+1)/2) prod_{i<M-M'} sqrt((2M-i)/(i+1))              fn_dwt.hpp:117-121
//   twiddle[t] = exp(-2 pi i t/N)
// The sine arguments are reduced exactly in integers before sinpi/cospi, and the weight sum
// is compensated (Neumaier), so each entry is within a few ulp of the exact value.

#include "common.cuh"
#include "dwt.cuh"

namespace pfsoft_dev {

namespace {

__host__ __device__ inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

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

}  // namespace

size_t tables_bytes(int B)
{
    const size_t N = 2 * (size_t)B;
    return 4 * align256(N * sizeof(double)) + align256(num_classes(B) * sizeof(double)) +
           align256(N * sizeof(double2));
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
    const int threads = 128;
    int blocks = (int)((num_classes(B) + threads - 1) / threads);
    if (blocks < 1) blocks = 1;
    tables_kernel<<<blocks, threads, 0, stream>>>(B, t->cosb, t->sinh, t->cosh, t->w, t->normf, t->twiddle);
    return cudaGetLastError();
}

}  // namespace pfsoft_dev
