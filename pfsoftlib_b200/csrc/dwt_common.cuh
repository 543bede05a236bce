// Device helpers shared by the discrete Wigner transform kernels (dwt.cu, dwt_batch.cu):
// recurrence coefficients, table seeds, the per-column recurrence state, the FP64 MMA, class
// scheduling order and team barriers.
#pragma once

#include "common.cuh"
#include "dwt.cuh"

namespace pfsoft_dev {
namespace dwtk {

constexpr int kWarps = 4;     // warps per CTA
constexpr int kLB = 32;       // degrees per reduction / coefficient chunk
constexpr double kPi = 3.141592653589793;

// Recurrence step degree l -> l+1 for orders (M, Mp) (fn_dwt.hpp:167-192):
//   d(l+1) = c1 d(l-1) + d(l) f1 (f2 + cos beta)
__device__ __forceinline__ void rec_coef(int l, int M, int Mp, double& c1, double& f1, double& f2)
{
    const double idx = (double)l;
    const double nrm = sqrt((2.0 * idx + 3.0) / (2.0 * idx + 1.0));
    const double nom = (idx + 1.0) * (2.0 * idx + 1.0);
    const double a1 = (idx + 1.0) * (idx + 1.0) - (double)M * M;   // exact integers
    const double a2 = (idx + 1.0) * (idx + 1.0) - (double)Mp * Mp;
    const double den = 1.0 / sqrt(a1 * a2);
    f1 = nrm * nom * den;
    c1 = 0.0;
    f2 = 0.0;
    if (l != 0) {
        const double t1 = sqrt((2.0 * idx + 3.0) / (2.0 * idx - 1.0)) * (idx + 1.0) / idx;
        const double t2 = sqrt((idx * idx - (double)M * M) * (idx * idx - (double)Mp * Mp));
        c1 = -t1 * t2 * den;
        f2 = -(double)M * Mp / (idx * (idx + 1.0));
    }
}

// Seed of one beta column with its scale count (see the header comment): nf_w * s * c where s
// and c are table powers {mantissa, exponent}.
__device__ __forceinline__ double seed_value(double nf_w, double2 s, double2 c, int& sc)
{
    int ev;
    const double v = frexp(nf_w * s.x * c.x, &ev);
    const int E = ev + (int)s.y + (int)c.y;
    if (E >= -900) {
        sc = 0;
        return -ldexp(v, E);
    }
    sc = (-900 - E + 599) / 600;
    return -ldexp(v, E + 600 * sc);
}

template <int TW>
__device__ __forceinline__ void team_sync(int team)
{
    if (TW == 1) {
        __syncwarp();
    } else {
        asm volatile("bar.sync %0, %1;" ::"r"(1 + team), "r"(32 * TW) : "memory");
    }
}

__device__ __forceinline__ double case_sign(const PairCase& p, int l, int M)
{
    return (p.rev && ((l - M) & 1)) ? -p.s0 : p.s0;
}

// One FP64 MMA: C(8x8) += A(8x4, row) * B(4x8, col). Fragments per lane (g = lane/4, t = lane%4):
// A[g][t], B[t][g], C[g][2t], C[g][2t+1].
__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b)
{
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
        : "+d"(c0), "+d"(c1)
        : "d"(a), "d"(b));
}

// Hint: bring [p, p + bytes) into L2 (bytes a multiple of 16, p 16-byte aligned).
__device__ __forceinline__ void prefetch_l2(const void* p, unsigned bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// Snake (boustrophedon) order over the longest-first class list: team `my` of `T` takes
// classes r*T + my in even rounds and r*T + T-1-my in odd rounds.
__device__ __forceinline__ int snake_class(int r, int T, int my) { return r * T + ((r & 1) ? (T - 1 - my) : my); }

// Length of the launch's class list and its i-th class (all classes in order when no subset is
// given; a subset keeps the longest-first order the snake relies on).
__device__ __forceinline__ int list_length(const DwtArgs& a) { return a.classes ? a.n_classes : num_classes(a.B); }
__device__ __forceinline__ int list_class(const DwtArgs& a, int i) { return a.classes ? __ldg(a.classes + i) : i; }

template <int KT>
struct ColumnState {
    double cb[KT], dcur[KT], dprev[KT], keep[KT];
    int sc[KT];
    bool scaled;

    __device__ __forceinline__ void seed(const DwtArgs& a, const int* kc, double nf, bool weighted, int M, int Mp)
    {
        bool any = false;
#pragma unroll
        for (int j = 0; j < KT; ++j) {
            const int k = kc[j];
            dprev[j] = 0.0;
            sc[j] = 0;
            dcur[j] = k < a.N ? seed_value(weighted ? nf * a.w[k] : nf, a.pw_sin[(size_t)(M - Mp) * a.N + k],
                                           a.pw_cos[(size_t)(M + Mp) * a.N + k], sc[j])
                              : 0.0;
            keep[j] = sc[j] ? 0.0 : 1.0;
            any |= sc[j] > 0;
        }
        scaled = __any_sync(0xffffffffu, any);
    }

    // d(l) of the lane's columns into row[lane + 32j]; a column still below 2^-300 stores 0
    __device__ __forceinline__ void store(double* row, int lane) const
    {
        if (!scaled) {
#pragma unroll
            for (int j = 0; j < KT; ++j) row[lane + 32 * j] = dcur[j];
        } else {
#pragma unroll
            for (int j = 0; j < KT; ++j) row[lane + 32 * j] = dcur[j] * keep[j];
        }
    }

    // d(l+1) = c1 d(l-1) + d(l) (a + b cos beta), with a = f1 f2 and b = f1
    __device__ __forceinline__ void advance(double c1, double a, double b)
    {
#pragma unroll
        for (int j = 0; j < KT; ++j) {
            const double t = fma(b, cb[j], a);
            const double nx = fma(c1, dprev[j], dcur[j] * t);
            dprev[j] = dcur[j];
            dcur[j] = nx;
        }
        if (scaled) {
            bool still = false;
#pragma unroll
            for (int j = 0; j < KT; ++j) {
                if (sc[j] && fabs(dcur[j]) >= 0x1p300) {
                    dcur[j] *= 0x1p-600;
                    dprev[j] *= 0x1p-600;
                    if (--sc[j] == 0) keep[j] = 1.0;
                }
                still |= sc[j] > 0;
            }
            scaled = __any_sync(0xffffffffu, still);
        }
    }
};

// Recurrence coefficients for degrees l .. l+31 of one warp: rc[i] = {c1, f1 f2, f1, -} for the
// step l+i -> l+i+1 (one lane per degree), read from the bandwidth's table. Steps past the last
// degree get zeros (the rows they feed are zero and never used), so the step loop has no guards.
__device__ __forceinline__ void fill_rc4(const DwtArgs& a, double* rc, int l, int M, int Mp, int lane)
{
    __syncwarp();
    const int d = l + lane;
    double2 cf = make_double2(0.0, 0.0);
    double f1 = 0.0;
    if (d < a.B) {
        const long long i = rc_offset(a.B, M, Mp) + (d - M);
        cf = __ldg(a.rc_cf + i);
        f1 = __ldg(a.rc_f1 + i);
    }
    *reinterpret_cast<double2*>(rc + 4 * lane) = cf;
    rc[4 * lane + 2] = f1;
    __syncwarp();
}

// One recurrence step: store d(l) into `row`, advance to d(l+1).
template <int KT>
__device__ __forceinline__ void gen_step(ColumnState<KT>& cs, double* row, int lane, const double* rc)
{
    cs.store(row, lane);
    const double2 ca = *reinterpret_cast<const double2*>(rc);
    cs.advance(ca.x, ca.y, rc[2]);
}

}  // namespace dwtk
}  // namespace pfsoft_dev
