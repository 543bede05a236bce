// Discrete Wigner transform (DWT) over beta for every order class, FP64 on CUDA cores (sm_100a).
//
// For the class (M, M'), M >= M' >= 0, one "team" of 1, 2 or 4 warps generates the reference's
// Wigner rows d_{M,M'}(l, beta_k), l = M..B-1, on chip with the three-term recurrence in l
// (include/PFSOFTlib_headers/fn_dwt.hpp:167-199) and applies them to the up to eight beta
// columns the reference serves from one matrix (src/fn_dsoft.cpp:137-283,
// src/fn_idsoft.cpp:127-283). Nothing is stored: lane `tl` of the team owns beta columns
// k = tl + t*team_threads (t < KT), keeps d(l-1, k) and d(l, k) in registers and advances them
// one degree per step.
//
//   forward  f^l_{m1,m2} = pi/(2B^2) sign(l) sum_k d(l, k) X[row][col][rev ? N-1-k : k]
//            (weighted rows). Per degree every lane forms 16 partial sums (8 columns x re/im)
//            over its KT betas; a 5-step butterfly transpose-reduce over the warp leaves each
//            sum in one lane pair, multi-warp teams add their warps through shared memory.
//   inverse  X[row][col][rev ? N-1-k : k] = sum_l d'(l, k) sign(l) (2B^2/pi) f^l_{m1,m2}
//            (unweighted rows). The coefficients are staged in shared memory in chunks of 32
//            degrees and broadcast; each lane accumulates its own betas, no reduction.
//
// Seeds. d(M, k) = -normf * sin(beta_k/2)^(M-M') * cos(beta_k/2)^(M+M') (* w_k) can fall far
// below the FP64 range (the reference's x87 long double hides this). Seeds are formed with a
// separate binary exponent; a column whose seed is below 2^-900 runs the recurrence scaled by
// 2^(600 s) and rescales when it grows past 2^300. While s > 0 its true magnitude is below
// 2^-300 and it contributes nothing at FP64 precision, so it is skipped.

#include "common.cuh"
#include "dwt.cuh"

namespace pfsoft_dev {

namespace {

constexpr int kWarps = 4;     // warps per CTA
constexpr int kLB = 32;       // degrees per reduction / coefficient chunk
constexpr double kPi = 3.141592653589793;

// x^p as (m, e) with x^p = m 2^e, m in [0.5, 1); x > 0
__device__ __forceinline__ void ext_pow(double x, int p, double& rm, int& re)
{
    int xe;
    double xm = frexp(x, &xe);
    rm = 1.0;
    re = 0;
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
}

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

// Seed of one beta column with its scale count (see the header comment).
__device__ __forceinline__ double seed_value(double nf_w, double sh, double ch, int sp, int cp, int& sc)
{
    double ms, mc;
    int es, ec, ev;
    ext_pow(sh, sp, ms, es);
    ext_pow(ch, cp, mc, ec);
    const double v = frexp(nf_w * ms * mc, &ev);
    const int E = ev + es + ec;
    if (E >= -900) {
        sc = 0;
        return -ldexp(v, E);
    }
    sc = (-900 - E + 599) / 600;
    return -ldexp(v, E + 600 * sc);
}

__device__ __forceinline__ void team_sync(int team, int team_warps)
{
    if (team_warps == 1) {
        __syncwarp();
    } else {
        asm volatile("bar.sync %0, %1;" ::"r"(1 + team), "r"(32 * team_warps) : "memory");
    }
}

// lane -> index of the fully reduced value it holds after warp_reduce16
__device__ __forceinline__ int reduced_index(int lane)
{
    return ((lane >> 4) & 1) * 8 + ((lane >> 3) & 1) * 4 + ((lane >> 2) & 1) * 2 + ((lane >> 1) & 1);
}

// Butterfly transpose-reduce of 16 values over the 32 lanes: 16 shuffles of a double.
__device__ __forceinline__ double warp_reduce16(double (&v)[16], int lane)
{
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const bool up = lane & 16;
        const double send = up ? v[i] : v[i + 8];
        const double keep = up ? v[i + 8] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const bool up = lane & 8;
        const double send = up ? v[i] : v[i + 4];
        const double keep = up ? v[i + 4] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const bool up = lane & 4;
        const double send = up ? v[i] : v[i + 2];
        const double keep = up ? v[i + 2] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
    }
    {
        const bool up = lane & 2;
        const double send = up ? v[0] : v[1];
        const double keep = up ? v[1] : v[0];
        v[0] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
    }
    v[0] += __shfl_xor_sync(0xffffffffu, v[0], 1);
    return v[0];
}

__device__ __forceinline__ double case_sign(const PairCase& p, int l, int M)
{
    return (p.rev && ((l - M) & 1)) ? -p.s0 : p.s0;
}

template <int KT>
__global__ void __launch_bounds__(kWarps * 32) dwt_forward_kernel(const double2* __restrict__ X,
                                                                  double* __restrict__ out, const DwtArgs a)
{
    __shared__ double s_rc[kWarps][kLB][3];
    __shared__ double s_red[kWarps][kLB][16];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int TW = a.team_warps;
    const int team = warp / TW;
    const int teams_per_cta = kWarps / TW;
    const int tthreads = 32 * TW;
    const int tl = (warp - team * TW) * 32 + lane;
    const int B = a.B, N = a.N;
    const int ncls = num_classes(B);
    const double norm = kPi / (double)(B * 2 * B);   // src/fn_dsoft.cpp:119

    int kcol[KT];
    double cb[KT];
#pragma unroll
    for (int t = 0; t < KT; ++t) {
        kcol[t] = tl + t * tthreads;
        cb[t] = kcol[t] < N ? a.cosb[kcol[t]] : 0.0;
    }

    for (int cls = blockIdx.x * teams_per_cta + team; cls < ncls; cls += gridDim.x * teams_per_cta) {
        int M, Mp;
        class_orders(cls, M, Mp);
        PairCase pc[8];
        const int nc = class_cases(M, Mp, N, pc);

        double2 s[8][KT];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const double2* col = X + ((size_t)pc[c < nc ? c : 0].row * N + pc[c < nc ? c : 0].col) * N;
            const bool rev = pc[c < nc ? c : 0].rev;
#pragma unroll
            for (int t = 0; t < KT; ++t) {
                const int k = kcol[t];
                s[c][t] = (c < nc && k < N) ? __ldg(col + (rev ? N - 1 - k : k)) : make_double2(0.0, 0.0);
            }
        }

        const double nf = a.normf[cls];
        double dcur[KT], dprev[KT];
        int sc[KT];
        bool any = false;
#pragma unroll
        for (int t = 0; t < KT; ++t) {
            const int k = kcol[t];
            dprev[t] = 0.0;
            sc[t] = 0;
            dcur[t] = k < N ? seed_value(nf * a.w[k], a.sinh[k], a.cosh[k], M - Mp, M + Mp, sc[t]) : 0.0;
            any |= sc[t] > 0;
        }
        bool scaled = __any_sync(0xffffffffu, any);

        const int myv = reduced_index(lane);
        const int myc = myv >> 1;
        for (int l = M; l < B; ++l) {
            const int li = l - M;
            const int slot = li & (kLB - 1);
            if (slot == 0) {
                __syncwarp();
                const int ll = l + lane;
                if (ll < B - 1) {
                    double c1, f1, f2;
                    rec_coef(ll, M, Mp, c1, f1, f2);
                    s_rc[warp][lane][0] = c1;
                    s_rc[warp][lane][1] = f1;
                    s_rc[warp][lane][2] = f2;
                }
                __syncwarp();
            }
            double acc[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) acc[i] = 0.0;
#pragma unroll
            for (int t = 0; t < KT; ++t) {
                const double d = (scaled && sc[t]) ? 0.0 : dcur[t];
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    acc[2 * c] = fma(d, s[c][t].x, acc[2 * c]);
                    acc[2 * c + 1] = fma(d, s[c][t].y, acc[2 * c + 1]);
                }
            }
            const double val = warp_reduce16(acc, lane);
            if (TW == 1) {
                if (!(lane & 1) && myc < nc) {
                    const PairCase& p = pc[myc];
                    out[2 * coef_index(l, p.m1, p.m2) + (myv & 1)] = norm * case_sign(p, l, M) * val;
                }
            } else {
                if (!(lane & 1)) s_red[warp][slot][myv] = val;
                if (slot == kLB - 1 || l == B - 1) {
                    team_sync(team, TW);
                    const int l0 = l - slot;
                    const int cnt = (slot + 1) * 16;
                    for (int e = tl; e < cnt; e += tthreads) {
                        const int lj = e >> 4, v = e & 15, c = v >> 1;
                        if (c < nc) {
                            double sum = 0.0;
                            for (int w = 0; w < TW; ++w) sum += s_red[team * TW + w][lj][v];
                            const PairCase& p = pc[c];
                            const int ld = l0 + lj;
                            out[2 * coef_index(ld, p.m1, p.m2) + (v & 1)] = norm * case_sign(p, ld, M) * sum;
                        }
                    }
                    team_sync(team, TW);
                }
            }
            if (l + 1 < B) {
                const double c1 = s_rc[warp][slot][0], f1 = s_rc[warp][slot][1], f2 = s_rc[warp][slot][2];
#pragma unroll
                for (int t = 0; t < KT; ++t) {
                    const double nx = fma(c1, dprev[t], (dcur[t] * f1) * (f2 + cb[t]));
                    dprev[t] = dcur[t];
                    dcur[t] = nx;
                }
                if (scaled) {
                    bool still = false;
#pragma unroll
                    for (int t = 0; t < KT; ++t) {
                        if (sc[t] && fabs(dcur[t]) >= 0x1p300) {
                            dcur[t] *= 0x1p-600;
                            dprev[t] *= 0x1p-600;
                            --sc[t];
                        }
                        still |= sc[t] > 0;
                    }
                    scaled = __any_sync(0xffffffffu, still);
                }
            }
        }
        __syncwarp();
    }
}

template <int KT>
__global__ void __launch_bounds__(kWarps * 32) dwt_inverse_kernel(const double2* __restrict__ coeffs,
                                                                  double2* __restrict__ X, const DwtArgs a)
{
    __shared__ double s_rc[kWarps][kLB][3];
    __shared__ double2 s_g[kWarps][8][kLB];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int TW = a.team_warps;
    const int team = warp / TW;
    const int teams_per_cta = kWarps / TW;
    const int tthreads = 32 * TW;
    const int tl = (warp - team * TW) * 32 + lane;
    const int B = a.B, N = a.N;
    const int ncls = num_classes(B);
    const double norm = (double)(B * 2 * B) / kPi;   // src/fn_idsoft.cpp:109

    int kcol[KT];
    double cb[KT];
#pragma unroll
    for (int t = 0; t < KT; ++t) {
        kcol[t] = tl + t * tthreads;
        cb[t] = kcol[t] < N ? a.cosb[kcol[t]] : 0.0;
    }

    for (int cls = blockIdx.x * teams_per_cta + team; cls < ncls; cls += gridDim.x * teams_per_cta) {
        int M, Mp;
        class_orders(cls, M, Mp);
        PairCase pc[8];
        const int nc = class_cases(M, Mp, N, pc);

        const double nf = a.normf[cls];
        double dcur[KT], dprev[KT];
        int sc[KT];
        bool any = false;
#pragma unroll
        for (int t = 0; t < KT; ++t) {
            const int k = kcol[t];
            dprev[t] = 0.0;
            sc[t] = 0;
            dcur[t] = k < N ? seed_value(nf, a.sinh[k], a.cosh[k], M - Mp, M + Mp, sc[t]) : 0.0;
            any |= sc[t] > 0;
        }
        bool scaled = __any_sync(0xffffffffu, any);

        double2 acc[8][KT];
#pragma unroll
        for (int c = 0; c < 8; ++c)
#pragma unroll
            for (int t = 0; t < KT; ++t) acc[c][t] = make_double2(0.0, 0.0);

        for (int l = M; l < B; ++l) {
            const int slot = (l - M) & (kLB - 1);
            if (slot == 0) {
                team_sync(team, TW);   // the previous chunk is consumed by every warp of the team
                for (int e = tl; e < 8 * kLB; e += tthreads) {
                    const int c = e / kLB, j = e - c * kLB, ld = l + j;
                    double2 g = make_double2(0.0, 0.0);
                    if (c < nc && ld < B) {
                        const PairCase& p = pc[c];
                        const double f = norm * case_sign(p, ld, M);
                        const double2 x = __ldg(coeffs + coef_index(ld, p.m1, p.m2));
                        g = make_double2(f * x.x, f * x.y);
                    }
                    s_g[team][c][j] = g;
                }
                const int ll = l + lane;
                if (ll < B - 1) {
                    double c1, f1, f2;
                    rec_coef(ll, M, Mp, c1, f1, f2);
                    s_rc[warp][lane][0] = c1;
                    s_rc[warp][lane][1] = f1;
                    s_rc[warp][lane][2] = f2;
                }
                team_sync(team, TW);
            }
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const double2 g = s_g[team][c][slot];
#pragma unroll
                for (int t = 0; t < KT; ++t) {
                    const double d = (scaled && sc[t]) ? 0.0 : dcur[t];
                    acc[c][t].x = fma(d, g.x, acc[c][t].x);
                    acc[c][t].y = fma(d, g.y, acc[c][t].y);
                }
            }
            if (l + 1 < B) {
                const double c1 = s_rc[warp][slot][0], f1 = s_rc[warp][slot][1], f2 = s_rc[warp][slot][2];
#pragma unroll
                for (int t = 0; t < KT; ++t) {
                    const double nx = fma(c1, dprev[t], (dcur[t] * f1) * (f2 + cb[t]));
                    dprev[t] = dcur[t];
                    dcur[t] = nx;
                }
                if (scaled) {
                    bool still = false;
#pragma unroll
                    for (int t = 0; t < KT; ++t) {
                        if (sc[t] && fabs(dcur[t]) >= 0x1p300) {
                            dcur[t] *= 0x1p-600;
                            dprev[t] *= 0x1p-600;
                            --sc[t];
                        }
                        still |= sc[t] > 0;
                    }
                    scaled = __any_sync(0xffffffffu, still);
                }
            }
        }
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            if (c < nc) {
                double2* col = X + ((size_t)pc[c].row * N + pc[c].col) * N;
#pragma unroll
                for (int t = 0; t < KT; ++t) {
                    const int k = kcol[t];
                    if (k < N) col[pc[c].rev ? N - 1 - k : k] = acc[c][t];
                }
            }
        }
        team_sync(team, TW);   // s_g / s_rc reuse by the next class
    }
}

__global__ void zero_nyquist_kernel(double2* X, int B)
{
    const int N = 2 * B;
    const long long total = (long long)(2 * N - 1) * N;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const long long v = i / N;
        const int k = (int)(i - v * N);
        int row, col;
        if (v < N) {
            row = B;
            col = (int)v;
        } else {
            col = B;
            row = (int)(v - N);
            if (row >= B) ++row;   // skip (B, B), covered above
        }
        X[((size_t)row * N + col) * N + k] = make_double2(0.0, 0.0);
    }
}

template <int KT>
cudaError_t launch_fwd(const double2* X, double2* coeffs, const DwtArgs& a, int nblocks, cudaStream_t s)
{
    dwt_forward_kernel<KT><<<nblocks, kWarps * 32, 0, s>>>(X, reinterpret_cast<double*>(coeffs), a);
    return cudaGetLastError();
}

template <int KT>
cudaError_t launch_inv(const double2* coeffs, double2* X, const DwtArgs& a, int nblocks, cudaStream_t s)
{
    dwt_inverse_kernel<KT><<<nblocks, kWarps * 32, 0, s>>>(coeffs, X, a);
    return cudaGetLastError();
}

int cols_per_lane(const DwtArgs& a) { return (a.N + 32 * a.team_warps - 1) / (32 * a.team_warps); }

}  // namespace

int dwt_team_warps(int N)
{
    if (N <= 128) return 1;
    if (N <= 256) return 2;
    return 4;
}

cudaError_t dwt_forward_launch(const double2* X, double2* coeffs, const DwtArgs& a, int nblocks, cudaStream_t s)
{
    const int kt = cols_per_lane(a);
    if (kt <= 1) return launch_fwd<1>(X, coeffs, a, nblocks, s);
    if (kt <= 2) return launch_fwd<2>(X, coeffs, a, nblocks, s);
    if (kt <= 4) return launch_fwd<4>(X, coeffs, a, nblocks, s);
    if (kt <= 8) return launch_fwd<8>(X, coeffs, a, nblocks, s);
    return cudaErrorInvalidValue;
}

cudaError_t dwt_inverse_launch(const double2* coeffs, double2* X, const DwtArgs& a, int nblocks, cudaStream_t s)
{
    const int kt = cols_per_lane(a);
    if (kt <= 1) return launch_inv<1>(coeffs, X, a, nblocks, s);
    if (kt <= 2) return launch_inv<2>(coeffs, X, a, nblocks, s);
    if (kt <= 4) return launch_inv<4>(coeffs, X, a, nblocks, s);
    if (kt <= 8) return launch_inv<8>(coeffs, X, a, nblocks, s);
    return cudaErrorInvalidValue;
}

cudaError_t zero_nyquist_launch(double2* X, int B, cudaStream_t s)
{
    const int N = 2 * B;
    const long long total = (long long)(2 * N - 1) * N;
    int blocks = (int)((total + 255) / 256);
    if (blocks > 4096) blocks = 4096;
    zero_nyquist_kernel<<<blocks, 256, 0, s>>>(X, B);
    return cudaGetLastError();
}

}  // namespace pfsoft_dev
