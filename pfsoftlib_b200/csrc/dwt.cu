// Discrete Wigner transform (DWT) over beta for every order class, FP64 (sm_100a).
//
// For the class (M, M'), M >= M' >= 0, one "team" of TW warps generates the reference's Wigner
// rows d_{M,M'}(l, beta_k), l = M..B-1, on chip with the three-term recurrence in l
// (include/PFSOFTlib_headers/fn_dwt.hpp:167-199) and applies them to the up to eight beta
// columns the reference serves from one matrix (src/fn_dsoft.cpp:137-283,
// src/fn_idsoft.cpp:127-283). The matrix is never stored: warp w of the team owns beta columns
// [w*KW, w*KW + KW), KW = 32*KT, and lane i runs the recurrence for columns w*KW + i + 32j,
// keeping d(l-1, k) and d(l, k) in registers. A few degrees at a time the fresh rows go to
// shared memory and the contraction over beta runs on the FP64 MMA (mma.sync m8n8k4 f64):
//
//   forward  F[l][v] = sum_k D[l][k] S[k][v], S[k][v] = component (v&1) of
//            X[row][col][rev ? N-1-k : k] for case v/2 (weighted rows, 8 degrees per MMA tile);
//            the TW warps' partial sums over their beta ranges are added in shared memory and
//            written as f^l = pi/(2B^2) sign(l) F[l].
//   inverse  S[k][v] = sum_l D[l][k] G[l][v], G = (2B^2/pi) sign(l) f^l staged in shared memory
//            in chunks of 32 degrees (prefetched one chunk ahead); 4 degrees per MMA; each warp
//            owns its columns, so nothing is reduced across warps.
//
// Seeds. d(M, k) = -normf * sin(beta_k/2)^(M-M') * cos(beta_k/2)^(M+M') (* w_k) can fall far
// below the FP64 range (the reference's x87 long double hides this). Seeds are formed with a
// separate binary exponent; a column whose seed is below 2^-900 runs the recurrence scaled by
// 2^(600 s) and rescales when it grows past 2^300. While s > 0 its true magnitude is below
// 2^-300 and it contributes nothing at FP64 precision, so it is skipped.
//
// Scheduling: a persistent grid; classes (longest first) are dealt to teams in snake order.

#include "common.cuh"
#include "dwt.cuh"
#include "dwt_common.cuh"

namespace pfsoft_dev {

namespace {

using namespace dwtk;

template <int KT>
struct FwdSmem {
    static constexpr int KW = 32 * KT;
    static constexpr int DS = KW + 4;   // padded row stride: A-fragment loads hit distinct banks
    static constexpr size_t d_off = 0;                                       // [kWarps][2][8][DS]
    static constexpr size_t rc_off = d_off + (size_t)kWarps * 2 * 8 * DS;     // [kWarps][kLB][4]
    static constexpr size_t red_off = rc_off + (size_t)kWarps * kLB * 4;     // [2][kWarps][8][16]
    static constexpr size_t doubles = red_off + (size_t)2 * kWarps * 8 * 16;
};

template <int KT, int TEAMS>
struct InvSmem {
    static constexpr int KW = 32 * KT;
    static constexpr int DS = KW + 8;   // padded row stride for the transposed A-fragment loads
    // coefficient row stride: with one team per CTA 16 values + 4, so that the B-fragment loads of
    // the four t4 rows hit distinct banks; with four teams 16, which keeps two CTAs per SM
    static constexpr int GS = TEAMS == 1 ? 20 : 16;
    static constexpr size_t d_off = 0;                                       // [kWarps][2][8][DS]
    static constexpr size_t rc_off = d_off + (size_t)kWarps * 2 * 8 * DS;     // [kWarps][kLB][4]
    static constexpr size_t g_off = rc_off + (size_t)kWarps * kLB * 4;       // [TEAMS][2][kLB][GS]
    static constexpr size_t doubles = g_off + (size_t)TEAMS * 2 * kLB * GS;
};

// CTAs per SM the register budget is cut for (measured on B200 at B = 128: the 2-column, 4-warp
// teams gain 12-16 % over 255-register, 2-CTA kernels at 3-4 CTAs per SM; the inverse spills
// past 3).
constexpr int fwd_min_blocks(int KT, int TW, int CS) { return KT == 2 && TW == 4 ? 4 : (CS == 2 ? 4 : 1); }
constexpr int inv_min_blocks(int KT, int TW, int CS) { return KT == 2 && TW == 4 ? 3 : (CS == 2 ? 3 : 1); }

// Team layout shared by both directions: TW column warps x CS case warps. Warp `wt` of the team
// owns beta columns [cw*KW, cw*KW + KW) (cw = wt / CS) and, with CS = 2, only the four cases
// 4h .. 4h+3 (h = wt % CS, one MMA n-tile); the pair of case warps runs the same recurrence
// (FP64 pipe) so that each holds half of the MMA operands (tensor pipe) in registers.
template <int KT, int TW, int CS>
struct Team {
    static constexpr int WARPS = TW * CS;
    static constexpr int PER_CTA = kWarps / WARPS;
    static constexpr int NT = 2 / CS;   // MMA n-tiles (groups of 4 cases) per warp
    int warp, lane, g, t4, team, wt, cw, h, tl;
    __device__ __forceinline__ Team()
    {
        warp = threadIdx.x >> 5;
        lane = threadIdx.x & 31;
        g = lane >> 2;
        t4 = lane & 3;
        team = warp / WARPS;
        wt = warp - team * WARPS;
        cw = wt / CS;
        h = wt - cw * CS;
        tl = wt * 32 + lane;
    }
};

// Forward DWT (see the header comment). The rows of 8-degree block b+1 are generated while
// block b is contracted (two row buffers).
template <int KT, int TW, int CS>
__global__ void __launch_bounds__(kWarps * 32, fwd_min_blocks(KT, TW, CS))
    dwt_forward_kernel(const double2* __restrict__ X, double* __restrict__ out, const DwtArgs a)
{
    using L = FwdSmem<KT>;
    using TM = Team<KT, TW, CS>;
    constexpr int KW = L::KW, DS = L::DS, NSUB = KW / 4, QPS = NSUB / 8;   // subtiles per step
    constexpr int NT = TM::NT;
    extern __shared__ double smem[];
    const TM tm;
    const int lane = tm.lane, g = tm.g, t4 = tm.t4;
    double* s_d = smem + L::d_off + (size_t)tm.warp * 2 * 8 * DS;
    double* s_rc = smem + L::rc_off + (size_t)tm.warp * kLB * 4;
    double* s_red = smem + L::red_off;   // [2][warp][8][16]
    const int B = a.B, N = a.N;
    const int ncls = list_length(a);
    const double norm = kPi / (double)(B * 2 * B);   // src/fn_dsoft.cpp:119

    int kc[KT];
    ColumnState<KT> cs;
#pragma unroll
    for (int j = 0; j < KT; ++j) {
        kc[j] = tm.cw * KW + lane + 32 * j;
        cs.cb[j] = kc[j] < N ? a.cosb[kc[j]] : 0.0;
    }

    const int T = gridDim.x * TM::PER_CTA;
    const int my = blockIdx.x * TM::PER_CTA + tm.team;
    int redbuf = 0;
    for (int r = 0;; ++r) {
        const int ci = snake_class(r, T, my);
        if (ci >= ncls) break;
        const int cls = list_class(a, ci);
        int M, Mp;
        class_orders(cls, M, Mp);
        const int nc = class_case_count(M, Mp);

        // B fragments: S[k][v] for k = cw*KW + 4q + t4 and v = 2*case + (re, im), case = 4n + g/2
        // for this warp's n-tiles n
        double sb[NT][NSUB];
        PairCase po[NT];   // output cases 4n + t4 held by this lane
#pragma unroll
        for (int n = 0; n < NT; ++n) {
            const int nn = CS == 2 ? tm.h : n;
            const int c = 4 * nn + (g >> 1), comp = g & 1;
            const bool ok = c < nc;
            const PairCase p = class_case(M, Mp, ok ? c : 0, N);
            const double* col = reinterpret_cast<const double*>(X + ((size_t)p.row * N + p.col) * N) + comp;
#pragma unroll
            for (int q = 0; q < NSUB; ++q) {
                const int k = tm.cw * KW + 4 * q + t4;
                sb[n][q] = (ok && k < N) ? __ldg(col + 2 * (p.rev ? N - 1 - k : k)) : 0.0;
            }
            po[n] = class_case(M, Mp, 4 * nn + t4 < nc ? 4 * nn + t4 : 0, N);
        }
        // the case this thread sums in the cross-warp reduction (tl & 7), fixed for the class
        const PairCase pred = class_case(M, Mp, (tm.tl & 7) < nc ? (tm.tl & 7) : 0, N);

        {
            // the next class's beta columns (this warp's slice) into L2 while this one runs
            const int nx = snake_class(r + 1, T, my);
            if (nx < ncls && lane < 8) {
                int M2, Mp2;
                class_orders(list_class(a, nx), M2, Mp2);
                if (lane < class_case_count(M2, Mp2)) {
                    const PairCase p = class_case(M2, Mp2, lane, N);
                    const int k0 = tm.cw * KW, k1 = min(N, k0 + KW);
                    if (k0 < k1) {
                        const int lo = p.rev ? N - k1 : k0;
                        prefetch_l2(X + ((size_t)p.row * N + p.col) * N + lo, (unsigned)(k1 - k0) * sizeof(double2));
                    }
                }
            }
        }
        cs.seed(a, kc, a.normf[cls], true, M, Mp);
        fill_rc4(a, s_rc, M, M, Mp, lane);
#pragma unroll
        for (int s = 0; s < 8; ++s) gen_step<KT>(cs, s_d + s * DS, lane, s_rc + 4 * s);   // block 0
        __syncwarp();
        const int nblk = (B - M + 7) >> 3;
        int cur = 0;
        for (int blk = 0; blk < nblk; ++blk) {
            const int l0 = M + 8 * blk;
            const double* dc = s_d + cur * 8 * DS;
            double* dn = s_d + (cur ^ 1) * 8 * DS;
            double acc[2][NT][2];
#pragma unroll
            for (int e = 0; e < 2; ++e)
#pragma unroll
                for (int n = 0; n < NT; ++n) acc[e][n][0] = acc[e][n][1] = 0.0;
            auto mma_step = [&](int s) {
#pragma unroll
                for (int i = 0; i < QPS; ++i) {
                    const int q = s * QPS + i;
                    const double av = dc[g * DS + 4 * q + t4];
#pragma unroll
                    for (int n = 0; n < NT; ++n) dmma(acc[q & 1][n][0], acc[q & 1][n][1], av, sb[n][q]);
                }
            };
            if (blk + 1 < nblk) {
                // contract block blk while generating block blk+1 (degrees beyond B - 1 are
                // generated too; their rows only reach outputs that are never stored)
                const int off = 8 * (blk + 1);
                if ((off & (kLB - 1)) == 0) fill_rc4(a, s_rc, M + off, M, Mp, lane);
                const double* rcb = s_rc + 4 * (off & (kLB - 1));
#pragma unroll
                for (int s = 0; s < 8; ++s) {
                    mma_step(s);
                    gen_step<KT>(cs, dn + s * DS, lane, rcb + 4 * s);
                }
            } else {
#pragma unroll
                for (int s = 0; s < 8; ++s) mma_step(s);
            }
            // lane holds the partial F[l0+g][case 4n + t4] = (r[n][0], r[n][1])
            double rr[NT][2];
#pragma unroll
            for (int n = 0; n < NT; ++n) {
                rr[n][0] = acc[0][n][0] + acc[1][n][0];
                rr[n][1] = acc[0][n][1] + acc[1][n][1];
            }
            if (TW == 1) {
                const int l = l0 + g;
#pragma unroll
                for (int n = 0; n < NT; ++n) {
                    const int c = 4 * (CS == 2 ? tm.h : n) + t4;
                    if (l < B && c < nc) {
                        const double f = norm * case_sign(po[n], l, M);
                        *reinterpret_cast<double2*>(out + 2 * coef_index(l, po[n].m1, po[n].m2)) =
                            make_double2(f * rr[n][0], f * rr[n][1]);
                    }
                }
            } else {
                // partial sums of the column warps meet in a double-buffered slot: the buffer
                // written here was last read before the previous team barrier
                double* red = s_red + ((size_t)redbuf * kWarps + tm.warp) * 128 + g * 16;
#pragma unroll
                for (int n = 0; n < NT; ++n)
                    *reinterpret_cast<double2*>(red + 8 * (CS == 2 ? 0 : n) + 2 * t4) = make_double2(rr[n][0], rr[n][1]);
                team_sync<TM::WARPS>(tm.team);
                for (int e = tm.tl; e < 64; e += 32 * TM::WARPS) {
                    const int gg = e >> 3, c = e & 7;
                    const int l = l0 + gg;
                    if (c < nc && l < B) {
                        // case c lives in n-tile c/4: slot (c%4) of warp (cw, h = c/4) when CS = 2
                        double2 sum = make_double2(0.0, 0.0);
#pragma unroll
                        for (int w = 0; w < TW; ++w) {
                            const int wsrc = tm.team * TM::WARPS + w * CS + (CS == 2 ? (c >> 2) : 0);
                            const int slot = CS == 2 ? 2 * (c & 3) : 2 * c;
                            const double2 v = *reinterpret_cast<const double2*>(
                                s_red + ((size_t)redbuf * kWarps + wsrc) * 128 + gg * 16 + slot);
                            sum.x += v.x;
                            sum.y += v.y;
                        }
                        const double f = norm * case_sign(pred, l, M);   // c == tl & 7
                        *reinterpret_cast<double2*>(out + 2 * coef_index(l, pred.m1, pred.m2)) = make_double2(f * sum.x, f * sum.y);
                    }
                }
                redbuf ^= 1;
            }
            __syncwarp();
            cur ^= 1;
        }
    }
}

// The Nyquist bins of X (row B with every column, column B with every other row; every beta),
// which no order class writes: set to zero, element i = first, first + stride, ...
__device__ __forceinline__ void nyquist_zero(double2* X, int B, long long first, long long stride)
{
    const int N = 2 * B;
    const long long total = (long long)(2 * N - 1) * N;
    for (long long i = first; i < total; i += stride) {
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

// Inverse DWT (see the header comment). Each lane ends with case 4n + t4 of its n-tiles at
// columns cw*KW + 8p + g. The rows of 8-degree block b+1 are generated while block b is
// applied (two MMA k-steps of 4 degrees). Coefficients move through registers one 32-degree
// chunk ahead of their use; the first chunk of the next class is fetched during this one.
template <int KT, int TW, int CS>
__global__ void __launch_bounds__(kWarps * 32, inv_min_blocks(KT, TW, CS))
    dwt_inverse_kernel(const double2* __restrict__ coeffs, double2* __restrict__ X, const DwtArgs a)
{
    using L = InvSmem<KT, kWarps / (TW * CS)>;
    using TM = Team<KT, TW, CS>;
    constexpr int KW = L::KW, DS = L::DS, NSUB8 = KW / 8;
    constexpr int NT = TM::NT;
    constexpr int TT = 32 * TM::WARPS;           // team threads
    constexpr int PER = (8 * kLB + TT - 1) / TT; // coefficients fetched per thread per chunk
    extern __shared__ double smem[];
    const TM tm;
    const int lane = tm.lane, g = tm.g, t4 = tm.t4;
    double* s_d = smem + L::d_off + (size_t)tm.warp * 2 * 8 * DS;
    double* s_rc = smem + L::rc_off + (size_t)tm.warp * kLB * 4;
    constexpr int GS = L::GS;
    // one team per CTA: consecutive lanes stage the cases of one degree (one contiguous row, no
    // bank conflicts); four one-warp teams measured faster with consecutive degrees per lane
    constexpr bool kCaseFirst = kWarps / (TW * CS) == 1;
    double* s_g = smem + L::g_off + (size_t)tm.team * 2 * kLB * GS;   // [2][kLB][GS]
    const int B = a.B, N = a.N;
    const int ncls = list_length(a);
    const double norm = (double)(B * 2 * B) / kPi;   // src/fn_idsoft.cpp:109

    int kc[KT];
    ColumnState<KT> cs;
#pragma unroll
    for (int j = 0; j < KT; ++j) {
        kc[j] = tm.cw * KW + lane + 32 * j;
        cs.cb[j] = kc[j] < N ? a.cosb[kc[j]] : 0.0;
    }

    // coefficients of class (M, Mp) for degrees l .. l+31, scaled and signed, into registers
    double2 pf[PER];
    auto fetch = [&](int M, int Mp, int l) {
        const int nc = class_case_count(M, Mp);
#pragma unroll
        for (int i = 0; i < PER; ++i) {
            const int e = tm.tl + i * TT;
            const int c = kCaseFirst ? (e & 7) : e / kLB, ld = l + (kCaseFirst ? (e >> 3) : e % kLB);
            double2 v = make_double2(0.0, 0.0);
            if (e < 8 * kLB && c < nc && ld < B) {
                const PairCase p = class_case(M, Mp, c, N);
                const double f = norm * case_sign(p, ld, M);
                const double2 x = __ldg(coeffs + coef_index(ld, p.m1, p.m2));
                v = make_double2(f * x.x, f * x.y);
            }
            pf[i] = v;
        }
    };
    auto stash = [&](int buf) {
#pragma unroll
        for (int i = 0; i < PER; ++i) {
            const int e = tm.tl + i * TT;
            const int c = kCaseFirst ? (e & 7) : e / kLB, j = kCaseFirst ? (e >> 3) : e % kLB;
            if (e < 8 * kLB) *reinterpret_cast<double2*>(s_g + (buf * kLB + j) * GS + 2 * c) = pf[i];
        }
    };

    const int T = gridDim.x * TM::PER_CTA;
    const int my = blockIdx.x * TM::PER_CTA + tm.team;
    int ci = snake_class(0, T, my);
    int M = 0, Mp = 0;
    if (ci < ncls) {
        class_orders(list_class(a, ci), M, Mp);
        fetch(M, Mp, M);
    }
    for (int r = 0; ci < ncls; ++r) {
        const int nc = class_case_count(M, Mp);
        const int nxt = snake_class(r + 1, T, my);
        int M2 = 0, Mp2 = 0;
        if (nxt < ncls) class_orders(list_class(a, nxt), M2, Mp2);

        double acc[NSUB8][NT][2];
#pragma unroll
        for (int p = 0; p < NSUB8; ++p)
#pragma unroll
            for (int n = 0; n < NT; ++n) acc[p][n][0] = acc[p][n][1] = 0.0;

        cs.seed(a, kc, a.normf[list_class(a, ci)], false, M, Mp);
        team_sync<TM::WARPS>(tm.team);   // the previous class is done with s_g
        stash(0);                        // chunk 0 (fetched ahead)
        fill_rc4(a, s_rc, M, M, Mp, lane);
#pragma unroll
        for (int s = 0; s < 8; ++s) gen_step<KT>(cs, s_d + s * DS, lane, s_rc + 4 * s);   // block 0
        team_sync<TM::WARPS>(tm.team);   // chunk 0 and block 0 rows visible
        if (M + kLB < B) fetch(M, Mp, M + kLB);
        else if (nxt < ncls) fetch(M2, Mp2, M2);

        const int nblk = (B - M + 7) >> 3;
        int cur = 0;
        for (int blk = 0; blk < nblk; ++blk) {
            const int off = 8 * blk;
            const double* dc = s_d + cur * 8 * DS;
            double* dn = s_d + (cur ^ 1) * 8 * DS;
            // B fragments for the two k-steps (degrees off + t4 and off + 4 + t4)
            const double* gb = s_g + ((((off >> 5) & 1) * kLB) + (off & (kLB - 1)) + t4) * GS;
            double bv0[NT], bv1[NT];
#pragma unroll
            for (int n = 0; n < NT; ++n) {
                const int v = 8 * (CS == 2 ? tm.h : n) + g;
                bv0[n] = gb[v];
                bv1[n] = gb[4 * GS + v];
            }
            auto mma_step = [&](int s) {
                // subtiles spread over the 8 steps: step s issues the first k-half of subtile s and
                // the second k-half of subtile (s + 4) mod 8, so that the two MMAs into one
                // accumulator are four steps apart (measured: -2 % per B=128 iDSOFT against both
                // halves in the same step); subtiles with p % 8 >= 4 thus take their second half
                // first, as dwt_batch_kernel does too
                constexpr int PS = (NSUB8 + 7) / 8;
                const int s1 = (s + 4) & 7;
                double av0[PS], av1[PS];
#pragma unroll
                for (int i = 0; i < PS; ++i) {
                    const int p = s + 8 * i, p1 = s1 + 8 * i;
                    if (p < NSUB8) av0[i] = dc[t4 * DS + 8 * p + g];
                    if (p1 < NSUB8) av1[i] = dc[(4 + t4) * DS + 8 * p1 + g];
                }
#pragma unroll
                for (int i = 0; i < PS; ++i) {
                    const int p = s + 8 * i;
                    if (p < NSUB8) {
#pragma unroll
                        for (int n = 0; n < NT; ++n) dmma(acc[p][n][0], acc[p][n][1], av0[i], bv0[n]);
                    }
                }
#pragma unroll
                for (int i = 0; i < PS; ++i) {
                    const int p1 = s1 + 8 * i;
                    if (p1 < NSUB8) {
#pragma unroll
                        for (int n = 0; n < NT; ++n) dmma(acc[p1][n][0], acc[p1][n][1], av1[i], bv1[n]);
                    }
                }
            };
            if (blk + 1 < nblk) {
                const int offn = off + 8;
                const bool boundary = (offn & (kLB - 1)) == 0;
                if (boundary) {
                    // publish the prefetched chunk (its buffer was last read two chunks ago)
                    stash((offn >> 5) & 1);
                    fill_rc4(a, s_rc, M + offn, M, Mp, lane);
                }
                const double* rcb = s_rc + 4 * (offn & (kLB - 1));
#pragma unroll
                for (int s = 0; s < 8; ++s) {
                    mma_step(s);
                    gen_step<KT>(cs, dn + s * DS, lane, rcb + 4 * s);
                }
                if (boundary) {
                    team_sync<TM::WARPS>(tm.team);   // new chunk visible; the old one no longer read
                    if (M + offn + kLB < B) fetch(M, Mp, M + offn + kLB);
                    else if (nxt < ncls) fetch(M2, Mp2, M2);
                } else {
                    __syncwarp();
                }
            } else {
#pragma unroll
                for (int s = 0; s < 8; ++s) mma_step(s);
            }
            cur ^= 1;
        }
#pragma unroll
        for (int n = 0; n < NT; ++n) {
            const int c = 4 * (CS == 2 ? tm.h : n) + t4;
            if (c < nc) {
                const PairCase pcase = class_case(M, Mp, c, N);
                double2* col = X + ((size_t)pcase.row * N + pcase.col) * N;
#pragma unroll
                for (int p = 0; p < NSUB8; ++p) {
                    const int k = tm.cw * KW + 8 * p + g;
                    // evict-first: the grid is next read by the inverse FFT from HBM (measured
                    // -1 % per iDSOFT at B = 128 and 256 against plain stores)
                    if (k < N) __stcs(col + (pcase.rev ? N - 1 - k : k), make_double2(acc[p][n][0], acc[p][n][1]));
                }
            }
        }
        ci = nxt;
        M = M2;
        Mp = Mp2;
    }
    if (a.zero_nyquist) nyquist_zero(X, B, (long long)blockIdx.x * blockDim.x + threadIdx.x, (long long)gridDim.x * blockDim.x);
}

__global__ void zero_nyquist_kernel(double2* X, int B)
{
    nyquist_zero(X, B, blockIdx.x * (long long)blockDim.x + threadIdx.x, (long long)gridDim.x * blockDim.x);
}

// Resident CTAs on all SMs (the persistent grid).
template <typename K>
int persistent_blocks(K kernel, size_t smem)
{
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kWarps * 32, smem) != cudaSuccess || per < 1) per = 1;
    return sms * per;
}

template <int KT, int TW, int CS>
cudaError_t launch_fwd(const double2* X, double2* coeffs, const DwtArgs& a, int nblocks, cudaStream_t s)
{
    const size_t smem = FwdSmem<KT>::doubles * sizeof(double);
    auto k = dwt_forward_kernel<KT, TW, CS>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (nblocks <= 0) nblocks = persistent_blocks(k, smem);
    k<<<nblocks, kWarps * 32, smem, s>>>(X, reinterpret_cast<double*>(coeffs), a);
    return cudaGetLastError();
}

template <int KT, int TW, int CS>
cudaError_t launch_inv(const double2* coeffs, double2* X, const DwtArgs& a, int nblocks, cudaStream_t s)
{
    const size_t smem = InvSmem<KT, kWarps / (TW * CS)>::doubles * sizeof(double);
    auto k = dwt_inverse_kernel<KT, TW, CS>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (nblocks <= 0) nblocks = persistent_blocks(k, smem);
    k<<<nblocks, kWarps * 32, smem, s>>>(coeffs, X, a);
    return cudaGetLastError();
}

}  // namespace

DwtArgs dwt_args_for(const BandTables& t)
{
    DwtArgs a;
    a.B = t.B;
    a.N = t.N;
    a.cosb = t.cosb;
    a.sinh = t.sinh;
    a.cosh = t.cosh;
    a.w = t.w;
    a.normf = t.normf;
    a.pw_sin = t.pw_sin;
    a.pw_cos = t.pw_cos;
    a.team_warps = dwt_team_warps(t.N);
    a.rc_cf = t.rc_cf;
    a.rc_f1 = t.rc_f1;
    a.classes = nullptr;
    a.n_classes = 0;
    a.zero_nyquist = 0;
    return a;
}

int dwt_team_warps(int N)
{
    if (N <= 128) return 1;
    return 4;
}

// Team shapes by beta-column count N = 2B: KT columns per lane, TW column warps, CS case warps
// (CS = 2 splits the eight cases over two warps that share the recurrence). g_case_split[dir]
// overrides CS for N > 64 (0 = default), as chosen by the autotuner.
int g_case_split[2] = {0, 0};

cudaError_t dwt_forward_launch(const double2* X, double2* coeffs, const DwtArgs& a, int nblocks, cudaStream_t s)
{
    const int N = a.N;
    const bool split = g_case_split[0] == 2;
    if (N <= 32) return launch_fwd<1, 1, 1>(X, coeffs, a, nblocks, s);
    if (N <= 64) return launch_fwd<2, 1, 1>(X, coeffs, a, nblocks, s);
    if (N <= 128) return split ? launch_fwd<4, 1, 2>(X, coeffs, a, nblocks, s) : launch_fwd<4, 1, 1>(X, coeffs, a, nblocks, s);
    if (N <= 256) return split ? launch_fwd<4, 2, 2>(X, coeffs, a, nblocks, s) : launch_fwd<2, 4, 1>(X, coeffs, a, nblocks, s);
    if (N <= 512) return split ? launch_fwd<8, 2, 2>(X, coeffs, a, nblocks, s) : launch_fwd<4, 4, 1>(X, coeffs, a, nblocks, s);
    return cudaErrorInvalidValue;
}

cudaError_t dwt_inverse_launch(const double2* coeffs, double2* X, const DwtArgs& a, int nblocks, cudaStream_t s)
{
    const int N = a.N;
    const bool split = g_case_split[1] == 2;
    if (N <= 32) return launch_inv<1, 1, 1>(coeffs, X, a, nblocks, s);
    if (N <= 64) return launch_inv<2, 1, 1>(coeffs, X, a, nblocks, s);
    if (N <= 128) return split ? launch_inv<4, 1, 2>(coeffs, X, a, nblocks, s) : launch_inv<4, 1, 1>(coeffs, X, a, nblocks, s);
    if (N <= 256) return split ? launch_inv<4, 2, 2>(coeffs, X, a, nblocks, s) : launch_inv<2, 4, 1>(coeffs, X, a, nblocks, s);
    if (N <= 512) return split ? launch_inv<8, 2, 2>(coeffs, X, a, nblocks, s) : launch_inv<4, 4, 1>(coeffs, X, a, nblocks, s);
    return cudaErrorInvalidValue;
}

void dwt_set_case_split(int dir, int cs)
{
    if (dir >= 0 && dir < 2) g_case_split[dir] = cs;
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
