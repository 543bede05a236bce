// Split-precision discrete Wigner transform on the 5th-generation tensor cores (sm_100a).
//
// For one order class (M, M') and four transforms of one bandwidth the DWT is a real matrix
// product (see dwt_batch.cu for the case/column conventions):
//   forward  F[l][c] = sum_k D[l][k] S[k][c]     l = M..B-1, k = beta samples, c = (transform, case, re/im)
//   inverse  S[k][c] = sum_l D[l][k] G[l][c]
// D (the Wigner-d rows, generated on chip by the FP64 three-term recurrence as in the FP64
// kernels) and S / G (FP64 data) are turned into fixed point and cut into six balanced 8-bit
// digits each: with a per-row scale r_l for D and a per-column power-of-two scale s_c for the
// other operand, x = round(v * scale * 2^47) = sum_i d_i 256^i, d_i in [-128, 127]. A digit is an
// integer that bf16 holds exactly. Digit planes are multiplied on the tensor cores
// (tcgen05.mma kind::f16, bf16 x bf16 -> f32 in tensor memory) and summed by significance
// e = sigma_D + sigma_S (sigma = 0 for the top digit); the planes with e > 5 are dropped. A
// product of two digit planes summed over K <= 256 is an integer below 2^22, so the f32
// accumulators of e <= 3 (at most four such sums) are exact, and the rounding in e = 4, 5 sits
// 2^-32 below the result. The epilogue reads the six accumulators back, adds the five correction
// planes smallest first in FP64 and the leading plane last in one rounding, then undoes the
// scales. FP64 stays for the seeds, the recurrence, the weights and that final sum.
//
// Layout: one CTA (8 warps) per SM holds all 512 tensor-memory columns; accumulator plane e of
// the 64 output columns sits at columns 64e .. 64e+63, one row per lane. The K dimension is
// cut into chunks of 32; a chunk's digit planes of D (A operand) and of S or G (B operand) are
// written to shared memory by all threads, double buffered, and one thread issues the chunk's
// MMAs; an mbarrier signalled by tcgen05.commit says when a buffer may be rewritten.
//   A (forward, K-major, rows l):   plane s, row r, k:   s*SA + (k/8)*PA + (r/8)*128 + (r%8)*16 + (k%8)*2
//   A (inverse, MN-major, rows k):  plane s, row m, l:   s*SA + (m/8)*PA + (l/8)*128 + (l%8)*16 + (m%8)*2
//   B (K-major, columns n = 64*s + c): (k/8)*PB + (n/8)*128 + (n%8)*16 + (k%8)*2
// Every wait is bounded; a wait that runs out sets *status and the CTA leaves after freeing its
// tensor memory.

#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "dwt.cuh"
#include "dwt_common.cuh"
#include "tc_sm100.cuh"

namespace pfsoft_dev {

namespace {

using namespace dwtk;

constexpr int kTT = 4;                 // transforms per work item
constexpr int kCols = 16 * kTT;        // output columns per digit plane
constexpr int kPlanes = 6;             // digits per operand
constexpr int kKC = 32;                // K per chunk
constexpr int kThreads = 256;
constexpr uint32_t kTmemCols = 512;
constexpr uint64_t kWaitNs = 2000000000ull;   // 2 s

// Shared memory (bytes). Both directions use the same buffer sizes.
constexpr int kPAf = 128 * 16 + 16;                 // forward A: k-group stride
constexpr int kSAf = (kKC / 8) * kPAf;              // forward A: plane stride
constexpr int kPAi = kKC * 16 + 16;                 // inverse A: m-group stride
constexpr int kSAi = (128 / 8) * kPAi;              // inverse A: plane stride
constexpr int kABuf = kPlanes * (kSAf > kSAi ? kSAf : kSAi);
constexpr int kPB = kPlanes * kCols * 16 + 16;      // B: k-group stride
constexpr int kBBuf = (kKC / 8) * kPB;
constexpr int kOffA = 0;
constexpr int kOffB = kOffA + 2 * kABuf;
constexpr int kOffRc = kOffB + 2 * kBBuf;            // recurrence coefficients, 256 rows x 4 doubles
constexpr int kOffRs = kOffRc + 256 * 4 * 8;         // row scale * 2^47 (256 doubles)
constexpr int kOffIrs = kOffRs + 256 * 8;            // 1 / row scale (256 doubles)
constexpr int kOffCs = kOffIrs + 256 * 8;            // column scale * 2^47 (64 doubles)
constexpr int kOffIcs = kOffCs + kCols * 8;          // 1 / column scale (64 doubles)
constexpr int kOffRed = kOffIcs + kCols * 8;         // reduction scratch (256 doubles)
constexpr int kOffMisc = kOffRed + 256 * 8;          // mbarriers, tmem address, item index
constexpr int kSmemBytes = kOffMisc + 64;

static_assert(kOffB % 16 == 0 && kABuf % 16 == 0 && kBBuf % 16 == 0, "operand buffers must stay 16-byte aligned");

constexpr double kTwo47 = 140737488355328.0;        // 2^47
// 2^52 + sum_{i<6} 128 * 256^i: adding it to x * 2^47 (|x| < 0.5) leaves round(x * 2^47) + C in
// the low 48 bits of the double, C making every byte a digit plus 128.
constexpr double kMagic = 4503599627370496.0 + 141289400074368.0;

struct SplitItem {
    int group, cls, t0, nt, tile, pad0, pad1, pad2;
};

// The six digits (most significant first) of the fixed-point value in a magic-biased double, as
// bf16 bit patterns.
__device__ __forceinline__ void to_digits(double z, uint16_t (&d)[kPlanes])
{
    const unsigned long long bits = (unsigned long long)__double_as_longlong(z);
    const uint32_t lo = (uint32_t)bits, hi = (uint32_t)(bits >> 32);
    const uint32_t bias = 0x4B000000u;
    uint32_t u[kPlanes];
    asm("prmt.b32 %0, %1, %2, 0x7441;" : "=r"(u[0]) : "r"(hi), "r"(bias));   // byte 5
    asm("prmt.b32 %0, %1, %2, 0x7440;" : "=r"(u[1]) : "r"(hi), "r"(bias));   // byte 4
    asm("prmt.b32 %0, %1, %2, 0x7443;" : "=r"(u[2]) : "r"(lo), "r"(bias));   // byte 3
    asm("prmt.b32 %0, %1, %2, 0x7442;" : "=r"(u[3]) : "r"(lo), "r"(bias));
    asm("prmt.b32 %0, %1, %2, 0x7441;" : "=r"(u[4]) : "r"(lo), "r"(bias));
    asm("prmt.b32 %0, %1, %2, 0x7440;" : "=r"(u[5]) : "r"(lo), "r"(bias));   // byte 0
#pragma unroll
    for (int s = 0; s < kPlanes; ++s) {
        const float f = __uint_as_float(u[s]) - 8388736.0f;   // 2^23 + 128: the digit, exactly
        d[s] = __bfloat16_as_ushort(__float2bfloat16_rn(f));
    }
}

__device__ __forceinline__ void store_digits(unsigned char* base, int plane_stride, double z)
{
    uint16_t d[kPlanes];
    to_digits(z, d);
#pragma unroll
    for (int s = 0; s < kPlanes; ++s) *reinterpret_cast<uint16_t*>(base + s * plane_stride) = d[s];
}

__device__ __forceinline__ void store_zero_digits(unsigned char* base, int plane_stride)
{
    const uint16_t zero = __bfloat16_as_ushort(__float2bfloat16_rn(0.0f));
#pragma unroll
    for (int s = 0; s < kPlanes; ++s) *reinterpret_cast<uint16_t*>(base + s * plane_stride) = zero;
}

// scale * 2^47 for a column whose largest magnitude is m (|v * scale| < 0.5), and 1 / scale
__device__ __forceinline__ void column_scale(double m, double& cs47, double& ics)
{
    if (!(m > 0.0)) {
        cs47 = kTwo47;
        ics = 1.0;
        return;
    }
    int e;
    frexp(m, &e);
    cs47 = ldexp(1.0, 46 - e);   // 2^-(e+1) * 2^47
    ics = ldexp(1.0, e + 1);
}

// Issues the MMAs of one K-step of 16: A plane s times the B planes 0 .. 5-s into accumulator
// planes s .. 5 (tensor-memory columns 64s ..), pieces of at most 256 columns.
__device__ __forceinline__ void issue_kstep(uint32_t tmem, uint32_t a_base, int a_plane, uint32_t a_lbo, uint32_t a_sbo,
                                            bool a_mn, uint32_t b_base, bool first)
{
#pragma unroll
    for (int s = 0; s < kPlanes; ++s) {
        const int total = kCols * (kPlanes - s);
#pragma unroll
        for (int n0 = 0; n0 < total; n0 += 256) {
            const int n = total - n0 < 256 ? total - n0 : 256;
            const uint64_t ad = tc::sdesc(a_base + s * a_plane, a_lbo, a_sbo);
            const uint64_t bd = tc::sdesc(b_base + (n0 / 8) * 128, kPB, 128);
            tc::mma_bf16(tmem + kCols * s + n0, ad, bd, tc::idesc_bf16(128, n, a_mn, false), !(first && s == 0));
        }
    }
}

// One transform's 16 columns of row `lane` of this warp's lane quarter: planes combined in FP64.
__device__ __forceinline__ void combine16(uint32_t taddr, int col, double (&out)[16])
{
    float v[16];
    double corr[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) corr[j] = 0.0;
#pragma unroll
    for (int e = kPlanes - 1; e >= 1; --e) {
        tc::tmem_ld16(taddr + kCols * e + col, v);
        tc::tmem_wait_ld();
        const double w = ldexp(1.0, -14 - 8 * e);
#pragma unroll
        for (int j = 0; j < 16; ++j) corr[j] = fma((double)v[j], w, corr[j]);
    }
    tc::tmem_ld16(taddr + col, v);
    tc::tmem_wait_ld();
#pragma unroll
    for (int j = 0; j < 16; ++j) out[j] = fma((double)v[j], 0x1p-14, corr[j]);
}

__device__ __forceinline__ double block_max(double v, double* red, int tid)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((tid & 31) == 0) red[tid >> 5] = v;
    __syncthreads();
    double m = red[0];
#pragma unroll
    for (int w = 1; w < kThreads / 32; ++w) m = fmax(m, red[w]);
    __syncthreads();
    return m;
}

template <int DIR>
__global__ void __launch_bounds__(kThreads, 1) dwt_split_kernel(const DwtGroup* __restrict__ groups,
                                                                 const SplitItem* __restrict__ items, int n_items,
                                                                 int* __restrict__ counter, int* __restrict__ status)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    double* s_rc = reinterpret_cast<double*>(smem + kOffRc);
    double* s_rs = reinterpret_cast<double*>(smem + kOffRs);
    double* s_irs = reinterpret_cast<double*>(smem + kOffIrs);
    double* s_cs = reinterpret_cast<double*>(smem + kOffCs);
    double* s_ics = reinterpret_cast<double*>(smem + kOffIcs);
    double* s_red = reinterpret_cast<double*>(smem + kOffRed);
    uint64_t* s_mbar = reinterpret_cast<uint64_t*>(smem + kOffMisc);        // [2]
    uint32_t* s_taddr = reinterpret_cast<uint32_t*>(smem + kOffMisc + 16);
    int* s_item = reinterpret_cast<int*>(smem + kOffMisc + 20);
    int* s_fail = reinterpret_cast<int*>(smem + kOffMisc + 24);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0) {
        tc::tmem_alloc(s_taddr, kTmemCols);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        tc::mbar_init(&s_mbar[0], 1);
        tc::mbar_init(&s_mbar[1], 1);
        tc::mbar_fence_init();
        *s_fail = 0;
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *s_taddr;
    const uint32_t smem_base = tc::smem_u32(smem);
    int commits[2] = {0, 0};   // commits issued to each buffer's mbarrier (uniform over the CTA)
    int chunk = 0;             // chunks issued by this CTA
    bool ok = true;

    auto wait_buffer = [&](int b) -> bool {   // the MMAs of the buffer's last chunk have finished
        if (commits[b] == 0) return true;
        return tc::mbar_wait_bounded(&s_mbar[b], (uint32_t)((commits[b] - 1) & 1), kWaitNs);
    };

    for (;;) {
        if (tid == 0) *s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int idx = *s_item;
        __syncthreads();
        if (idx >= n_items) break;
        const SplitItem it = items[idx];
        const DwtGroup gr = groups[it.group];
        const int B = gr.B, N = gr.N;
        int M, Mp;
        class_orders(it.cls, M, Mp);
        const int nc = class_case_count(M, Mp);
        const int R = B - M;   // degrees l = M .. B-1
        const double nf = gr.normf[it.cls];

        // recurrence coefficients of rows 0 .. R-1 (row r = degree M + r) and the row scales
        double wmax = 0.0;
        if (DIR == 0) {
            for (int k = tid; k < N; k += kThreads) wmax = fmax(wmax, fabs(gr.w[k]));
            wmax = block_max(wmax, s_red, tid);
        }
        for (int r = tid; r < R; r += kThreads) {
            double c1, f1, f2;
            rec_coef(M + r, M, Mp, c1, f1, f2);
            s_rc[4 * r] = c1;
            s_rc[4 * r + 1] = f1 * f2;
            s_rc[4 * r + 2] = f1;
            const double bound = (DIR == 0 ? wmax : 1.0) * sqrt((double)(M + r) + 0.5);
            const double rs = 0.49 / bound;
            s_rs[r] = rs * kTwo47;
            s_irs[r] = 1.0 / rs;
        }
        // column scales of the B operand over this item's K range
        {
            const int tq = tid >> 3, sub = tid & 7;            // (transform, case) pair, 8 threads each
            const int t = tq >> 3, q = tq & 7;
            double mre = 0.0, mim = 0.0;
            if (t < it.nt && q < nc) {
                const PairCase p = class_case(M, Mp, q, N);
                if (DIR == 0) {
                    const double2* col = gr.X[it.t0 + t] + ((size_t)p.row * N + p.col) * N;
                    for (int k = sub; k < N; k += 8) {
                        const double2 v = __ldg(col + k);
                        mre = fmax(mre, fabs(v.x));
                        mim = fmax(mim, fabs(v.y));
                    }
                } else {
                    const double norm = (double)(B * 2 * B) / kPi;
                    const double2* cf = gr.coeffs[it.t0 + t];
                    for (int r = sub; r < R; r += 8) {
                        const int l = M + r;
                        const double rs = 0.49 / sqrt((double)l + 0.5);
                        const double2 v = __ldg(cf + coef_index(l, p.m1, p.m2));
                        const double f = norm / rs;
                        mre = fmax(mre, fabs(f * v.x));
                        mim = fmax(mim, fabs(f * v.y));
                    }
                }
            }
#pragma unroll
            for (int o = 4; o > 0; o >>= 1) {
                mre = fmax(mre, __shfl_xor_sync(0xffffffffu, mre, o));
                mim = fmax(mim, __shfl_xor_sync(0xffffffffu, mim, o));
            }
            if (sub == 0) {
                column_scale(mre, s_cs[16 * t + 2 * q], s_ics[16 * t + 2 * q]);
                column_scale(mim, s_cs[16 * t + 2 * q + 1], s_ics[16 * t + 2 * q + 1]);
            }
        }
        __syncthreads();

        if (DIR == 0) {
            // ------------------------------------------------------------------ forward
            // generation: warp w handles rows of group g (16 rows), lane = beta column of the chunk;
            // it runs the recurrence from the seed and stores only its own rows.
            const int g = warp < 4 ? warp : 11 - warp;
            const int r_lo = 16 * g, r_hi = min(16 * g + 16, R);
            const int nchunks = N / kKC;
            for (int kc = 0; kc < nchunks; ++kc) {
                const int b = chunk & 1;
                if (!wait_buffer(b)) ok = false;
                ok = !__syncthreads_or(!ok);
                if (!ok) break;
                unsigned char* A = smem + kOffA + b * kABuf;
                unsigned char* Bm = smem + kOffB + b * kBBuf;
                const int k = kc * kKC + lane;
                if (r_lo < R) {
                    const double cb = gr.cosb[k];
                    int sc = 0;
                    double dcur = seed_value(nf * gr.w[k], gr.pw_sin[(size_t)(M - Mp) * N + k],
                                             gr.pw_cos[(size_t)(M + Mp) * N + k], sc);
                    double dprev = 0.0;
                    unsigned char* colp = A + (lane >> 3) * kPAf + (lane & 7) * 2;
                    for (int r = 0; r < r_hi; ++r) {
                        if (r >= r_lo) {
                            const double v = sc ? 0.0 : dcur;
                            store_digits(colp + (r >> 3) * 128 + (r & 7) * 16, kSAf, fma(v, s_rs[r], kMagic));
                        }
                        const double2 ca = *reinterpret_cast<const double2*>(s_rc + 4 * r);
                        const double t = fma(s_rc[4 * r + 2], cb, ca.y);
                        const double nx = fma(ca.x, dprev, dcur * t);
                        dprev = dcur;
                        dcur = nx;
                        if (sc && fabs(dcur) >= 0x1p300) {
                            dcur *= 0x1p-600;
                            dprev *= 0x1p-600;
                            --sc;
                        }
                    }
                }
                // B operand: S digits of the chunk, column n = 16 t + 2 q + (re, im)
                for (int i = 0; i < 4; ++i) {
                    const int e = tid + kThreads * i;
                    const int tq = e >> 5, kl = e & 31;
                    const int t = tq >> 3, q = tq & 7;
                    const int n = 16 * t + 2 * q;
                    unsigned char* p0 = Bm + (kl >> 3) * kPB + (n >> 3) * 128 + (n & 7) * 16 + (kl & 7) * 2;
                    if (t < it.nt && q < nc) {
                        const PairCase p = class_case(M, Mp, q, N);
                        const int kk = kc * kKC + kl;
                        const double2 v = __ldg(gr.X[it.t0 + t] + ((size_t)p.row * N + p.col) * N + (p.rev ? N - 1 - kk : kk));
                        store_digits(p0, kCols * 16, fma(v.x, s_cs[n], kMagic));
                        store_digits(p0 + 16, kCols * 16, fma(v.y, s_cs[n + 1], kMagic));
                    } else {
                        store_zero_digits(p0, kCols * 16);
                        store_zero_digits(p0 + 16, kCols * 16);
                    }
                }
                tc::fence_proxy_async();
                tc::fence_before_sync();
                __syncthreads();
                if (tid == 0) {
                    tc::fence_after_sync();
                    const uint32_t a0 = smem_base + kOffA + b * kABuf, b0 = smem_base + kOffB + b * kBBuf;
                    issue_kstep(tmem, a0, kSAf, kPAf, 128, false, b0, kc == 0);
                    issue_kstep(tmem, a0 + 2 * kPAf, kSAf, kPAf, 128, false, b0 + 2 * kPB, false);
                    tc::mma_commit(&s_mbar[b]);
                }
                ++commits[b];
                ++chunk;
            }
            if (!ok) break;
            // epilogue: row r = 32 (warp % 4) + lane, transforms 2 (warp / 4) + {0, 1}
            if (!wait_buffer((chunk - 1) & 1)) ok = false;
            ok = !__syncthreads_or(!ok);
            if (!ok) break;
            tc::fence_after_sync();
            const int r = 32 * (warp & 3) + lane, l = M + r;
            const uint32_t taddr = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
            const double norm = kPi / (double)(B * 2 * B);   // src/fn_dsoft.cpp:119
            for (int tt = 0; tt < 2; ++tt) {
                const int t = 2 * (warp >> 2) + tt;
                double v[16];
                combine16(taddr, 16 * t, v);
                if (r < R && t < it.nt) {
                    double2* out = gr.coeffs[it.t0 + t];
                    const double irs = s_irs[r];
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        if (q < nc) {
                            const PairCase p = class_case(M, Mp, q, N);
                            const double f = norm * case_sign(p, l, M) * irs;
                            out[coef_index(l, p.m1, p.m2)] =
                                make_double2(f * v[2 * q] * s_ics[16 * t + 2 * q], f * v[2 * q + 1] * s_ics[16 * t + 2 * q + 1]);
                        }
                    }
                }
            }
            tc::fence_before_sync();
            __syncthreads();   // accumulators are overwritten by the next item
        } else {
            // ------------------------------------------------------------------ inverse
            // warps 0-3 generate: thread = beta column m of the tile, rows advance over the chunks
            const int kb = 128 * it.tile;
            const int m = tid & 127, k = kb + m;
            const bool gen = tid < 128;
            double cb = 0.0, dcur = 0.0, dprev = 0.0;
            int sc = 0;
            if (gen && k < N) {
                cb = gr.cosb[k];
                dcur = seed_value(nf, gr.pw_sin[(size_t)(M - Mp) * N + k], gr.pw_cos[(size_t)(M + Mp) * N + k], sc);
            }
            const double norm = (double)(B * 2 * B) / kPi;   // src/fn_idsoft.cpp:109
            const int nchunks = (R + kKC - 1) / kKC;
            for (int lc = 0; lc < nchunks; ++lc) {
                const int b = chunk & 1;
                if (!wait_buffer(b)) ok = false;
                ok = !__syncthreads_or(!ok);
                if (!ok) break;
                unsigned char* A = smem + kOffA + b * kABuf;
                unsigned char* Bm = smem + kOffB + b * kBBuf;
                const int r0 = lc * kKC;
                if (gen) {
                    unsigned char* colp = A + (m >> 3) * kPAi + (m & 7) * 2;
                    for (int j = 0; j < kKC; ++j) {
                        const int r = r0 + j;
                        unsigned char* p = colp + (j >> 3) * 128 + (j & 7) * 16;
                        if (r < R && k < N) {
                            const double v = sc ? 0.0 : dcur;
                            store_digits(p, kSAi, fma(v, s_rs[r], kMagic));
                            const double2 ca = *reinterpret_cast<const double2*>(s_rc + 4 * r);
                            const double t = fma(s_rc[4 * r + 2], cb, ca.y);
                            const double nx = fma(ca.x, dprev, dcur * t);
                            dprev = dcur;
                            dcur = nx;
                            if (sc && fabs(dcur) >= 0x1p300) {
                                dcur *= 0x1p-600;
                                dprev *= 0x1p-600;
                                --sc;
                            }
                        } else {
                            store_zero_digits(p, kSAi);
                        }
                    }
                } else {
                    // B operand: G digits, rows l of the chunk, column n = 16 t + 2 q + (re, im);
                    // G = norm * sign * coefficient / (row scale), scaled per column
                    const int u = tid - 128;
                    for (int i = 0; i < 8; ++i) {
                        const int e = u + 128 * i;            // (t, q) pair e / 32, row j = e % 32
                        const int tq = e >> 5, j = e & 31;
                        const int t = tq >> 3, q = tq & 7;
                        const int n = 16 * t + 2 * q, r = r0 + j;
                        unsigned char* p0 = Bm + (j >> 3) * kPB + (n >> 3) * 128 + (n & 7) * 16 + (j & 7) * 2;
                        if (t < it.nt && q < nc && r < R) {
                            const PairCase p = class_case(M, Mp, q, N);
                            const int l = M + r;
                            const double2 x = __ldg(gr.coeffs[it.t0 + t] + coef_index(l, p.m1, p.m2));
                            const double f = norm * case_sign(p, l, M) * s_irs[r];
                            store_digits(p0, kCols * 16, fma(f * x.x, s_cs[n], kMagic));
                            store_digits(p0 + 16, kCols * 16, fma(f * x.y, s_cs[n + 1], kMagic));
                        } else {
                            store_zero_digits(p0, kCols * 16);
                            store_zero_digits(p0 + 16, kCols * 16);
                        }
                    }
                }
                tc::fence_proxy_async();
                tc::fence_before_sync();
                __syncthreads();
                if (tid == 0) {
                    tc::fence_after_sync();
                    const uint32_t a0 = smem_base + kOffA + b * kABuf, b0 = smem_base + kOffB + b * kBBuf;
                    issue_kstep(tmem, a0, kSAi, 128, kPAi, true, b0, lc == 0);
                    if (r0 + 16 < R) issue_kstep(tmem, a0 + 256, kSAi, 128, kPAi, true, b0 + 2 * kPB, false);
                    tc::mma_commit(&s_mbar[b]);
                }
                ++commits[b];
                ++chunk;
            }
            if (!ok) break;
            if (!wait_buffer((chunk - 1) & 1)) ok = false;
            ok = !__syncthreads_or(!ok);
            if (!ok) break;
            tc::fence_after_sync();
            // epilogue: row m = 32 (warp % 4) + lane of the tile, transforms 2 (warp / 4) + {0, 1}
            const int mm = 32 * (warp & 3) + lane, kk = kb + mm;
            const uint32_t taddr = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
            for (int tt = 0; tt < 2; ++tt) {
                const int t = 2 * (warp >> 2) + tt;
                double v[16];
                combine16(taddr, 16 * t, v);
                if (kk < N && t < it.nt) {
                    double2* X = gr.X[it.t0 + t];
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        if (q < nc) {
                            const PairCase p = class_case(M, Mp, q, N);
                            X[((size_t)p.row * N + p.col) * N + (p.rev ? N - 1 - kk : kk)] =
                                make_double2(v[2 * q] * s_ics[16 * t + 2 * q], v[2 * q + 1] * s_ics[16 * t + 2 * q + 1]);
                        }
                    }
                }
            }
            tc::fence_before_sync();
            __syncthreads();
        }
    }
    // leave: a failed wait may leave MMAs in flight; give them the same bound once more
    if (!ok) {
        if (tid == 0) {
            *s_fail = 1;
            atomicExch(status, 1);
        }
        for (int b = 0; b < 2; ++b) wait_buffer(b);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, kTmemCols);
}

}  // namespace

bool dwt_split_supported(int B) { return B >= 16 && B <= 128 && B % 16 == 0; }

size_t dwt_split_item_bytes() { return sizeof(SplitItem); }

// Work items of one group for the split kernel: forward (class, 4 transforms), inverse (class,
// 128 beta columns, 4 transforms); longest first.
void dwt_split_items(int direction, int group, int B, int T, std::vector<unsigned char>& out, int* n_items)
{
    std::vector<std::pair<int, SplitItem> > v;
    const int N = 2 * B, tiles = direction == 0 ? 1 : (N + 127) / 128;
    for (int c = 0; c < num_classes(B); ++c) {
        int M, Mp;
        class_orders(c, M, Mp);
        for (int t0 = 0; t0 < T; t0 += kTT)
            for (int tile = 0; tile < tiles; ++tile) {
                SplitItem it{group, c, t0, T - t0 < kTT ? T - t0 : kTT, tile, 0, 0, 0};
                v.push_back(std::make_pair(B - M, it));
            }
    }
    std::stable_sort(v.begin(), v.end(), [](const std::pair<int, SplitItem>& a, const std::pair<int, SplitItem>& b) {
        return a.first > b.first;
    });
    out.resize(v.size() * sizeof(SplitItem));
    for (size_t i = 0; i < v.size(); ++i) std::memcpy(out.data() + i * sizeof(SplitItem), &v[i].second, sizeof(SplitItem));
    *n_items = (int)v.size();
}

int g_split_sms = 0;

cudaError_t dwt_split_prepare()
{
    cudaError_t e = cudaFuncSetAttribute(dwt_split_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(dwt_split_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
    int dev = 0;
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&g_split_sms, cudaDevAttrMultiProcessorCount, dev);
    return e;
}

cudaError_t dwt_split_launch(int direction, const DwtGroup* d_groups, const void* d_items, int n_items, int* d_counter,
                             int* d_status, cudaStream_t s)
{
    if (n_items <= 0) return cudaSuccess;
    if (g_split_sms <= 0) return cudaErrorNotReady;   // dwt_split_prepare was not called
    const int blocks = n_items < g_split_sms ? n_items : g_split_sms;
    const SplitItem* it = static_cast<const SplitItem*>(d_items);
    if (direction == 0)
        dwt_split_kernel<0><<<blocks, kThreads, kSmemBytes, s>>>(d_groups, it, n_items, d_counter, d_status);
    else
        dwt_split_kernel<1><<<blocks, kThreads, kSmemBytes, s>>>(d_groups, it, n_items, d_counter, d_status);
    return cudaGetLastError();
}

}  // namespace pfsoft_dev
