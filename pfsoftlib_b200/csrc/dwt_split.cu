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
//   A (forward, MN-major, rows l):  plane s, row r, beta k:  s*SA + (r/8)*PA + (k/8)*128 + (k%8)*16 + (r%8)*2
//   A (inverse, K-major, rows k):   plane s, row m, degree j: s*SA + (j/8)*PA + (m/8)*128 + (m%8)*16 + (j%8)*2
//   B (K-major, columns n = 64*s + c): (k/8)*PB + (n/8)*128 + (n%8)*16 + (k%8)*2
// so that a 16-byte unit holds eight consecutive degrees of one beta column (A) or eight
// consecutive K of one column (B): each thread writes whole units.
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
constexpr int kGenWarps = 7;           // forward: warps 1-7 generate, warp 0 issues the MMAs
constexpr uint32_t kTmemCols = 512;
constexpr uint64_t kWaitNs = 2000000000ull;   // 2 s

// Shared memory (bytes). Both directions use the same buffer sizes.
constexpr int kPAk = 128 * 16 + 16;                 // K-major A (inverse): stride of 8-wide K groups
constexpr int kSAk = (kKC / 8) * kPAk;              // K-major A: plane stride
constexpr int kPAm = kKC * 16 + 16;                 // MN-major A (forward): stride of 8-row M groups
constexpr int kSAm = (128 / 8) * kPAm;              // MN-major A: plane stride
constexpr int kABuf = kPlanes * (kSAk > kSAm ? kSAk : kSAm);
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
constexpr int kOffCk = kOffRed + 256 * 8;           // forward: recurrence state every 16 rows, [8][256] double2
constexpr int kOffCkSc = kOffCk + 8 * 256 * 16;      // forward: scale count at those rows, [8][256] int8
constexpr int kOffCb = kOffCkSc + 8 * 256;           // forward: cos(beta) per column (256 doubles)
constexpr int kOffCase = kOffCb + 256 * 8;          // the item's symmetry cases (8 PairCase)
constexpr int kOffMisc = kOffCase + 8 * 32;          // mbarriers, tmem address, item index
constexpr int kSmemBytes = kOffMisc + 64;
static_assert(kSmemBytes <= 227 * 1024, "shared memory");

static_assert(kOffB % 16 == 0 && kABuf % 16 == 0 && kBBuf % 16 == 0, "operand buffers must stay 16-byte aligned");
static_assert(sizeof(PairCase) <= 32, "case table entry");

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
    // f = u - 128 exactly; an integer of at most 8 significant bits has zero low 16 bits in
    // binary32, so its bf16 pattern is the high half
#pragma unroll
    for (int s = 0; s < kPlanes; ++s) {
        const float f = __uint_as_float(u[s]) - 8388736.0f;   // 2^23 + 128
        d[s] = (uint16_t)(__float_as_uint(f) >> 16);
    }
}

// Digits of eight values that share a 16-byte core-matrix unit (eight consecutive K or MN
// positions of one row), one 32-bit word per two values and plane.
struct Digits8 {
    uint32_t w[kPlanes][4];
};

__device__ __forceinline__ void put_digits(Digits8& D, int j, double z)
{
    uint16_t d[kPlanes];
    to_digits(z, d);
#pragma unroll
    for (int s = 0; s < kPlanes; ++s) {
        if (j & 1)
            D.w[s][j >> 1] |= (uint32_t)d[s] << 16;
        else
            D.w[s][j >> 1] = d[s];
    }
}

__device__ __forceinline__ void store_unit8(unsigned char* base, int plane_stride, const Digits8& D)
{
#pragma unroll
    for (int s = 0; s < kPlanes; ++s)
        *reinterpret_cast<uint4*>(base + s * plane_stride) = make_uint4(D.w[s][0], D.w[s][1], D.w[s][2], D.w[s][3]);
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
                                            bool a_mn, uint32_t b_base, bool first, int M = 128)
{
#pragma unroll
    for (int s = 0; s < kPlanes; ++s) {
        const int total = kCols * (kPlanes - s);
#pragma unroll
        for (int n0 = 0; n0 < total; n0 += 256) {
            const int n = total - n0 < 256 ? total - n0 : 256;
            const uint64_t ad = tc::sdesc(a_base + s * a_plane, a_lbo, a_sbo);
            const uint64_t bd = tc::sdesc(b_base + (n0 / 8) * 128, kPB, 128);
            tc::mma_bf16(tmem + kCols * s + n0, ad, bd, tc::idesc_bf16(M, n, a_mn, false), !(first && s == 0));
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

    // the recurrence step d(l+1) = d(l) (f1 f2 + f1 cos beta) + c1 d(l-1) (fn_dwt.hpp:167-199),
    // ordered so that only one FMA depends on d(l); columns whose seed was scaled by 2^600 store 0
    // until they are back in range
    auto step = [&](double& dcur, double& dprev, int& sc, double cb, int r) {
        const double2 ca = *reinterpret_cast<const double2*>(s_rc + 4 * r);
        const double t = fma(s_rc[4 * r + 2], cb, ca.y);
        const double u = ca.x * dprev;
        const double nx = fma(dcur, t, u);
        dprev = dcur;
        dcur = nx;
        if (sc && fabs(dcur) >= 0x1p300) {
            dcur *= 0x1p-600;
            dprev *= 0x1p-600;
            --sc;
        }
    };

    PairCase* s_case = reinterpret_cast<PairCase*>(smem + kOffCase);
    int wgroup = -1;       // group whose largest weight is in wmax
    double wmax = 0.0;
    if (tid == kThreads - 1) *s_item = atomicAdd(counter, 1);
    for (;;) {
        __syncthreads();
        const int idx = *s_item;
        __syncthreads();
        if (idx >= n_items) break;
        // the next item, read after this one (the last warp has the least generation work)
        if (tid == kThreads - 1) *s_item = atomicAdd(counter, 1);
        const SplitItem it = items[idx];
        const DwtGroup gr = groups[it.group];
        const int B = gr.B, N = gr.N;
        int M, Mp;
        class_orders(it.cls, M, Mp);
        const int nc = class_case_count(M, Mp);
        const int R = B - M;   // degrees l = M .. B-1
        const double nf = gr.normf[it.cls];

        // recurrence coefficients of rows 0 .. R-1 (row r = degree M + r) and the row scales
        if (DIR == 0 && it.group != wgroup) {
            double w = 0.0;
            for (int k = tid; k < N; k += kThreads) w = fmax(w, fabs(gr.w[k]));
            wmax = block_max(w, s_red, tid);
            wgroup = it.group;
        }
        const long long rc0 = rc_offset(B, M, Mp);
        for (int r = tid; r < R; r += kThreads) {   // M + r < B: every row has a table entry
            const double2 cf = __ldg(gr.rc_cf + rc0 + r);
            s_rc[4 * r] = cf.x;
            s_rc[4 * r + 1] = cf.y;
            s_rc[4 * r + 2] = __ldg(gr.rc_f1 + rc0 + r);
            const double bound = (DIR == 0 ? wmax : 1.0) * sqrt((double)(M + r) + 0.5);
            const double rs = 0.49 / bound;
            s_rs[r] = rs * kTwo47;
            s_irs[r] = 1.0 / rs;
        }
        // column scales of the B operand: largest magnitudes precomputed per bin (forward) or per
        // (class, case) (inverse) in the table past each transform's spectrum (dwt_split_scales)
        if (tid < kCols / 2) {
            const int t = tid >> 3, q = tid & 7;
            double2 mx = make_double2(0.0, 0.0);
            if (t < it.nt && q < nc) {
                const double2* aux = gr.X[it.t0 + t] + (size_t)N * N * N;
                if (DIR == 0) {
                    const PairCase p = class_case(M, Mp, q, N);
                    mx = aux[(size_t)p.row * N + p.col];
                } else {
                    mx = aux[(size_t)it.cls * 8 + q];
                }
            }
            column_scale(mx.x, s_cs[16 * t + 2 * q], s_ics[16 * t + 2 * q]);
            column_scale(mx.y, s_cs[16 * t + 2 * q + 1], s_ics[16 * t + 2 * q + 1]);
        }
        if (tid < 8) s_case[tid] = class_case(M, Mp, tid < nc ? tid : 0, N);
        __syncthreads();

        if (DIR == 0) {
            // ------------------------------------------------------------------ forward
            // checkpoints: thread = beta column runs the recurrence over all rows once and keeps its
            // state at every 16th row; each chunk then regenerates its rows 16 at a time
            double2* s_ck = reinterpret_cast<double2*>(smem + kOffCk);
            signed char* s_cksc = reinterpret_cast<signed char*>(smem + kOffCkSc);
            double* s_cb = reinterpret_cast<double*>(smem + kOffCb);
            // warps 1-7 regenerate rows in contiguous ranges of `rows` rows (a multiple of 8, so
            // that a thread writes whole 16-byte units); warp 0 issues the MMAs
            const int rows = (((R + kGenWarps - 1) / kGenWarps) + 7) & ~7;
            if (tid < N) {
                const int k = tid;
                const double cb = gr.cosb[k];
                s_cb[k] = cb;
                int sc = 0;
                double dcur = seed_value(nf * gr.w[k], gr.pw_sin[(size_t)(M - Mp) * N + k],
                                         gr.pw_cos[(size_t)(M + Mp) * N + k], sc);
                double dprev = 0.0;
                for (int r = 0, g = 0, next = 0; r < R; ++r) {
                    if (r == next) {
                        s_ck[g * 256 + k] = make_double2(dcur, dprev);
                        s_cksc[g * 256 + k] = (signed char)sc;
                        ++g;
                        next += rows;
                    }
                    step(dcur, dprev, sc, cb, r);
                }
            }
            // B operand tasks of the generating threads u = tid - 32: task e = u + 224 i is column
            // n = e % 64 (transform n / 16, case (n / 2) % 8, re / im n % 2) at beta octet e / 64;
            // its eight values are prefetched one chunk ahead
            constexpr int kTasks = kCols * (kKC / 8);
            constexpr int kSv = (kTasks + 32 * kGenWarps - 1) / (32 * kGenWarps);
            double sv[kSv][8];
            auto load_s = [&](int kc) {
#pragma unroll
                for (int i = 0; i < kSv; ++i) {
                    const int e = (tid - 32) + 32 * kGenWarps * i;
                    const int n = e & (kCols - 1), o = e / kCols;
                    const int t = n >> 4, q = (n >> 1) & 7;
                    const bool live = e < kTasks && t < it.nt && q < nc;
                    const PairCase p = s_case[q];
                    const double* col = live ? reinterpret_cast<const double*>(gr.X[it.t0 + t] + ((size_t)p.row * N + p.col) * N) + (n & 1)
                                             : nullptr;
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const int kk = kc * kKC + 8 * o + j;
                        sv[i][j] = live ? __ldg(col + 2 * (p.rev ? N - 1 - kk : kk)) : 0.0;
                    }
                }
            };
            if (warp > 0) load_s(0);
            __syncthreads();
            const bool m64 = R <= 64;   // one M = 64 tile: rows 16q .. 16q+15 in lanes 32q .. 32q+15
            const int gw = warp - 1;
            const int r_lo = warp > 0 ? gw * rows : R, r_hi = min(r_lo + rows, (R + 7) & ~7);
            const int nchunks = N / kKC;
            for (int kc = 0; kc < nchunks; ++kc) {
                const int b = chunk & 1;
                if (tid == 0 && !wait_buffer(b)) ok = false;   // one waiter; the barrier below holds the rest
                ok = !__syncthreads_or(!ok);
                if (!ok) break;
                unsigned char* A = smem + kOffA + b * kABuf;
                unsigned char* Bm = smem + kOffB + b * kBBuf;
                if (warp > 0) {
                    // B operand: one 16-byte unit per plane for eight consecutive beta of column n
#pragma unroll
                    for (int i = 0; i < kSv; ++i) {
                        const int e = (tid - 32) + 32 * kGenWarps * i;
                        if (e < kTasks) {
                            const int n = e & (kCols - 1), o = e / kCols;
                            Digits8 D;
#pragma unroll
                            for (int j = 0; j < 8; ++j) put_digits(D, j, fma(sv[i][j], s_cs[n], kMagic));
                            store_unit8(Bm + o * kPB + (n >> 3) * 128 + (n & 7) * 16, kCols * 16, D);
                        }
                    }
                    if (kc + 1 < nchunks) load_s(kc + 1);   // in flight during the generation below
                    // A operand (MN-major): thread = beta column lane of the chunk, rows r_lo .. r_hi-1
                    // from the checkpoint, one 16-byte unit per plane for eight rows
                    if (r_lo < r_hi) {
                        const int k = kc * kKC + lane;
                        const double cb = s_cb[k];
                        const double2 st = s_ck[gw * 256 + k];
                        int sc = s_cksc[gw * 256 + k];
                        double dcur = st.x, dprev = st.y;
                        unsigned char* colp = A + (lane >> 3) * 128 + (lane & 7) * 16;
                        for (int r8 = r_lo; r8 < r_hi; r8 += 8) {
                            Digits8 D;
#pragma unroll
                            for (int j = 0; j < 8; ++j) {
                                const int r = r8 + j;
                                if (r < R) {
                                    put_digits(D, j, fma(sc ? 0.0 : dcur, s_rs[r], kMagic));
                                    step(dcur, dprev, sc, cb, r);
                                } else {
                                    put_digits(D, j, kMagic);
                                }
                            }
                            store_unit8(colp + (r8 >> 3) * kPAm, kSAm, D);
                        }
                    }
                }
                tc::fence_proxy_async();
                tc::fence_before_sync();
                __syncthreads();
                if (tid == 0) {
                    tc::fence_after_sync();
                    const uint32_t a0 = smem_base + kOffA + b * kABuf, b0 = smem_base + kOffB + b * kBBuf;
                    const int mt = m64 ? 64 : 128;
                    issue_kstep(tmem, a0, kSAm, 128, kPAm, true, b0, kc == 0, mt);
                    issue_kstep(tmem, a0 + 256, kSAm, 128, kPAm, true, b0 + 2 * kPB, false, mt);
                    tc::mma_commit(&s_mbar[b]);
                }
                ++commits[b];
                ++chunk;
            }
            if (!ok) break;
            // epilogue: lane quarter warp % 4, transforms 2 (warp / 4) + {0, 1}
            if (tid == 0 && !wait_buffer((chunk - 1) & 1)) ok = false;
            ok = !__syncthreads_or(!ok);
            if (!ok) break;
            tc::fence_after_sync();
            const int r = m64 ? (lane < 16 ? 16 * (warp & 3) + lane : 1 << 20) : 32 * (warp & 3) + lane;
            const int l = M + r;
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
                            const PairCase p = s_case[q];
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
            // warps 0-3 generate: thread = beta column m of the tile, rows advance over the chunks;
            // warps 4-7 bring in the coefficients
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
            // B operand tasks of the loading threads u = tid - 160 (warps 5-7; warp 4 issues the
            // MMAs): task e = u + 96 i is column n = e % 64 at row octet e / 64 of the chunk; its
            // eight coefficients are prefetched one chunk ahead and signed and scaled when stored
            constexpr int kTasks = kCols * (kKC / 8);
            constexpr int kGv = (kTasks + 95) / 96;
            const bool loader = tid >= 160;
            double gv[kGv][8];
            auto load_g = [&](int lc) {   // raw loads only, every address in range, so they all fly at once
#pragma unroll
                for (int i = 0; i < kGv; ++i) {
                    const int e = min((tid - 160) + 96 * i, kTasks - 1);
                    const int n = e & (kCols - 1), o = e / kCols;
                    const int t = min(n >> 4, it.nt - 1), q = (n >> 1) & 7;
                    const PairCase p = s_case[q];
                    const double* cf = reinterpret_cast<const double*>(gr.coeffs[it.t0 + t]) + (n & 1);
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const int l = M + min(lc * kKC + 8 * o + j, R - 1);
                        gv[i][j] = __ldg(cf + 2 * coef_index(l, p.m1, p.m2));
                    }
                }
            };
            if (loader) load_g(0);
            for (int lc = 0; lc < nchunks; ++lc) {
                const int b = chunk & 1;
                if (tid == 0 && !wait_buffer(b)) ok = false;   // one waiter; the barrier below holds the rest
                ok = !__syncthreads_or(!ok);
                if (!ok) break;
                unsigned char* A = smem + kOffA + b * kABuf;
                unsigned char* Bm = smem + kOffB + b * kBBuf;
                const int r0 = lc * kKC;
                if (gen) {
                    // A operand (K-major): thread = beta column m of the tile, one 16-byte unit per
                    // plane for eight consecutive rows
                    unsigned char* colp = A + (m >> 3) * 128 + (m & 7) * 16;
#pragma unroll 1
                    for (int j8 = 0; j8 < kKC; j8 += 8) {
                        Digits8 D;
#pragma unroll
                        for (int jj = 0; jj < 8; ++jj) {
                            const int r = r0 + j8 + jj;
                            if (r < R && k < N) {
                                put_digits(D, jj, fma(sc ? 0.0 : dcur, s_rs[r], kMagic));
                                step(dcur, dprev, sc, cb, r);
                            } else {
                                put_digits(D, jj, kMagic);
                            }
                        }
                        store_unit8(colp + (j8 >> 3) * kPAk, kSAk, D);
                    }
                } else if (loader) {
#pragma unroll
                    for (int i = 0; i < kGv; ++i) {
                        const int e = (tid - 160) + 96 * i;
                        if (e < kTasks) {
                            const int n = e & (kCols - 1), o = e / kCols;
                            const int t = n >> 4, q = (n >> 1) & 7;
                            const bool live = t < it.nt && q < nc;
                            const PairCase p = s_case[q];
                            Digits8 D;
#pragma unroll
                            for (int j = 0; j < 8; ++j) {
                                // G = norm * sign * coefficient / (row scale), zero outside the class
                                const int r = r0 + 8 * o + j, l = M + r;
                                const double g = (live && r < R) ? norm * case_sign(p, l, M) * s_irs[r] * gv[i][j] : 0.0;
                                put_digits(D, j, fma(g, s_cs[n], kMagic));
                            }
                            store_unit8(Bm + o * kPB + (n >> 3) * 128 + (n & 7) * 16, kCols * 16, D);
                        }
                    }
                    if (lc + 1 < nchunks) load_g(lc + 1);
                }
                tc::fence_proxy_async();
                tc::fence_before_sync();
                __syncthreads();
                if (tid == 128) {
                    tc::fence_after_sync();
                    const uint32_t a0 = smem_base + kOffA + b * kABuf, b0 = smem_base + kOffB + b * kBBuf;
                    issue_kstep(tmem, a0, kSAk, kPAk, 128, false, b0, lc == 0);
                    if (r0 + 16 < R) issue_kstep(tmem, a0 + 2 * kPAk, kSAk, kPAk, 128, false, b0 + 2 * kPB, false);
                    tc::mma_commit(&s_mbar[b]);
                }
                ++commits[b];
                ++chunk;
            }
            if (!ok) break;
            if (tid == 0 && !wait_buffer((chunk - 1) & 1)) ok = false;
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
                            const PairCase p = s_case[q];
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
        if (tid == 0)
            for (int b = 0; b < 2; ++b) wait_buffer(b);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, kTmemCols);
}

// Largest |re|, |im| over beta of every bin column of a spectrum, into the table past it
// (forward operand scales). One warp per bin, gridDim.z = transforms.
__global__ void split_binmax_kernel(double2* const* X, int N)
{
    const long long bin = (long long)blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (bin >= (long long)N * N) return;
    const double2* col = X[blockIdx.z] + bin * N;
    double mre = 0.0, mim = 0.0;
    for (int k = lane; k < N; k += 32) {
        const double2 v = __ldg(col + k);
        mre = fmax(mre, fabs(v.x));
        mim = fmax(mim, fabs(v.y));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mre = fmax(mre, __shfl_xor_sync(0xffffffffu, mre, o));
        mim = fmax(mim, __shfl_xor_sync(0xffffffffu, mim, o));
    }
    if (lane == 0) X[blockIdx.z][(size_t)N * N * N + bin] = make_double2(mre, mim);
}

// Largest |re|, |im| over the degrees of each (class, case) of the inverse operand
// norm * coefficient / (row scale), into the table past the spectrum. One thread per (class, case).
__global__ void split_coefmax_kernel(double2* const* X, const double2* const* coeffs, int B)
{
    const int N = 2 * B;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= num_classes(B) * 8) return;
    const int cls = i >> 3, q = i & 7;
    int M, Mp;
    class_orders(cls, M, Mp);
    double mre = 0.0, mim = 0.0;
    if (q < class_case_count(M, Mp)) {
        const PairCase p = class_case(M, Mp, q, N);
        const double2* cf = coeffs[blockIdx.z];
        const double norm = (double)(B * 2 * B) / kPi;
        for (int l = M; l < B; ++l) {
            const double f = norm * (sqrt((double)l + 0.5) / 0.49);
            const double2 x = __ldg(cf + coef_index(l, p.m1, p.m2));
            mre = fmax(mre, fabs(f * x.x));
            mim = fmax(mim, fabs(f * x.y));
        }
    }
    X[blockIdx.z][(size_t)N * N * N + i] = make_double2(mre, mim);
}

}  // namespace

bool dwt_split_supported(int B) { return B >= 16 && B <= 128 && B % 16 == 0; }

size_t dwt_split_item_bytes() { return sizeof(SplitItem); }

size_t dwt_split_aux_elems(int B)
{
    const size_t n2 = (size_t)4 * B * B, c8 = (size_t)8 * num_classes(B);
    return n2 > c8 ? n2 : c8;
}

cudaError_t dwt_split_scales(int direction, int B, int T, double2* const* d_ws, const double2* const* d_coeffs,
                             cudaStream_t s)
{
    const int N = 2 * B;
    if (direction == 0) {
        dim3 grid((unsigned)(((long long)N * N + 7) / 8), 1, (unsigned)T);
        split_binmax_kernel<<<grid, 256, 0, s>>>(d_ws, N);
    } else {
        dim3 grid((unsigned)((num_classes(B) * 8 + 255) / 256), 1, (unsigned)T);
        split_coefmax_kernel<<<grid, 256, 0, s>>>(d_ws, d_coeffs, B);
    }
    return cudaGetLastError();
}

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
