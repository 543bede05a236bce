// Discrete Wigner transform for batches of transforms, and for uneven bandwidths in one launch
// (sm_100a, FP64 tensor cores).
//
// A CTA takes one work item -- an order class (M, M') of one bandwidth group for up to TT
// transforms -- from an atomic counter over a longest-first item list, so items of every
// bandwidth share one persistent launch. Its 2*TT warps share the Wigner rows: for each chunk
// of 32 degrees they generate d_{M,M'}(l, beta_k) cooperatively with the three-term recurrence
// (include/PFSOFTlib_headers/fn_dwt.hpp:167-199), each lane advancing its own beta columns,
// into one shared-memory tile; then warp (t, h) contracts that tile for transform t and the
// four symmetry cases 4h .. 4h+3 (one MMA n-tile) on the FP64 MMA:
//
//   forward  F_t[l][v] = sum_k D[l][k] S_t[k][v]   (S_t fragments held in registers per item)
//   inverse  S_t[k][v] = sum_l D[l][k] G_t[l][v]   (accumulated in registers over all chunks)
//
// with v = 2*case + (re, im), S_t[k][v] the beta column of the case's FFT bin, read at pi - beta
// when the case is reversed, and G_t the scaled, signed coefficients (see class_case in
// common.cuh for the per-coefficient symmetry rule of src/fn_dsoft.cpp:137-283). One
// recurrence therefore serves TT transforms, and no warp ever needs another warp's partial sums.

#include "common.cuh"
#include "dwt.cuh"
#include "dwt_common.cuh"

namespace pfsoft_dev {

namespace {

using namespace dwtk;

constexpr int kChunk = 32;   // degrees per shared Wigner tile

template <int TT, int NMAX, int DIR>
struct BatchSmem {
    static constexpr int DS = NMAX + (DIR == 0 ? 4 : 8);   // padded row stride (bank-conflict free)
    static constexpr size_t d_off = 0;                      // [kChunk][DS]
    static constexpr size_t rc_off = d_off + (size_t)kChunk * DS;    // [kChunk][4]
    static constexpr int GS = 24;                                   // inverse: padded row of 16 values
    static constexpr size_t g_off = rc_off + (size_t)kChunk * 4;     // inverse: [TT][kChunk][GS]
    static constexpr size_t doubles = g_off + (DIR == 1 ? (size_t)TT * kChunk * GS : 0) + 2;
};

// Generation columns of one lane: the 2*TT warps split NMAXC columns, KG per lane (lanes whose
// columns lie beyond the tile generate nothing).
template <int KG, int NMAXC>
struct GenState {
    double cb[KG], dcur[KG], dprev[KG], keep[KG];
    int sc[KG];
    bool scaled;

    __device__ __forceinline__ void seed(const DwtGroup& gr, const int* kc, double nf, bool weighted, int M, int Mp)
    {
        bool any = false;
#pragma unroll
        for (int j = 0; j < KG; ++j) {
            const int k = kc[j];
            dprev[j] = 0.0;
            sc[j] = 0;
            if (k < gr.N) {
                cb[j] = gr.cosb[k];
                dcur[j] = seed_value(weighted ? nf * gr.w[k] : nf, gr.pw_sin[(size_t)(M - Mp) * gr.N + k],
                                     gr.pw_cos[(size_t)(M + Mp) * gr.N + k], sc[j]);
            } else {
                cb[j] = 0.0;
                dcur[j] = 0.0;
            }
            keep[j] = sc[j] ? 0.0 : 1.0;
            any |= sc[j] > 0;
        }
        scaled = __any_sync(0xffffffffu, any);
    }

    __device__ __forceinline__ void step(double* row, const int* kc, const double* rc)
    {
#pragma unroll
        for (int j = 0; j < KG; ++j)
            if (kc[j] < NMAXC) row[kc[j]] = scaled ? dcur[j] * keep[j] : dcur[j];
        const double2 ca = *reinterpret_cast<const double2*>(rc);
        const double b = rc[2];
#pragma unroll
        for (int j = 0; j < KG; ++j) {
            const double t = fma(b, cb[j], ca.y);
            const double nx = fma(ca.x, dprev[j], dcur[j] * t);
            dprev[j] = dcur[j];
            dcur[j] = nx;
        }
        if (scaled) {
            bool still = false;
#pragma unroll
            for (int j = 0; j < KG; ++j) {
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

// Recurrence coefficients for degrees l .. l+31 into rc (warp 0 only; one lane per degree), from
// the bandwidth's table; steps past the last degree get zeros (their rows are never used).
__device__ __forceinline__ void rc_chunk(const DwtGroup& gr, double* rc, int l, int M, int Mp, int lane)
{
    const int d = l + lane;
    double2 cf = make_double2(0.0, 0.0);
    double f1 = 0.0;
    if (d < gr.B) {
        const long long i = rc_offset(gr.B, M, Mp) + (d - M);
        cf = __ldg(gr.rc_cf + i);
        f1 = __ldg(gr.rc_f1 + i);
    }
    *reinterpret_cast<double2*>(rc + 4 * lane) = cf;
    rc[4 * lane + 2] = f1;
}

template <int TT, int NMAX, int DIR>
__global__ void __launch_bounds__(64 * TT) dwt_batch_kernel(const DwtGroup* __restrict__ groups,
                                                           const DwtItem* __restrict__ items, int n_items,
                                                           int* __restrict__ counter)
{
    using L = BatchSmem<TT, NMAX, DIR>;
    constexpr int DS = L::DS;
    constexpr int NW = 2 * TT;                       // warps
    constexpr int KG = (NMAX + 32 * NW - 1) / (32 * NW);   // generation columns per lane
    constexpr int NSUB4 = NMAX / 4;                   // forward: k-subtiles of 4 columns
    constexpr int NSUB8 = NMAX / 8;                   // inverse: m-subtiles of 8 columns
    constexpr int PER = (TT * 8 * kChunk + 64 * TT - 1) / (64 * TT);   // inverse: coefficients per thread per chunk
    extern __shared__ double smem[];
    double* s_d = smem + L::d_off;
    double* s_rc = smem + L::rc_off;
    double* s_g = smem + L::g_off;
    int* s_item = reinterpret_cast<int*>(smem + L::doubles - 2);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, t4 = lane & 3;
    const int tslot = warp >> 1, h = warp & 1;
    int kc[KG];
#pragma unroll
    for (int j = 0; j < KG; ++j) kc[j] = warp * (32 * KG) + lane + 32 * j;

    for (;;) {
        if (tid == 0) *s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int idx = *s_item;
        __syncthreads();   // every thread has the index before thread 0 may overwrite it
        if (idx >= n_items) break;
        const DwtItem it = items[idx];
        const DwtGroup gr = groups[it.group];
        const int B = gr.B, N = gr.N;
        int M, Mp;
        class_orders(it.cls, M, Mp);
        const int nc = class_case_count(M, Mp);
        const bool active = tslot < it.nt;
        const int tr = it.t0 + tslot;

        GenState<KG, NMAX> gs;
        gs.seed(gr, kc, gr.normf[it.cls], DIR == 0, M, Mp);

        if (DIR == 0) {
            // ---------------------------------------------------------------- forward
            const double norm = kPi / (double)(B * 2 * B);   // src/fn_dsoft.cpp:119
            double sb[NSUB4];
            PairCase po;
            {
                const int c = 4 * h + (g >> 1), comp = g & 1;
                const bool ok = active && c < nc;
                const PairCase p = class_case(M, Mp, ok ? c : 0, N);
                const double* col = ok ? reinterpret_cast<const double*>(gr.X[tr] + ((size_t)p.row * N + p.col) * N) + comp : nullptr;
#pragma unroll
                for (int q = 0; q < NSUB4; ++q) {
                    const int k = 4 * q + t4;
                    sb[q] = (ok && k < N) ? __ldg(col + 2 * (p.rev ? N - 1 - k : k)) : 0.0;
                }
                const int co = 4 * h + t4;
                po = class_case(M, Mp, co < nc ? co : 0, N);
            }
            for (int c0 = M; c0 < B; c0 += kChunk) {
                if (warp == 0) rc_chunk(gr, s_rc, c0, M, Mp, lane);
                __syncthreads();
#pragma unroll 4
                for (int s = 0; s < kChunk; ++s) gs.step(s_d + s * DS, kc, s_rc + 4 * s);
                __syncthreads();
                if (active) {
                    const int nb = min(kChunk, B - c0);
                    for (int b0 = 0; b0 < nb; b0 += 8) {
                        double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
                        const double* dr = s_d + (b0 + g) * DS + t4;
#pragma unroll
                        for (int q = 0; q < NSUB4; ++q)
                            if (4 * q < N) dmma(acc[q & 1][0], acc[q & 1][1], dr[4 * q], sb[q]);
                        const int l = c0 + b0 + g;
                        const int co = 4 * h + t4;
                        if (l < B && co < nc) {
                            const double f = norm * case_sign(po, l, M);
                            *reinterpret_cast<double2*>(gr.coeffs[tr] + coef_index(l, po.m1, po.m2)) =
                                make_double2(f * (acc[0][0] + acc[1][0]), f * (acc[0][1] + acc[1][1]));
                        }
                    }
                }
                __syncthreads();   // the tile is rewritten by the next chunk
            }
        } else {
            // ---------------------------------------------------------------- inverse
            const double norm = (double)(B * 2 * B) / kPi;   // src/fn_idsoft.cpp:109
            double acc[NSUB8][2];
#pragma unroll
            for (int p = 0; p < NSUB8; ++p) acc[p][0] = acc[p][1] = 0.0;
            double2 pf[PER];
            // scaled, signed coefficients of degrees l .. l+31 for the item's transforms
            auto fetch = [&](int l) {
#pragma unroll
                for (int i = 0; i < PER; ++i) {
                    const int e = tid + i * 64 * TT;          // e = (t * kChunk + j) * 8 + c
                    const int t = e / (8 * kChunk), j = (e >> 3) % kChunk, c = e & 7, ld = l + j;
                    double2 v = make_double2(0.0, 0.0);
                    if (t < it.nt && c < nc && ld < B) {
                        const PairCase p = class_case(M, Mp, c, N);
                        const double f = norm * case_sign(p, ld, M);
                        const double2 x = __ldg(gr.coeffs[it.t0 + t] + coef_index(ld, p.m1, p.m2));
                        v = make_double2(f * x.x, f * x.y);
                    }
                    pf[i] = v;
                }
            };
            fetch(M);
            for (int c0 = M; c0 < B; c0 += kChunk) {
#pragma unroll
                for (int i = 0; i < PER; ++i) {
                    const int e = tid + i * 64 * TT;
                    const int t = e / (8 * kChunk), j = (e >> 3) % kChunk, c = e & 7;
                    if (t < TT) *reinterpret_cast<double2*>(s_g + ((size_t)t * kChunk + j) * L::GS + 2 * c) = pf[i];
                }
                if (warp == 0) rc_chunk(gr, s_rc, c0, M, Mp, lane);
                __syncthreads();
                if (c0 + kChunk < B) fetch(c0 + kChunk);   // in flight during this chunk
#pragma unroll 4
                for (int s = 0; s < kChunk; ++s) gs.step(s_d + s * DS, kc, s_rc + 4 * s);
                __syncthreads();
                if (active) {
                    const int nb = min(kChunk, B - c0);
                    const double* gt = s_g + (size_t)tslot * kChunk * L::GS + 8 * h + g;
                    for (int b0 = 0; b0 < nb; b0 += 8) {
                        const double bv0 = gt[(b0 + t4) * L::GS], bv1 = gt[(b0 + 4 + t4) * L::GS];
                        const double* d0 = s_d + (b0 + t4) * DS + g;
                        const double* d1 = s_d + (b0 + 4 + t4) * DS + g;
                        // narrower bandwidths in a wider launch skip empty tiles; the two k-halves
                        // of an accumulator are issued a full round apart, the second half first
                        // for subtiles with p % 8 >= 4: the order dwt_inverse_kernel sums them in,
                        // so that a transform gives the same bits batched or alone
#pragma unroll
                        for (int p = 0; p < NSUB8; ++p)
                            if (8 * p < N) dmma(acc[p][0], acc[p][1], (p & 4) ? d1[8 * p] : d0[8 * p], (p & 4) ? bv1 : bv0);
#pragma unroll
                        for (int p = 0; p < NSUB8; ++p)
                            if (8 * p < N) dmma(acc[p][0], acc[p][1], (p & 4) ? d0[8 * p] : d1[8 * p], (p & 4) ? bv0 : bv1);
                    }
                }
                __syncthreads();   // tile and coefficient chunk are rewritten by the next chunk
            }
            const int c = 4 * h + t4;
            if (active && c < nc) {
                const PairCase pcase = class_case(M, Mp, c, N);
                double2* col = gr.X[tr] + ((size_t)pcase.row * N + pcase.col) * N;
#pragma unroll
                for (int p = 0; p < NSUB8; ++p) {
                    const int k = 8 * p + g;
                    if (k < N) __stcs(col + (pcase.rev ? N - 1 - k : k), make_double2(acc[p][0], acc[p][1]));   // evict-first, as dwt_inverse_kernel
                }
            }
        }
    }
}

template <int TT, int NMAX, int DIR>
cudaError_t launch_batch(const DwtGroup* g, const DwtItem* it, int n, int* counter, cudaStream_t s)
{
    const size_t smem = BatchSmem<TT, NMAX, DIR>::doubles * sizeof(double);
    auto k = dwt_batch_kernel<TT, NMAX, DIR>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, 64 * TT, smem) != cudaSuccess || per < 1) per = 1;
    int blocks = sms * per;
    if (blocks > n) blocks = n > 0 ? n : 1;
    k<<<blocks, 64 * TT, smem, s>>>(g, it, n, counter);
    return cudaGetLastError();
}

template <int DIR>
cudaError_t dispatch_nmax(int tpc, int nmax, const DwtGroup* g, const DwtItem* it, int n, int* counter,
                          cudaStream_t s)
{
    if (nmax <= 64) {
        if (tpc == 1) return launch_batch<1, 64, DIR>(g, it, n, counter, s);
        if (tpc == 2) return launch_batch<2, 64, DIR>(g, it, n, counter, s);
        return launch_batch<4, 64, DIR>(g, it, n, counter, s);
    }
    if (nmax <= 128) {
        if (tpc == 1) return launch_batch<1, 128, DIR>(g, it, n, counter, s);
        if (tpc == 2) return launch_batch<2, 128, DIR>(g, it, n, counter, s);
        return launch_batch<4, 128, DIR>(g, it, n, counter, s);
    }
    if (nmax <= 256) {
        if (tpc == 1) return launch_batch<1, 256, DIR>(g, it, n, counter, s);
        if (tpc == 2) return launch_batch<2, 256, DIR>(g, it, n, counter, s);
        return launch_batch<4, 256, DIR>(g, it, n, counter, s);
    }
    return cudaErrorInvalidValue;
}

}  // namespace

int dwt_batch_transforms_per_cta(int nmax) { return nmax <= 128 ? 4 : 2; }

size_t dwt_batch_smem_bytes(int direction, int tpc, int nmax)
{
    const int n = nmax <= 64 ? 64 : (nmax <= 128 ? 128 : 256);
    const int ds = n + (direction == 0 ? 4 : 8);
    return ((size_t)kChunk * ds + (size_t)kChunk * 4 + (direction == 1 ? (size_t)tpc * kChunk * 24 : 0) + 2) * sizeof(double);
}

cudaError_t dwt_batch_launch(int direction, const DwtGroup* d_groups, const DwtItem* d_items, int n_items,
                             int* d_counter, int tpc, int nmax, cudaStream_t s)
{
    if (n_items <= 0) return cudaSuccess;
    if (tpc != 1 && tpc != 2 && tpc != 4) return cudaErrorInvalidValue;
    return direction == 0 ? dispatch_nmax<0>(tpc, nmax, d_groups, d_items, n_items, d_counter, s)
                          : dispatch_nmax<1>(tpc, nmax, d_groups, d_items, n_items, d_counter, s);
}

}  // namespace pfsoft_dev
