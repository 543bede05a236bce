// Split-precision discrete Wigner transform on the 5th-generation tensor cores (sm_100a), as
// exact products of 8-bit digit planes.
//
// For one order class (M, M') and up to two transforms of one bandwidth the DWT is a real matrix
// product (see dwt_batch.cu for the case / column conventions):
//   forward  F[l][c] = sum_k D[l][k] S[k][c]     l = M..B-1, k = beta samples, c = (transform, case, re/im)
//   inverse  S[k][c] = sum_l D[l][k] G[l][c]
// D (the Wigner-d rows, generated on chip by the FP64 three-term recurrence of
// include/PFSOFTlib_headers/fn_dwt.hpp:167-199, as in the FP64 kernels) and S / G (FP64 data)
// are turned into 48-bit fixed point with a per-row scale for D and a per-column power-of-two
// scale for the other operand: x = round(v * scale * 2^47) = sum_i d_i 256^(5-i), d_i in
// [-128, 127] (one FMA against a magic constant leaves x + sum 128*256^i in the low 48 bits of
// a double; each byte XOR 0x80 is a signed digit). Digit planes are multiplied with
// tcgen05.mma kind::i8 (signed 8-bit x signed 8-bit -> exact S32 in tensor memory): plane s of
// the generated operand times the concatenated planes 0..5-s of the data operand lands in
// accumulator planes s..5 (significance e = s + t; the 15 products with e > 5 are dropped). A
// plane product summed over any K <= 2^16 is exact, so every bandwidth up to 256 (K = 512) is
// exact in the integer sums; the epilogue combines the six planes in FP64 (Horner in 2^-8,
// smallest first) and undoes the scales. FP64 stays for the seeds, the recurrence, the weights
// and that final sum.
//
// Work items, dealt to the persistent CTAs in snake order over one index space:
//   forward  (class, transforms t0..t0+nt-1, row tile): 128 degrees (M dimension) x all beta
//            (K, chunks of 32); a second row tile (degrees M+128 ..) runs the recurrence through
//            the first 128 degrees without storing them.
//   inverse  (class, transforms, beta tile): 128 beta (M dimension) x all degrees (K, chunks of 32).
// The items are not listed: a launch gets one segment per bandwidth group (host:
// dwt_split_segments, largest bandwidth first), and item i of a segment is class i / (pairs *
// tiles) -- classes run longest first (M ascending) -- then transform pair, then tile.
// One CTA of 12 warps per SM, roles fixed per warp:
//   warp 0      issues the MMAs (one lane) into one of two accumulator sets in tensor memory;
//   warps 1-3   loaders: the data operand of a chunk (spectrum bins or coefficients) to digit planes;
//   warps 4-7   epilogue: read an accumulator set back (warp w reads lanes 32(w%4) ..), combine, store;
//   warps 8-11  generators: the Wigner rows of a chunk to digit planes (forward: one warp per
//               chunk of 32 beta columns, all rows; inverse: the four warps on the tile's 128 beta
//               columns, 32 degrees per chunk).
// Chunks move through a ring of shared-memory stages (full / empty mbarriers; empty is signalled by
// tcgen05.commit), accumulator sets through accfull / accempty, so generation, loading, MMAs and the
// epilogue of different chunks and items overlap. Every wait is bounded (%globaltimer); a wait that
// runs out sets a CTA-wide abort flag, every role leaves, the MMA lane waits (bounded) for its
// committed MMAs before the tensor memory is freed, and *status is set to 1.
//
// Operand layouts in shared memory (no swizzle; see tc_sm100.cuh), per stage and plane:
//   A forward (MN-major, rows = degrees):  (r/16)*512 + (k/8)*128 + (k%8)*16 + (r%16)
//   A inverse (K-major, rows = beta):      (m/8)*256 + (j/16)*128 + (m%8)*16 + (j%16)
//   B both    (K-major, rows = columns):   (n/8)*256 + (k/16)*128 + (n%8)*16 + (k%16),
//             plane t of the data operand at rows 16*nt*t .. (planes concatenated along N)
// so that a generator lane writes whole 16-byte units of 16 consecutive degrees of its beta column,
// and a loader lane 8-byte halves of 8 consecutive K of one column.

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

constexpr int kNT = 2;                 // transforms per work item (at most)
constexpr int kPlanes = 6;             // digits per operand
constexpr int kKC = 32;                // K per chunk: one kind::i8 MMA
constexpr int kStages = 6;             // operand ring
constexpr int kAccSets = 2;
constexpr int kAccStride = 256;        // tensor-memory columns between the two accumulator sets
constexpr uint32_t kTmemCols = 512;
constexpr int kThreads = 384;
constexpr int kLoadWarp0 = 1, kLoadWarps = 3;
constexpr int kEpiWarp0 = 4;
constexpr int kGenWarp0 = 8, kGenWarps = 4;
constexpr uint64_t kWaitNs = 2000000000ull;   // 2 s

constexpr int kAPlane = 4096;                       // 128 rows x 32 bytes of K
constexpr int kABytes = kPlanes * kAPlane;          // 24 KB
constexpr int kBRows = 16 * kNT * kPlanes;          // 192
constexpr int kBBytes = kBRows / 8 * 256;           // 6 KB
constexpr int kStageBytes = kABytes + kBBytes;
constexpr int kOffCoef = kStages * kStageBytes;     // generators: 32 steps x {c1, f1 f2, f1, row scale} per warp
constexpr int kOffBar = kOffCoef + kGenWarps * 32 * 4 * 8;
// mbarriers: full[kStages], empty[kStages], accfull[2], accempty[2], drain, never (test knob)
constexpr int kBarFull = 0, kBarEmpty = kStages, kBarAccFull = 2 * kStages, kBarAccEmpty = 2 * kStages + kAccSets,
              kBarDrain = 2 * kStages + 2 * kAccSets, kBarNever = kBarDrain + 1, kNumBars = kBarNever + 1;
constexpr int kOffMisc = kOffBar + kNumBars * 8;    // tensor-memory address, abort flag
constexpr int kSmemBytes = kOffMisc + 16;
static_assert(kStageBytes % 1024 == 0, "stages stay 1 KB aligned");
static_assert(kSmemBytes <= 227 * 1024, "shared memory");
static_assert(16 * kNT * kPlanes <= kAccStride, "an accumulator set fits its column range");

constexpr double kTwo47 = 140737488355328.0;        // 2^47
// 2^52 + sum_{i<6} 128 * 256^i: adding it to x * 2^47 (|x| < 0.5) leaves round(x * 2^47) + C in
// the low 48 bits of the double, C making every byte a digit plus 128.
constexpr double kMagic = 4503599627370496.0 + 141289400074368.0;

// One bandwidth group of a launch: items first .. first+count-1, `pairs` transform pairs (T
// transforms) and `tiles` tiles per class.
struct SplitSeg {
    int group, first, count, pairs, tiles, T, pad0, pad1;
};

// Digit words of four magic-biased values: w[p] holds byte (5 - p) of each value (value i in
// byte i), XOR 0x80, i.e. plane p of the signed digits, most significant plane first.
__device__ __forceinline__ void pack4(double z0, double z1, double z2, double z3, uint32_t (&w)[kPlanes])
{
    const uint32_t L0 = (uint32_t)__double2loint(z0), H0 = (uint32_t)__double2hiint(z0);
    const uint32_t L1 = (uint32_t)__double2loint(z1), H1 = (uint32_t)__double2hiint(z1);
    const uint32_t L2 = (uint32_t)__double2loint(z2), H2 = (uint32_t)__double2hiint(z2);
    const uint32_t L3 = (uint32_t)__double2loint(z3), H3 = (uint32_t)__double2hiint(z3);
    const uint32_t a01 = tc::prmt(L0, L1, 0x5140), b01 = tc::prmt(L0, L1, 0x7362);
    const uint32_t a23 = tc::prmt(L2, L3, 0x5140), b23 = tc::prmt(L2, L3, 0x7362);
    const uint32_t h01 = tc::prmt(H0, H1, 0x5140), h23 = tc::prmt(H2, H3, 0x5140);
    w[5] = tc::prmt(a01, a23, 0x5410) ^ 0x80808080u;   // byte 0
    w[4] = tc::prmt(a01, a23, 0x7632) ^ 0x80808080u;   // byte 1
    w[3] = tc::prmt(b01, b23, 0x5410) ^ 0x80808080u;   // byte 2
    w[2] = tc::prmt(b01, b23, 0x7632) ^ 0x80808080u;   // byte 3
    w[1] = tc::prmt(h01, h23, 0x5410) ^ 0x80808080u;   // byte 4
    w[0] = tc::prmt(h01, h23, 0x7632) ^ 0x80808080u;   // byte 5
}

// 16 magic-biased values -> one 16-byte unit per plane at base + p * plane_stride
__device__ __forceinline__ void store_unit16(unsigned char* base, int plane_stride, const double (&z)[16])
{
    uint32_t w0[kPlanes], w1[kPlanes], w2[kPlanes], w3[kPlanes];
    pack4(z[0], z[1], z[2], z[3], w0);
    pack4(z[4], z[5], z[6], z[7], w1);
    pack4(z[8], z[9], z[10], z[11], w2);
    pack4(z[12], z[13], z[14], z[15], w3);
#pragma unroll
    for (int p = 0; p < kPlanes; ++p)
        *reinterpret_cast<uint4*>(base + p * plane_stride) = make_uint4(w0[p], w1[p], w2[p], w3[p]);
}

// 8 magic-biased values -> one 8-byte half unit per plane
__device__ __forceinline__ void store_unit8(unsigned char* base, int plane_stride, const double (&z)[8])
{
    uint32_t w0[kPlanes], w1[kPlanes];
    pack4(z[0], z[1], z[2], z[3], w0);
    pack4(z[4], z[5], z[6], z[7], w1);
#pragma unroll
    for (int p = 0; p < kPlanes; ++p) *reinterpret_cast<uint2*>(base + p * plane_stride) = make_uint2(w0[p], w1[p]);
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

// Item geometry shared by every role.
struct ItemGeo {
    const DwtGroup* gr;
    int B, N, M, Mp, R, nc, t0, nt, tile, cls, nchunks;
};

// Geometry of item i: its segment by a scan over the launch's few segments, then class,
// transform pair and tile. A forward row tile past the class's last degree has no chunks (every
// role skips it alike).
template <int DIR>
__device__ __forceinline__ ItemGeo item_geo(const DwtGroup* __restrict__ groups, const SplitSeg* __restrict__ segs,
                                            int nseg, int i)
{
    int sidx = 0;
    while (sidx + 1 < nseg && i >= segs[sidx + 1].first) ++sidx;
    const SplitSeg sg = segs[sidx];
    const int j = i - sg.first;
    const int per_cls = sg.pairs * sg.tiles;
    const int cls = j / per_cls, rem = j - cls * per_cls;
    const int pair = rem / sg.tiles;
    ItemGeo g;
    g.gr = groups + sg.group;
    g.B = g.gr->B;
    g.N = g.gr->N;
    class_orders(cls, g.M, g.Mp);
    g.R = g.B - g.M;
    g.nc = class_case_count(g.M, g.Mp);
    g.t0 = kNT * pair;
    g.nt = min(kNT, sg.T - g.t0);
    g.tile = rem - pair * sg.tiles;
    g.cls = cls;
    if (DIR == 0)
        g.nchunks = 128 * g.tile < g.R ? (g.N + kKC - 1) / kKC : 0;
    else
        g.nchunks = (g.R + kKC - 1) / kKC;
    return g;
}

// The CTA's r-th item in snake order over the longest-first list (-1 past the end).
__device__ __forceinline__ int cta_item(int r, int n_items)
{
    const int G = gridDim.x, b = blockIdx.x;
    const int i = r * G + ((r & 1) ? (G - 1 - b) : b);
    return i < n_items ? i : -1;
}

// Row table of a transform's operand-scale area: {scale * 2^47, 1 / scale} per degree l.
__device__ __forceinline__ const double2* row_table(const DwtGroup* gr, int t)
{
    const int N = gr->N, B = gr->B;
    const size_t a0 = (size_t)N * N > (size_t)8 * num_classes(B) ? (size_t)N * N : (size_t)8 * num_classes(B);
    return gr->X[t] + (size_t)N * N * N + a0;
}

// One recurrence step of a beta column (fn_dwt.hpp:167-199): d(l+1) = d(l)(f1 f2 + f1 cos b) + c1 d(l-1);
// a column whose seed was scaled by 2^600 rescales once it grows past 2^300 (and stores 0 meanwhile).
__device__ __forceinline__ void rec_step(double& dcur, double& dprev, int& sc, double cb, double2 cf, double f1)
{
    const double t = fma(f1, cb, cf.y);
    const double u = cf.x * dprev;
    const double nx = fma(dcur, t, u);
    dprev = dcur;
    dcur = nx;
    if (sc && fabs(dcur) >= 0x1p300) {
        dcur *= 0x1p-600;
        dprev *= 0x1p-600;
        --sc;
    }
}

template <int DIR>
__global__ void __launch_bounds__(kThreads, 1)
    dwt_split_kernel(const DwtGroup* __restrict__ groups, const SplitSeg* __restrict__ segs, int nseg, int n_items,
                     int* __restrict__ status, unsigned long long fail_ns)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kOffBar);
    uint32_t* s_taddr = reinterpret_cast<uint32_t*>(smem + kOffMisc);
    volatile int* s_abort = reinterpret_cast<volatile int*>(smem + kOffMisc + 4);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    if (warp == 0) {
        tc::tmem_alloc(s_taddr, kTmemCols);
        tc::tmem_relinquish();
    }
    if (tid == 32) {
        for (int s = 0; s < kStages; ++s) {
            tc::mbar_init(&bars[kBarFull + s], DIR == 0 ? 2 : 1 + kGenWarps);   // generator warp(s) + loader warp
            tc::mbar_init(&bars[kBarEmpty + s], 1);                           // tcgen05.commit
        }
        for (int a = 0; a < kAccSets; ++a) {
            tc::mbar_init(&bars[kBarAccFull + a], 1);
            tc::mbar_init(&bars[kBarAccEmpty + a], 4);   // the four epilogue warps
        }
        tc::mbar_init(&bars[kBarDrain], 1);
        tc::mbar_init(&bars[kBarNever], 1);
        tc::mbar_fence_init();
        *s_abort = 0;
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *s_taddr;
    const uint32_t smem_base = tc::smem_u32(smem);

    if (warp == 0) {
        // ------------------------------------------------------------------ MMA issue
        bool ok = true;
        if (fail_ns) ok = tc::mbar_wait_bounded(&bars[kBarNever], 0, fail_ns, s_abort);   // test knob: nothing arrives
        int g = 0, n = 0;   // chunks and (non-empty) items issued
        for (int r = 0; ok; ++r) {
            const int idx = cta_item(r, n_items);
            if (idx < 0) break;
            const ItemGeo it = item_geo<DIR>(groups, segs, nseg, idx);
            if (it.nchunks == 0) continue;
            const int a = n & 1, ua = n >> 1;
            ++n;
            if (!tc::mbar_wait_bounded(&bars[kBarAccEmpty + a], (uint32_t)((ua & 1) ^ 1), kWaitNs, s_abort)) {
                ok = false;
                break;
            }
            tc::fence_after_sync();
            const uint32_t dbase = tmem + (uint32_t)(a * kAccStride);
            const int cols = 16 * it.nt;
            for (int c = 0; c < it.nchunks; ++c, ++g) {
                const int s = g % kStages, u = g / kStages;
                if (!tc::mbar_wait_bounded(&bars[kBarFull + s], (uint32_t)(u & 1), kWaitNs, s_abort)) {
                    ok = false;
                    break;
                }
                tc::fence_after_sync();
                if (lane == 0) {
                    const uint32_t a0 = smem_base + s * kStageBytes, b0 = a0 + kABytes;
                    const uint64_t bd = tc::sdesc(b0, 128, 256);
#pragma unroll
                    for (int p = 0; p < kPlanes; ++p) {
                        const uint64_t ad = DIR == 0 ? tc::sdesc(a0 + p * kAPlane, 128, 512) : tc::sdesc(a0 + p * kAPlane, 128, 256);
                        tc::mma_s8(dbase + (uint32_t)(cols * p), ad, bd, tc::idesc_s8(128, cols * (kPlanes - p), DIR == 0, false),
                                   !(c == 0 && p == 0));
                    }
                    tc::mma_commit(&bars[kBarEmpty + s]);
                }
                __syncwarp();
            }
            if (!ok) break;
            if (lane == 0) tc::mma_commit(&bars[kBarAccFull + a]);
            __syncwarp();
        }
        // every MMA issued by this lane has completed before the tensor memory can be freed
        if (lane == 0) {
            tc::mma_commit(&bars[kBarDrain]);
            const uint64_t t0 = tc::globaltimer_ns();
            while (!tc::mbar_try_wait(&bars[kBarDrain], 0))
                if (tc::globaltimer_ns() - t0 > kWaitNs) break;
        }
        __syncwarp();
    } else if (warp >= kLoadWarp0 && warp < kLoadWarp0 + kLoadWarps) {
        // ------------------------------------------------------------------ loaders (data operand)
        const int L = warp - kLoadWarp0;
        int g = 0;
        for (int r = 0;; ++r) {
            const int idx = cta_item(r, n_items);
            if (idx < 0 || *s_abort) break;
            const ItemGeo it = item_geo<DIR>(groups, segs, nseg, idx);
            const int N = it.N, B = it.B, nt = it.nt;
            if (DIR == 0 && lane < 16 && (g % kLoadWarps) == L) {
                // the next item's bin columns into L2 while this one runs
                const int nx = cta_item(r + 1, n_items);
                if (nx >= 0) {
                    const ItemGeo in = item_geo<DIR>(groups, segs, nseg, nx);
                    const int t = lane >> 3, q = lane & 7;
                    if (t < in.nt && q < in.nc) {
                        const PairCase p = class_case(in.M, in.Mp, q, in.N);
                        prefetch_l2(in.gr->X[in.t0 + t] + ((size_t)p.row * in.N + p.col) * in.N, (unsigned)in.N * 16u);
                    }
                }
            }
            // per-lane column scales of the columns this lane converts: task e = lane + 32 i
            // is (octet o = e % 4, column pair cp = e / 4 = 2 (case) + transform), i < 2 * nt
            for (int c = 0; c < it.nchunks; ++c, ++g) {
                if ((g % kLoadWarps) != L) continue;
                const int s = g % kStages, u = g / kStages;
                unsigned char* Bm = smem + s * kStageBytes + kABytes;
                constexpr int kTasks = 8 * kNT * 4;   // column pairs x octets
                double raw[kTasks / 32][8][2];
                double2 mxv[kTasks / 32];   // the column's largest |re|, |im| (operand-scale table)
                int tq[kTasks / 32], to[kTasks / 32];
                // loads first (they fly while the stage is still being read by the MMAs): the data,
                // the columns' scale-table entries, and (inverse) the row scale of degree
                // M + 32c + lane, handed to the lanes that need it by shuffles below
                double irs_lane = 0.0;
                if (DIR == 1 && c * kKC + lane < it.R) irs_lane = __ldg(&row_table(it.gr, it.t0)[it.M + c * kKC + lane].y);
#pragma unroll
                for (int i = 0; i < kTasks / 32; ++i) {
                    const int e = lane + 32 * i;
                    const int o = e & 3, cpair = e >> 2;   // cpair = 8 t + q
                    const int t = cpair >> 3, q = cpair & 7;
                    tq[i] = cpair;
                    to[i] = o;
                    const bool live = t < nt && q < it.nc;
                    {
                        const double2* aux = it.gr->X[it.t0 + (live ? t : 0)] + (size_t)N * N * N;
                        const PairCase p = class_case(it.M, it.Mp, live ? q : 0, N);
                        mxv[i] = live ? (DIR == 0 ? __ldg(aux + (size_t)p.row * N + p.col) : __ldg(aux + (size_t)it.cls * 8 + q))
                                      : make_double2(0.0, 0.0);
                    }
                    if (DIR == 0) {
                        const PairCase p = class_case(it.M, it.Mp, live ? q : 0, N);
                        const double2* col = it.gr->X[it.t0 + (live ? t : 0)] + ((size_t)p.row * N + p.col) * N;
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            const int k = c * kKC + 8 * o + j;
                            double2 v = make_double2(0.0, 0.0);
                            if (live && k < N) v = __ldg(col + (p.rev ? N - 1 - k : k));
                            raw[i][j][0] = v.x;
                            raw[i][j][1] = v.y;
                        }
                    } else {
                        const PairCase p = class_case(it.M, it.Mp, live ? q : 0, N);
                        const double2* cf = it.gr->coeffs[it.t0 + (live ? t : 0)];
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            const int l = it.M + c * kKC + 8 * o + j;
                            double2 v = make_double2(0.0, 0.0);
                            if (live && l < B) v = __ldg(cf + coef_index(l, p.m1, p.m2));
                            raw[i][j][0] = v.x;
                            raw[i][j][1] = v.y;
                        }
                    }
                }
                if (!tc::mbar_wait_bounded(&bars[kBarEmpty + s], (uint32_t)((u & 1) ^ 1), kWaitNs, s_abort)) break;
#pragma unroll
                for (int i = 0; i < kTasks / 32; ++i) {
                    const int cpair = tq[i], o = to[i];
                    const int t = cpair >> 3, q = cpair & 7;
                    double irs8[8];
                    if (DIR == 1) {
#pragma unroll
                        for (int j = 0; j < 8; ++j) irs8[j] = __shfl_sync(0xffffffffu, irs_lane, 8 * o + j);
                    }
                    if (t >= nt || q >= it.nc) continue;   // columns never stored: left as they are
                    const double2 mx = mxv[i];
                    const double sgn_norm = DIR == 0 ? 1.0 : (double)(B * 2 * B) / kPi;   // src/fn_idsoft.cpp:109
                    PairCase p = class_case(it.M, it.Mp, q, N);
                    double cs_re, cs_im, ics_unused;
                    column_scale(mx.x, cs_re, ics_unused);
                    column_scale(mx.y, cs_im, ics_unused);
                    double zr[8], zi[8];
                    if (DIR == 0) {
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            zr[j] = fma(raw[i][j][0], cs_re, kMagic);
                            zi[j] = fma(raw[i][j][1], cs_im, kMagic);
                        }
                    } else {
                        // G = norm * sign(l) * f / (row scale), zero past the last degree
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            const int l = it.M + c * kKC + 8 * o + j;
                            double f = 0.0;
                            if (l < B) f = sgn_norm * case_sign(p, l, it.M) * irs8[j];
                            zr[j] = fma(f * raw[i][j][0], cs_re, kMagic);
                            zi[j] = fma(f * raw[i][j][1], cs_im, kMagic);
                        }
                    }
                    const int n = 16 * t + 2 * q;   // re column; im is n + 1
                    const int plane_rows = 16 * nt;
                    // rows n, n+1 of plane 0; plane p at rows + 16 nt p: (n/8)*256 + (k/16)*128 + (n%8)*16 + k%16
                    unsigned char* unit = Bm + (n >> 3) * 256 + (o >> 1) * 128 + (n & 7) * 16 + (o & 1) * 8;
                    const int pstride = plane_rows / 8 * 256;
                    store_unit8(unit, pstride, zr);
                    store_unit8(unit + 16, pstride, zi);
                }
                tc::fence_proxy_async();
                __syncwarp();
                if (lane == 0) tc::mbar_arrive(&bars[kBarFull + s]);
            }
            if (*s_abort) break;
        }
    } else if (warp >= kEpiWarp0 && warp < kEpiWarp0 + 4) {
        // ------------------------------------------------------------------ epilogue
        const int q4 = warp & 3;   // tensor-memory lane quarter
        int n = 0;
        for (int r = 0;; ++r) {
            const int idx = cta_item(r, n_items);
            if (idx < 0) break;
            const ItemGeo it = item_geo<DIR>(groups, segs, nseg, idx);
            if (it.nchunks == 0) continue;
            const int a = n & 1, ua = n >> 1;
            ++n;
            if (!tc::mbar_wait_bounded(&bars[kBarAccFull + a], (uint32_t)(ua & 1), kWaitNs, s_abort)) break;
            tc::fence_after_sync();
            const int N = it.N, B = it.B;
            const int row = 32 * q4 + lane;
            const uint32_t taddr = tmem + ((uint32_t)(32 * q4) << 16) + (uint32_t)(a * kAccStride);
            const int cols = 16 * it.nt;
            // forward: degree l of this lane; inverse: beta k
            const int l = it.M + 128 * it.tile + row;
            const int k = 128 * it.tile + row;
            const bool live = DIR == 0 ? (l < B) : (k < N);
            double rowf = 0.0;
            if (DIR == 0 && live) rowf = (kPi / (double)(B * 2 * B)) * __ldg(&row_table(it.gr, it.t0)[l].y);   // src/fn_dsoft.cpp:119
            for (int t = 0; t < it.nt; ++t) {
                // the eight columns' scale-table entries, in flight while the accumulators are read
                const double2* aux = it.gr->X[it.t0 + t] + (size_t)N * N * N;
                double2 mxq[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    mxq[q] = make_double2(0.0, 0.0);
                    if (q < it.nc) {
                        const PairCase p = class_case(it.M, it.Mp, q, N);
                        mxq[q] = DIR == 0 ? __ldg(aux + (size_t)p.row * N + p.col) : __ldg(aux + (size_t)it.cls * 8 + q);
                    }
                }
                int32_t acc[kPlanes][16];
#pragma unroll
                for (int e = 0; e < kPlanes; ++e) tc::tmem_ld16(taddr + (uint32_t)(cols * e + 16 * t), acc[e]);
                tc::tmem_wait_ld();
                double v[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    double h = (double)acc[5][j];
                    h = fma(h, 0x1p-8, (double)acc[4][j]);
                    h = fma(h, 0x1p-8, (double)acc[3][j]);
                    h = fma(h, 0x1p-8, (double)acc[2][j]);
                    h = fma(h, 0x1p-8, (double)acc[1][j]);
                    v[j] = fma(h, 0x1p-8, (double)acc[0][j]) * 0x1p-14;
                }
                if (!live) continue;
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    if (q >= it.nc) break;
                    const PairCase p = class_case(it.M, it.Mp, q, N);
                    const double2 mx = mxq[q];
                    double unused, ics_re, ics_im;
                    column_scale(mx.x, unused, ics_re);
                    column_scale(mx.y, unused, ics_im);
                    if (DIR == 0) {
                        const double f = rowf * case_sign(p, l, it.M);
                        it.gr->coeffs[it.t0 + t][coef_index(l, p.m1, p.m2)] =
                            make_double2(f * v[2 * q] * ics_re, f * v[2 * q + 1] * ics_im);
                    } else {
                        it.gr->X[it.t0 + t][((size_t)p.row * N + p.col) * N + (p.rev ? N - 1 - k : k)] =
                            make_double2(v[2 * q] * ics_re, v[2 * q + 1] * ics_im);
                    }
                }
            }
            tc::fence_before_sync();
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(&bars[kBarAccEmpty + a]);
        }
    } else if (warp >= kGenWarp0) {
        // ------------------------------------------------------------------ generators (Wigner rows)
        // The recurrence coefficients and row scales of 32 steps at a time are loaded by the warp's
        // lanes in one coalesced load (a batch ahead, into registers) and published to the warp's
        // shared-memory slot; the steps read them from there, so no step waits on global memory.
        const int w = warp - kGenWarp0;
        double* s_cf = reinterpret_cast<double*>(smem + kOffCoef) + w * 128;
        double2 pcf = make_double2(0.0, 0.0);
        double pf1 = 0.0, prs = 0.0;
        auto fetch = [&](const DwtGroup* gr, long long rc0, const double2* rows, int M, int R, int base) {
            const int rr = base + lane;
            pcf = make_double2(0.0, 0.0);
            pf1 = 0.0;
            prs = 0.0;
            if (rr < R) {
                pcf = __ldg(gr->rc_cf + rc0 + rr);
                pf1 = __ldg(gr->rc_f1 + rc0 + rr);
                prs = __ldg(&rows[M + rr].x);
            }
        };
        auto publish = [&]() {
            __syncwarp();
            *reinterpret_cast<double2*>(s_cf + 4 * lane) = pcf;
            *reinterpret_cast<double2*>(s_cf + 4 * lane + 2) = make_double2(pf1, prs);
            __syncwarp();
        };
        int g = 0;
        for (int r = 0;; ++r) {
            const int idx = cta_item(r, n_items);
            if (idx < 0 || *s_abort) break;
            const ItemGeo it = item_geo<DIR>(groups, segs, nseg, idx);
            const int N = it.N, R = it.R, M = it.M;
            const DwtGroup* gr = it.gr;
            const long long rc0 = rc_offset(it.B, it.M, it.Mp);
            const double nf = gr->normf[it.cls];
            const double2* rows = row_table(gr, it.t0);
            if (DIR == 0) {
                // forward: this warp's chunks (beta columns 32c + lane), rows of the item's tile
                const int r0 = 128 * it.tile, rn = min(R - r0, 128), end = r0 + rn;
                for (int c = 0; c < it.nchunks; ++c, ++g) {
                    if ((g % kGenWarps) != w) continue;
                    const int s = g % kStages, u = g / kStages;
                    const int k = c * kKC + lane;
                    double cb = 0.0, dcur = 0.0, dprev = 0.0;
                    int sc = 0;
                    if (k < N) {
                        cb = gr->cosb[k];
                        dcur = seed_value(nf * gr->w[k], gr->pw_sin[(size_t)(it.M - it.Mp) * N + k],
                                          gr->pw_cos[(size_t)(it.M + it.Mp) * N + k], sc);
                    }
                    fetch(gr, rc0, rows, M, R, 0);
                    int base = 0;
                    for (; base < r0; base += 32) {   // second row tile: run through the first 128 degrees
                        publish();
                        fetch(gr, rc0, rows, M, R, base + 32);
#pragma unroll 8
                        for (int j = 0; j < 32; ++j)
                            rec_step(dcur, dprev, sc, cb, *reinterpret_cast<const double2*>(s_cf + 4 * j), s_cf[4 * j + 2]);
                    }
                    if (!tc::mbar_wait_bounded(&bars[kBarEmpty + s], (uint32_t)((u & 1) ^ 1), kWaitNs, s_abort)) break;
                    unsigned char* A = smem + s * kStageBytes + lane * 16;   // (k/8)*128 + (k%8)*16 = lane*16
                    for (; base < end; base += 32) {
                        publish();
                        fetch(gr, rc0, rows, M, R, base + 32);
#pragma unroll 1
                        for (int h = 0; h < 2; ++h) {
                            const int b16 = base + 16 * h;
                            if (b16 >= end) break;
                            double z[16];
#pragma unroll
                            for (int j = 0; j < 16; ++j) {
                                const int q = 16 * h + j;
                                if (b16 + j < R) {
                                    z[j] = fma(sc ? 0.0 : dcur, s_cf[4 * q + 3], kMagic);
                                    rec_step(dcur, dprev, sc, cb, *reinterpret_cast<const double2*>(s_cf + 4 * q), s_cf[4 * q + 2]);
                                } else {
                                    z[j] = kMagic;
                                }
                            }
                            if (k < N) store_unit16(A + ((b16 - r0) >> 4) * 512, kAPlane, z);
                        }
                    }
                    tc::fence_proxy_async();
                    __syncwarp();
                    if (lane == 0) tc::mbar_arrive(&bars[kBarFull + s]);
                }
            } else {
                // inverse: beta column k of the tile for this lane, 32 degrees per chunk
                const int m = 32 * w + lane;
                const int k = 128 * it.tile + m;
                double cb = 0.0, dcur = 0.0, dprev = 0.0;
                int sc = 0;
                if (k < N) {
                    cb = gr->cosb[k];
                    dcur = seed_value(nf, gr->pw_sin[(size_t)(it.M - it.Mp) * N + k], gr->pw_cos[(size_t)(it.M + it.Mp) * N + k], sc);
                }
                fetch(gr, rc0, rows, M, R, 0);
                for (int c = 0; c < it.nchunks; ++c, ++g) {
                    const int s = g % kStages, u = g / kStages;
                    publish();
                    fetch(gr, rc0, rows, M, R, (c + 1) * kKC);
                    if (!tc::mbar_wait_bounded(&bars[kBarEmpty + s], (uint32_t)((u & 1) ^ 1), kWaitNs, s_abort)) break;
                    unsigned char* A = smem + s * kStageBytes + (m >> 3) * 256 + (m & 7) * 16;
#pragma unroll 1
                    for (int h = 0; h < 2; ++h) {
                        double z[16];
#pragma unroll
                        for (int j = 0; j < 16; ++j) {
                            const int q = 16 * h + j;
                            if (c * kKC + q < R) {
                                z[j] = fma(sc ? 0.0 : dcur, s_cf[4 * q + 3], kMagic);
                                rec_step(dcur, dprev, sc, cb, *reinterpret_cast<const double2*>(s_cf + 4 * q), s_cf[4 * q + 2]);
                            } else {
                                z[j] = kMagic;
                            }
                        }
                        store_unit16(A + h * 128, kAPlane, z);
                    }
                    tc::fence_proxy_async();
                    __syncwarp();
                    if (lane == 0) tc::mbar_arrive(&bars[kBarFull + s]);
                }
            }
            if (*s_abort) break;
        }
    }

    tc::fence_before_sync();
    __syncthreads();
    if (*s_abort && tid == 0) atomicExch(status, 1);
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, kTmemCols);
    }
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

// Row scales of the generated operand, {0.49 / bound * 2^47, bound / 0.49} per degree l, bound =
// |d~^l| <= sqrt(l + 1/2) (times the largest weight for the forward's weighted rows), into the
// row table of every transform of the group. One block per transform.
__global__ void split_rows_kernel(double2* const* X, const double* w, int B, int weighted)
{
    __shared__ double red[8];
    const int N = 2 * B;
    double m = 0.0;
    if (weighted)
        for (int k = threadIdx.x; k < N; k += blockDim.x) m = fmax(m, fabs(w[k]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    double wmax = 1.0;
    if (weighted) {
        wmax = red[0];
        for (int i = 1; i < (int)(blockDim.x >> 5); ++i) wmax = fmax(wmax, red[i]);
    }
    const size_t a0 = (size_t)N * N > (size_t)8 * num_classes(B) ? (size_t)N * N : (size_t)8 * num_classes(B);
    double2* rows = X[blockIdx.z] + (size_t)N * N * N + a0;
    for (int l = threadIdx.x; l < B; l += blockDim.x) {
        const double bound = wmax * sqrt((double)l + 0.5);
        const double rs = 0.49 / bound;
        rows[l] = make_double2(rs * kTwo47, 1.0 / rs);
    }
}

}  // namespace

bool dwt_split_supported(int B) { return B >= 1 && B <= 256; }

size_t dwt_split_aux_elems(int B)
{
    const size_t n2 = (size_t)4 * B * B, c8 = (size_t)8 * num_classes(B);
    return (n2 > c8 ? n2 : c8) + (size_t)B;
}

cudaError_t dwt_split_scales(int direction, int B, int T, double2* const* d_ws, const double2* const* d_coeffs,
                             const double* w, cudaStream_t s)
{
    const int N = 2 * B;
    if (direction == 0) {
        dim3 grid((unsigned)(((long long)N * N + 7) / 8), 1, (unsigned)T);
        split_binmax_kernel<<<grid, 256, 0, s>>>(d_ws, N);
    } else {
        dim3 grid((unsigned)((num_classes(B) * 8 + 255) / 256), 1, (unsigned)T);
        split_coefmax_kernel<<<grid, 256, 0, s>>>(d_ws, d_coeffs, B);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    split_rows_kernel<<<dim3(1, 1, (unsigned)T), 256, 0, s>>>(d_ws, w, B, direction == 0 ? 1 : 0);
    return cudaGetLastError();
}

// Segments of a launch over several groups (group index, bandwidth and transform count each),
// largest bandwidth first; returns the number of items. Forward: 128-degree row tiles (two above
// B = 128); inverse: 128-column beta tiles.
int dwt_split_segments(int direction, const std::vector<int>& group, const std::vector<int>& B,
                       const std::vector<int>& T, std::vector<unsigned char>& out)
{
    std::vector<int> order(group.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return B[a] > B[b]; });
    std::vector<SplitSeg> segs;
    int first = 0;
    for (int i : order) {
        SplitSeg sg{};
        sg.group = group[i];
        sg.first = first;
        sg.T = T[i];
        sg.pairs = (T[i] + kNT - 1) / kNT;
        sg.tiles = direction == 0 ? (B[i] + 127) / 128 : (2 * B[i] + 127) / 128;
        sg.count = num_classes(B[i]) * sg.pairs * sg.tiles;
        first += sg.count;
        segs.push_back(sg);
    }
    out.resize(segs.size() * sizeof(SplitSeg));
    if (!segs.empty()) std::memcpy(out.data(), segs.data(), out.size());
    return first;
}

size_t dwt_split_seg_bytes() { return sizeof(SplitSeg); }

int g_split_sms = 0;
unsigned long long g_split_fail_ns = 0;

cudaError_t dwt_split_prepare()
{
    cudaError_t e = cudaFuncSetAttribute(dwt_split_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(dwt_split_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
    int dev = 0;
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&g_split_sms, cudaDevAttrMultiProcessorCount, dev);
    return e;
}

void dwt_split_set_fail_ns(unsigned long long ns) { g_split_fail_ns = ns; }

cudaError_t dwt_split_launch(int direction, const DwtGroup* d_groups, const void* d_segs, int nseg, int n_items,
                             int* d_status, cudaStream_t s)
{
    if (n_items <= 0 || nseg <= 0) return cudaSuccess;
    if (g_split_sms <= 0) return cudaErrorNotReady;   // dwt_split_prepare was not called
    const int blocks = n_items < g_split_sms ? n_items : g_split_sms;
    const SplitSeg* sg = static_cast<const SplitSeg*>(d_segs);
    if (direction == 0)
        dwt_split_kernel<0><<<blocks, kThreads, kSmemBytes, s>>>(d_groups, sg, nseg, n_items, d_status, g_split_fail_ns);
    else
        dwt_split_kernel<1><<<blocks, kThreads, kSmemBytes, s>>>(d_groups, sg, nseg, n_items, d_status, g_split_fail_ns);
    return cudaGetLastError();
}

}  // namespace pfsoft_dev
