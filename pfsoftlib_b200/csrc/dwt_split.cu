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
// exact in the integer sums; the epilogue combines the six planes (two 64-bit integer partial
// sums, then FP64) and undoes the scales. FP64 stays for the seeds, the recurrence, the weights
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
//
// The data operand is digitised before the launch: split_fwd_prepare_kernel (the spectrum's bin
// columns over beta) and split_inv_prepare_kernel (the scaled coefficients, degrees of a class
// gathered from the packed layout) write each column's scale entries and its digit planes, one
// block per chunk already in the B operand's shared-memory layout, so that a chunk reaches its
// stage as one untiled bulk copy (cp.async.bulk, completion on an mbarrier by the byte count).
// One CTA of 12 warps per SM, roles fixed per warp:
//   warp 0      issues the MMAs (one lane) into one of two accumulator sets in tensor memory;
//   warp 1      issues each chunk's bulk copy as soon as its stage is empty;
//   warps 4-7   epilogue: read an accumulator set back (warp w reads lanes 32(w%4) ..), combine, store;
//   warps 8-11  generators: the Wigner rows of a chunk to digit planes (forward: one warp per
//               chunk of 32 beta columns, all rows, with warps 2-3 as two more; inverse: the four
//               warps on the tile's 128 beta columns, 32 degrees per chunk; warps 2-3 idle).
// Chunks move through a ring of shared-memory stages (full by the generators, copy by the bytes,
// empty by tcgen05.commit), accumulator sets through accfull / accempty, so copies, generation,
// MMAs and the epilogue of different chunks and items overlap. Every wait is bounded
// (%globaltimer); a wait that runs out sets a CTA-wide abort flag, every role leaves, the copy
// warp waits (bounded) for its copies in flight and the MMA lane for its committed MMAs before the
// CTA ends, and *status is set to 1.
//
// Operand layouts in shared memory (no swizzle; see tc_sm100.cuh), per stage and plane:
//   A forward (MN-major, rows = degrees):  (r/16)*512 + (k/8)*128 + (k%8)*16 + (r%16)
//   A inverse (K-major, rows = beta):      (m/8)*256 + (j/16)*128 + (m%8)*16 + (j%16)
//   B both    (K-major, rows = columns):   (n/8)*256 + (k/16)*128 + (n%8)*16 + (k%16), row n =
//             16 nt p + 16 t + 2 case + (re, im) for plane p of transform t (planes concatenated
//             along N, so planes 0..5-s of every transform are one B operand of N = 16 nt (6 - s)).
// The generator inner loops carry no data-dependent branch: rows past the class's last degree
// get zero recurrence coefficients and a zero row scale (digits 0), and a column still scaled by
// 2^600 (tiny seed, see dwt.cu) is checked for its rescale once per 16 degrees.

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "dwt.cuh"
#include "dwt_common.cuh"
#include "tc_sm100.cuh"

namespace pfsoft_dev {

// Chunks of 32 degrees the inverse operand of classes 0 .. (M, M')-1 occupies (class-major copy):
// sum over m < M of (m + 1) ceil((B - m) / 32), plus M' ceil((B - M) / 32). ceil((B - m) / 32) = v
// for m in [B - 32v, B - 32(v - 1) - 1], so the sum runs over at most eight blocks.
__host__ __device__ __forceinline__ long long inv_chunk_prefix(int B, int M, int Mp)
{
    long long s = 0;
    for (int v = 1; 32 * (v - 1) < B; ++v) {
        const int lo = B - 32 * v > 0 ? B - 32 * v : 0;
        const int hi = (M - 1) < (B - 32 * (v - 1) - 1) ? (M - 1) : (B - 32 * (v - 1) - 1);
        if (hi >= lo) s += (long long)v * ((long long)(lo + hi + 2) * (hi - lo + 1) / 2);
    }
    return s + (long long)Mp * ((B - M + 31) / 32);
}

namespace {

using namespace dwtk;

constexpr int kNT = 2;                 // transforms per work item (at most)
constexpr int kPlanes = 6;             // digits per operand
constexpr int kKC = 32;                // K per chunk: one kind::i8 MMA
constexpr int kStages = 7;             // operand ring
constexpr int kAccSets = 2;
constexpr int kAccStride = 256;        // tensor-memory columns between the two accumulator sets
constexpr uint32_t kTmemCols = 512;
constexpr int kThreads = 384;
constexpr int kLoadWarp = 1;           // bulk copies of the data operand
constexpr int kEpiWarp0 = 4;
// generators: warps 8-11 in both directions; forward also warps 2-3 (one warp per chunk)
constexpr int kGenWarp0 = 8, kGenWarpsInv = 4, kGenWarpsFwd = 6;
constexpr uint64_t kWaitNs = 2000000000ull;   // 2 s

constexpr int kAPlane = 4096;                       // 128 rows x 32 bytes of K
constexpr int kABytes = kPlanes * kAPlane;          // 24 KB
constexpr int kBRows = 16 * kNT * kPlanes;          // 192
constexpr int kBBytes = kBRows / 8 * 256;           // 6 KB
constexpr int kStageBytes = kABytes + kBBytes;
// data-operand digits of one chunk and transform: 6 planes x 16 rows x 32 K (the B layout)
constexpr int kDigT = kPlanes * 512;                // 3072
constexpr int kDigPair = kNT * kDigT;               // 6144: a transform pair's block
constexpr int kOffCoef = kStages * kStageBytes;     // generators: 32 steps x {c1, f1 f2, f1, row scale} per warp
constexpr int kOffEpi = kOffCoef + kGenWarpsFwd * 32 * 4 * 8;   // epilogue: 16 x {1/scale re, im} per warp
constexpr int kSegCache = 192;                      // segments kept in shared memory (32 B each)
constexpr int kOffSeg = kOffEpi + 4 * 16 * 16;     // the first kSegCache segments of the launch
constexpr int kOffCase = kOffSeg + kSegCache * 32;  // epilogue: the item's 8 cases, 32 B each, per warp
constexpr int kOffBar = kOffCase + 4 * 8 * 32;
// mbarriers: full[kStages] (generators), copy[kStages] (the data operand's bytes), empty[kStages],
// accfull[2], accempty[2], drain, never (test knob)
constexpr int kBarFull = 0, kBarCopy = kStages, kBarEmpty = 2 * kStages, kBarAccFull = 3 * kStages,
              kBarAccEmpty = 3 * kStages + kAccSets, kBarDrain = 3 * kStages + 2 * kAccSets, kBarNever = kBarDrain + 1,
              kNumBars = kBarNever + 1;
constexpr int kOffMisc = kOffBar + kNumBars * 8;    // tensor-memory address, abort flag
constexpr int kSmemBytes = kOffMisc + 16;
static_assert(kStageBytes % 1024 == 0 && kABytes % 16 == 0, "stages stay 1 KB aligned, B operands 16 B");
static_assert(kSmemBytes <= 227 * 1024, "shared memory");
static_assert(16 * kNT * kPlanes <= kAccStride, "an accumulator set fits its column range");

constexpr double kTwo47 = 140737488355328.0;        // 2^47
// 2^52 + sum_{i<6} 128 * 256^i: adding it to x * 2^47 (|x| < 0.5) leaves round(x * 2^47) + C in
// the low 48 bits of the double, C making every byte a digit plus 128.
constexpr double kMagic = 4503599627370496.0 + 141289400074368.0;
// An integer x with |x| < 2^51 added to the bit pattern of 2^52 + 2^51 is that double plus x.
constexpr long long kI2DBits = 0x4338000000000000LL;
constexpr double kI2DMagic = 6755399441055744.0;   // 2^52 + 2^51

// One bandwidth group of a launch: items first .. first+count-1, `pairs` transform pairs (T
// transforms) and `tiles` tiles per class, bandwidth B, N = 2B.
struct SplitSeg {
    int group, first, count, pairs, tiles, T, B, N;
};
static_assert(sizeof(SplitSeg) == 32, "segment cache entries");

// Operand area past each transform's spectrum (double2 offsets from X + N^3): the column scale
// table (two double2 per (class, case)), the row table (one per degree), then the data operand as
// digit blocks, one per chunk, already in the shared-memory layout of the MMA's B operand.
// Chunk j of a class-major list (forward: j = class * ceil(N / 32) + beta chunk; inverse:
// j = inv_chunk_prefix(B, M, M') + degree chunk). A transform pair (t0, t0 + 1) keeps one 6144-byte
// block per chunk, plane p of transform t0 + h at 512 (2p + h), stored in the area of transform
// t0 + (j & 1) at (j >> 1) * 6144; an unpaired last transform keeps 3072-byte blocks (plane p at
// 512 p) in its own area at j * 3072. A chunk of an item is then a single bulk copy.
__host__ __device__ __forceinline__ size_t aux_rows(int B) { return (size_t)16 * num_classes(B); }
__host__ __device__ __forceinline__ size_t aux_dig(int B) { return aux_rows(B) + (size_t)B; }
__host__ __device__ __forceinline__ int fwd_chunks(int N) { return (N + 31) / 32; }
__host__ __device__ __forceinline__ long long dig_chunks(int B)
{
    const long long f = (long long)num_classes(B) * fwd_chunks(2 * B), i = inv_chunk_prefix(B, B, 0);
    return f > i ? f : i;
}
// Byte offset of chunk j's block in the area of transform t0 + (j & 1) (pairs) or t0 (nt = 1),
// and that transform.
__host__ __device__ __forceinline__ long long dig_block_off(int nt, long long j)
{
    return nt == 2 ? (j >> 1) * kDigPair : j * kDigT;
}
__host__ __device__ __forceinline__ int dig_block_owner(int t0, int nt, long long j)
{
    return nt == 2 ? t0 + (int)(j & 1) : t0;
}

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

// One case of an item as the epilogue stores it: bin offset (row N + col) N, orders, beta
// reversal and sign factor (class_case).
struct CaseEnt {
    long long off;
    int m1, m2, rev, pad;
    double s0;
};
static_assert(sizeof(CaseEnt) == 32, "case entry size");

// Item geometry shared by every role.
struct ItemGeo {
    const DwtGroup* gr;
    int B, N, M, Mp, R, nc, t0, nt, tile, cls, nchunks;
};

__device__ __forceinline__ int seg_first(const SplitSeg* __restrict__ segs, const SplitSeg* s_seg, int j)
{
    return j < kSegCache ? s_seg[j].first : segs[j].first;
}

// Geometry of item i: its segment by a forward scan from the caller's hint (a role visits items
// in increasing order, so the scan is short; the segment starts are in shared memory), then class,
// transform pair and tile. A forward row tile past the class's last degree has no chunks (every
// role skips it alike).
template <int DIR>
__device__ __forceinline__ ItemGeo item_geo(const DwtGroup* __restrict__ groups, const SplitSeg* __restrict__ segs,
                                            const SplitSeg* s_seg, int nseg, int i, int& hint)
{
    int sidx = hint;
    if (i < seg_first(segs, s_seg, sidx)) sidx = 0;
    while (sidx + 1 < nseg && i >= seg_first(segs, s_seg, sidx + 1)) ++sidx;
    hint = sidx;
    const SplitSeg sg = sidx < kSegCache ? s_seg[sidx] : segs[sidx];
    const int j = i - sg.first;
    const int per_cls = sg.pairs * sg.tiles;
    const int cls = j / per_cls, rem = j - cls * per_cls;
    const int pair = rem / sg.tiles;
    ItemGeo g;
    g.gr = groups + sg.group;
    g.B = sg.B;
    g.N = sg.N;
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

// A chunk of the CTA's ring: chunk c of its r-th item (idx < 0: past the last item).
struct Loc {
    int r, c, idx;
    ItemGeo it;
};

// The first chunk at or after chunk c of the CTA's r-th item (items without chunks skipped).
template <int DIR>
__device__ __forceinline__ void locate(Loc& L, int r, int c, const DwtGroup* __restrict__ groups,
                                       const SplitSeg* __restrict__ segs, const SplitSeg* s_seg, int nseg, int n_items, int& hint)
{
    for (;;) {
        L.idx = cta_item(r, n_items);
        L.r = r;
        L.c = 0;
        if (L.idx < 0) return;
        L.it = item_geo<DIR>(groups, segs, s_seg, nseg, L.idx, hint);
        if (c < L.it.nchunks) {
            L.c = c;
            return;
        }
        c -= L.it.nchunks;
        ++r;
    }
}

__device__ __forceinline__ const double2* aux_of(const DwtGroup* gr, int t)
{
    const size_t N = (size_t)gr->N;
    return gr->X[t] + N * N * N;
}

// Loads issued where they stand (volatile: not sunk towards their first use), through the
// read-only path; the value is waited for only where it is first used.
__device__ __forceinline__ double ld_early(const double* p)
{
    double v;
    asm volatile("ld.global.nc.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ double2 ld_early(const double2* p)
{
    double2 v;
    asm volatile("ld.global.nc.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
    return v;
}

// seed_value (dwt_common.cuh) with frexp / ldexp done on the bit pattern: the same value and scale
// count. The product of normal table mantissas is normal; a zero product gives 0 (unscaled).
__device__ __forceinline__ double seed_bits(double nf_w, double2 s, double2 c, int& sc)
{
    const double x = nf_w * s.x * c.x;
    const unsigned long long bits = (unsigned long long)__double_as_longlong(x);
    const int ef = (int)((bits >> 52) & 0x7FF);
    sc = 0;
    if (ef == 0) return x == 0.0 ? 0.0 : seed_value(nf_w, s, c, sc);
    const int E = ef - 1022 + (int)s.y + (int)c.y;   // frexp exponent of x plus the table exponents
    int Eo = E;
    if (E < -900) {
        sc = (-900 - E + 599) / 600;
        Eo = E + 600 * sc;
    }
    const unsigned long long r = (bits & ~(0x7FFull << 52)) | ((unsigned long long)(1022 + Eo) << 52);
    return -__longlong_as_double((long long)r);
}

// One recurrence step of a beta column (fn_dwt.hpp:167-199): d(l+1) = d(l)(f1 f2 + f1 cos b) + c1 d(l-1).
__device__ __forceinline__ void rec_step(double& dcur, double& dprev, double cb, double2 cf, double f1)
{
    const double t = fma(f1, cb, cf.y);
    const double u = cf.x * dprev;
    const double nx = fma(dcur, t, u);
    dprev = dcur;
    dcur = nx;
}

// A column whose seed was scaled by 2^600 rescales once it has grown past 2^300 (it stores 0 while
// scaled: its true magnitude is below 2^-300). Checked every 16 degrees.
__device__ __forceinline__ void rescale_check(double& dcur, double& dprev, int& sc)
{
    if (sc && fabs(dcur) >= 0x1p300) {
        dcur *= 0x1p-600;
        dprev *= 0x1p-600;
        --sc;
    }
}

// 16 recurrence steps of the lane's column from the staged coefficients s_cf[4 q + {0..3}]
// (q = q0 .. q0+15), writing the magic-biased digits of the current row before each step.
__device__ __forceinline__ void gen16(double (&z)[16], double& dcur, double& dprev, int sc, double cb,
                                      const double* s_cf, int q0)
{
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const int q = q0 + j;
        const double2 fr = *reinterpret_cast<const double2*>(s_cf + 4 * q + 2);   // {f1, row scale}
        z[j] = fma(sc ? 0.0 : dcur, fr.y, kMagic);
        rec_step(dcur, dprev, cb, *reinterpret_cast<const double2*>(s_cf + 4 * q), fr.x);
    }
}

__device__ __forceinline__ void adv16(double& dcur, double& dprev, double cb, const double* s_cf, int q0)
{
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const int q = q0 + j;
        rec_step(dcur, dprev, cb, *reinterpret_cast<const double2*>(s_cf + 4 * q), s_cf[4 * q + 2]);
    }
}

// L moved on by dc >= 0 chunks of the ring: within its item without recomputing the geometry.
template <int DIR>
__device__ __forceinline__ void advance(Loc& L, int dc, const DwtGroup* __restrict__ groups,
                                        const SplitSeg* __restrict__ segs, const SplitSeg* s_seg, int nseg, int n_items,
                                        int& hint)
{
    if (L.idx < 0) return;
    if (L.c + dc < L.it.nchunks) {
        L.c += dc;
        return;
    }
    locate<DIR>(L, L.r + 1, L.c + dc - L.it.nchunks, groups, segs, s_seg, nseg, n_items, hint);
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
    SplitSeg* s_seg = reinterpret_cast<SplitSeg*>(smem + kOffSeg);
    for (int j = tid; j < min(nseg, kSegCache); j += kThreads) s_seg[j] = segs[j];
    int hint = 0;   // this warp's segment cursor (items are visited in increasing order)

    if (warp == 0) {
        tc::tmem_alloc(s_taddr, kTmemCols);
        tc::tmem_relinquish();
    }
    if (tid == 32) {
        for (int s = 0; s < kStages; ++s) {
            tc::mbar_init(&bars[kBarFull + s], DIR == 0 ? 1 : kGenWarpsInv);   // the chunk's generator warp(s)
            tc::mbar_init(&bars[kBarCopy + s], 1);                            // arrive.expect_tx + the bytes
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
            const ItemGeo it = item_geo<DIR>(groups, segs, s_seg, nseg, idx, hint);
            if (it.nchunks == 0) continue;
            const int a = n & 1, ua = n >> 1;
            ++n;
            if (!tc::mbar_wait_bounded(&bars[kBarAccEmpty + a], (uint32_t)((ua & 1) ^ 1), kWaitNs, s_abort)) {
                ok = false;
                break;
            }
            tc::fence_after_sync();
            const uint32_t dbase = tmem + (uint32_t)(a * kAccStride);
            for (int c = 0; c < it.nchunks; ++c, ++g) {
                const int s = g % kStages, u = g / kStages;
                if (!tc::mbar_wait_bounded(&bars[kBarFull + s], (uint32_t)(u & 1), kWaitNs, s_abort) ||
                    !tc::mbar_wait_bounded(&bars[kBarCopy + s], (uint32_t)(u & 1), kWaitNs, s_abort)) {
                    ok = false;
                    break;
                }
                tc::fence_after_sync();
                if (lane == 0) {
                    const uint32_t a0 = smem_base + s * kStageBytes, b0 = a0 + kABytes;
                    const uint64_t bd = tc::sdesc(b0, 128, 256);
                    const int cols = 16 * it.nt;
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
    } else if (warp == kLoadWarp) {
        // ------------------------------------------------------------------ copies (data operand)
        // Every chunk of the ring in order: once its stage is empty, one bulk copy brings the
        // chunk's digit block (both transforms of the pair) into the stage's B operand; copy[s]
        // completes on the byte count.
        Loc cur;
        locate<DIR>(cur, 0, 0, groups, segs, s_seg, nseg, n_items, hint);
        int g = 0;
        for (; cur.idx >= 0 && !*s_abort; ++g) {
            const int s = g % kStages, u = g / kStages;
            if (!tc::mbar_wait_bounded(&bars[kBarEmpty + s], (uint32_t)((u & 1) ^ 1), kWaitNs, s_abort)) break;
            const ItemGeo& it = cur.it;
            if (lane == 0) {
                const long long j = DIR == 0 ? (long long)it.cls * fwd_chunks(it.N) + cur.c
                                             : inv_chunk_prefix(it.B, it.M, it.Mp) + cur.c;
                const unsigned char* src = reinterpret_cast<const unsigned char*>(
                                               aux_of(it.gr, dig_block_owner(it.t0, it.nt, j)) + aux_dig(it.B)) +
                                           dig_block_off(it.nt, j);
                const uint32_t bytes = (uint32_t)(kDigT * it.nt);
                tc::mbar_arrive_expect_tx(&bars[kBarCopy + s], bytes);
                tc::bulk_g2s(smem + s * kStageBytes + kABytes, src, bytes, &bars[kBarCopy + s]);
            }
            __syncwarp();
            advance<DIR>(cur, 1, groups, segs, s_seg, nseg, n_items, hint);
        }
        // the copies of the last phases armed on each stage have landed before the CTA can end
        if (lane == 0)
            for (int k = 1; k <= kStages && g - k >= 0; ++k) {
                const int gg = g - k;
                const uint64_t t0 = tc::globaltimer_ns();
                while (!tc::mbar_try_wait(&bars[kBarCopy + gg % kStages], (uint32_t)((gg / kStages) & 1)))
                    if (tc::globaltimer_ns() - t0 > kWaitNs) break;
            }
        __syncwarp();
    } else if (warp >= kEpiWarp0 && warp < kEpiWarp0 + 4) {
        // ------------------------------------------------------------------ epilogue
        // The next item's column scales (lane i < 16: transform i / 8, case i % 8) and, forward, the
        // lane's row scale are loaded while the current item is read back; the current item's
        // column scales go through the warp's shared-memory slot.
        const int q4 = warp & 3;   // tensor-memory lane quarter
        const int row = 32 * q4 + lane;
        double2* s_ics = reinterpret_cast<double2*>(smem + kOffEpi) + 16 * q4;
        CaseEnt* s_ce = reinterpret_cast<CaseEnt*>(smem + kOffCase) + 8 * q4;
        auto next_item = [&](int& r) -> int {
            for (;; ++r) {
                const int idx = cta_item(r, n_items);
                if (idx < 0) return -1;
                if (item_geo<DIR>(groups, segs, s_seg, nseg, idx, hint).nchunks > 0) return idx;
            }
        };
        auto load_scales = [&](const ItemGeo& it, double2& ics, double& rowf) {
            const int t = lane >> 3, q = lane & 7;
            ics = make_double2(1.0, 1.0);
            if (lane < 16 && t < it.nt && q < it.nc) ics = ld_early(aux_of(it.gr, it.t0 + t) + (size_t)2 * (8 * it.cls + q) + 1);
            rowf = 0.0;
            const int l = it.M + 128 * it.tile + row;
            if (DIR == 0 && l < it.B) rowf = ld_early(&aux_of(it.gr, it.t0)[aux_rows(it.B) + l].y);
        };
        int r = 0;
        int idx = next_item(r);
        ItemGeo it{};
        double2 ics_c = make_double2(1.0, 1.0);
        double rowf_c = 0.0;
        if (idx >= 0) {
            it = item_geo<DIR>(groups, segs, s_seg, nseg, idx, hint);
            load_scales(it, ics_c, rowf_c);
        }
        int n = 0;
        while (idx >= 0) {
            ++r;
            const int nidx = next_item(r);
            ItemGeo nit{};
            double2 ics_n = make_double2(1.0, 1.0);
            double rowf_n = 0.0;
            if (nidx >= 0) {
                nit = item_geo<DIR>(groups, segs, s_seg, nseg, nidx, hint);
                load_scales(nit, ics_n, rowf_n);
            }
            const int a = n & 1, ua = n >> 1;
            ++n;
            if (!tc::mbar_wait_bounded(&bars[kBarAccFull + a], (uint32_t)(ua & 1), kWaitNs, s_abort)) break;
            tc::fence_after_sync();
            __syncwarp();
            if (lane < 16) s_ics[lane] = make_double2(ics_c.x * 0x1p-30, ics_c.y * 0x1p-30);   // powers of two: exact
            const int N = it.N, B = it.B;
            if (lane < it.nc) {   // the item's cases, once per item instead of per lane and value
                const PairCase p = class_case(it.M, it.Mp, lane, N);
                CaseEnt ce;
                ce.off = ((long long)p.row * N + p.col) * N;
                ce.m1 = p.m1;
                ce.m2 = p.m2;
                ce.rev = p.rev;
                ce.pad = 0;
                ce.s0 = p.s0;
                s_ce[lane] = ce;
            }
            __syncwarp();
            const uint32_t taddr = tmem + ((uint32_t)(32 * q4) << 16) + (uint32_t)(a * kAccStride);
            // forward: degree l of this lane; inverse: beta k
            const int l = it.M + 128 * it.tile + row;
            const int k = 128 * it.tile + row;
            const bool live = DIR == 0 ? (l < B) : (k < N);
            const int Ll = 2 * l + 1;
            const long long coff = DIR == 0 ? (long long)coef_offset(l) : 0;
            const double fnorm = DIR == 0 ? (kPi / (double)(B * 2 * B)) * rowf_c : 0.0;   // src/fn_dsoft.cpp:119
            for (int t = 0; t < it.nt; ++t) {
                double2* const outp = DIR == 0 ? it.gr->coeffs[it.t0 + t] : it.gr->X[it.t0 + t];
                int32_t acc[kPlanes][16];
#pragma unroll
                for (int e = 0; e < kPlanes; ++e) tc::tmem_ld16(taddr + (uint32_t)(16 * it.nt * e + 16 * t), acc[e]);
                tc::tmem_wait_ld();
                double v[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    // sum_e acc[e] 2^(-8e) = 2^-16 (hi + 2^-24 lo), hi and lo exact in 64 bits (|.| < 2^43);
                    // each converted exactly by adding it to the bits of 2^52 + 2^51 (FP64 add, no
                    // 64-bit integer conversion); the 2^-30 (2^-16 and the digits' 2^-14) rides in ics
                    const long long hi = (long long)acc[0][j] * 65536 + (long long)acc[1][j] * 256 + acc[2][j];
                    const long long lo = (long long)acc[3][j] * 65536 + (long long)acc[4][j] * 256 + acc[5][j];
                    const double hd = __longlong_as_double(hi + kI2DBits) - kI2DMagic;
                    const double ld = __longlong_as_double(lo + kI2DBits) - kI2DMagic;
                    v[j] = fma(ld, 0x1p-24, hd);
                }
                if (!live) continue;
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    if (q >= it.nc) break;
                    const CaseEnt ce = s_ce[q];
                    const double2 ics = s_ics[8 * t + q];
                    if (DIR == 0) {
                        // coef_index(l, m1, m2) and case_sign of class_case(M, M', q)
                        const int i1 = ce.m1 >= 0 ? ce.m1 : Ll + ce.m1, i2 = ce.m2 >= 0 ? ce.m2 : Ll + ce.m2;
                        const double f = fnorm * ((ce.rev && ((l - it.M) & 1)) ? -ce.s0 : ce.s0);
                        outp[coff + (long long)i2 * Ll + i1] = make_double2(f * v[2 * q] * ics.x, f * v[2 * q + 1] * ics.y);
                    } else {
                        outp[ce.off + (ce.rev ? N - 1 - k : k)] = make_double2(v[2 * q] * ics.x, v[2 * q + 1] * ics.y);
                    }
                }
            }
            tc::fence_before_sync();
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(&bars[kBarAccEmpty + a]);
            idx = nidx;
            it = nit;
            ics_c = ics_n;
            rowf_c = rowf_n;
        }
    } else if (warp >= kGenWarp0 || (DIR == 0 && warp > kLoadWarp && warp < kEpiWarp0)) {
        // ------------------------------------------------------------------ generators (Wigner rows)
        // The recurrence coefficients and row scales of 32 steps at a time are loaded by the warp's
        // lanes in one coalesced load (a batch ahead, into registers) and published to the warp's
        // shared-memory slot; the steps read them from there, so no step waits on global memory.
        // Rows past the class's last degree get zero coefficients and a zero row scale.
        constexpr int GW = DIR == 0 ? kGenWarpsFwd : kGenWarpsInv;
        const int w = warp >= kGenWarp0 ? warp - kGenWarp0 : kGenWarpsInv + warp - (kLoadWarp + 1);
        double* s_cf = reinterpret_cast<double*>(smem + kOffCoef) + w * 128;
        double2 pcf = make_double2(0.0, 0.0);
        double pf1 = 0.0, prs = 0.0;
        auto fetch = [&](const DwtGroup* gr, long long rc0, const double2* rows, int M, int R, int base) {
            const int rr = base + lane;
            pcf = make_double2(0.0, 0.0);
            pf1 = 0.0;
            prs = 0.0;
            if (rr < R) {
                pcf = ld_early(gr->rc_cf + rc0 + rr);
                pf1 = ld_early(gr->rc_f1 + rc0 + rr);
                prs = ld_early(&rows[M + rr].x);
            }
        };
        auto publish = [&]() {
            __syncwarp();
            *reinterpret_cast<double2*>(s_cf + 4 * lane) = pcf;
            *reinterpret_cast<double2*>(s_cf + 4 * lane + 2) = make_double2(pf1, prs);
            __syncwarp();
        };
        // The chunks of this warp, in ring order, with the seed inputs and the first coefficient
        // batch of the next one loaded while the current one is generated.
        auto locate_g = [&](Loc& L, int r, int c) { locate<DIR>(L, r, c, groups, segs, s_seg, nseg, n_items, hint); };
        struct SeedIn {
            double cb, wk, nf;
            double2 ps, pc;
        };
        auto load_seed = [&](const Loc& L, SeedIn& si) {
            si.cb = 0.0;
            si.wk = 1.0;
            si.nf = 0.0;
            si.ps = make_double2(0.0, 0.0);
            si.pc = make_double2(0.0, 0.0);
            if (L.idx < 0) return;
            const DwtGroup* gr = L.it.gr;
            const int N = L.it.N;
            const int k = DIR == 0 ? L.c * kKC + lane : 128 * L.it.tile + 32 * w + lane;
            if (k < N) {
                si.cb = ld_early(gr->cosb + k);
                if (DIR == 0) si.wk = ld_early(gr->w + k);
                si.ps = ld_early(gr->pw_sin + (size_t)(L.it.M - L.it.Mp) * N + k);
                si.pc = ld_early(gr->pw_cos + (size_t)(L.it.M + L.it.Mp) * N + k);
            }
            si.nf = ld_early(gr->normf + L.it.cls);
        };
        auto fetch_loc = [&](const Loc& L, int base) {
            if (L.idx < 0) {
                pcf = make_double2(0.0, 0.0);
                pf1 = 0.0;
                prs = 0.0;
                return;
            }
            fetch(L.it.gr, rc_offset(L.it.B, L.it.M, L.it.Mp), aux_of(L.it.gr, L.it.t0) + aux_rows(L.it.B), L.it.M, L.it.R,
                  base);
        };
        Loc cur;
        locate_g(cur, 0, DIR == 0 ? w : 0);
        int g = DIR == 0 ? w : 0;
        SeedIn si;
        load_seed(cur, si);
        fetch_loc(cur, 0);
        while (cur.idx >= 0 && !*s_abort) {
            Loc nx;
            if (DIR == 0) {
                nx = cur;
                advance<DIR>(nx, GW, groups, segs, s_seg, nseg, n_items, hint);
            } else {
                locate_g(nx, cur.r + 1, 0);
            }
            SeedIn sn;
            load_seed(nx, sn);
            const ItemGeo& it = cur.it;
            const int N = it.N, R = it.R;
            bool stop = false;
            if (DIR == 0) {
                // forward: beta columns 32c + lane of this warp's chunk c, rows of the item's tile
                const int s = g % kStages, u = g / kStages;
                const int k = cur.c * kKC + lane;
                const int r0 = 128 * it.tile, end = r0 + min(R - r0, 128);
                const double cb = si.cb;
                double dcur = 0.0, dprev = 0.0;
                int sc = 0;
                if (k < N) dcur = seed_bits(si.nf * si.wk, si.ps, si.pc, sc);
                bool scaled = __any_sync(0xffffffffu, sc > 0);
                int base = 0;
                for (; base < r0; base += 32) {   // second row tile: run through the first 128 degrees
                    publish();
                    fetch_loc(cur, base + 32);
#pragma unroll 1
                    for (int h = 0; h < 2; ++h) {
                        adv16(dcur, dprev, cb, s_cf, 16 * h);
                        if (scaled) {
                            rescale_check(dcur, dprev, sc);
                            scaled = __any_sync(0xffffffffu, sc > 0);
                        }
                    }
                }
                if (!tc::mbar_wait_bounded(&bars[kBarEmpty + s], (uint32_t)((u & 1) ^ 1), kWaitNs, s_abort)) break;
                unsigned char* A = smem + s * kStageBytes + lane * 16;   // (k/8)*128 + (k%8)*16 = lane*16
                for (; base < end; base += 32) {
                    publish();
                    if (base + 32 < end)
                        fetch_loc(cur, base + 32);
                    else
                        fetch_loc(nx, 0);
#pragma unroll 1
                    for (int h = 0; h < 2; ++h) {
                        const int b16 = base + 16 * h;
                        if (b16 >= end) break;
                        double z[16];
                        gen16(z, dcur, dprev, sc, cb, s_cf, 16 * h);
                        if (scaled) {
                            rescale_check(dcur, dprev, sc);
                            scaled = __any_sync(0xffffffffu, sc > 0);
                        }
                        if (k < N) store_unit16(A + ((b16 - r0) >> 4) * 512, kAPlane, z);
                    }
                }
                tc::fence_proxy_async();
                __syncwarp();
                if (lane == 0) tc::mbar_arrive(&bars[kBarFull + s]);
                g += GW;
            } else {
                // inverse: beta column k of the tile for this lane, 32 degrees per chunk
                const int m = 32 * w + lane;
                const int k = 128 * it.tile + m;
                const double cb = si.cb;
                double dcur = 0.0, dprev = 0.0;
                int sc = 0;
                if (k < N) dcur = seed_bits(si.nf, si.ps, si.pc, sc);
                bool scaled = __any_sync(0xffffffffu, sc > 0);
                for (int c = 0; c < it.nchunks; ++c, ++g) {
                    const int s = g % kStages, u = g / kStages;
                    publish();
                    if (c + 1 < it.nchunks)
                        fetch_loc(cur, (c + 1) * kKC);
                    else
                        fetch_loc(nx, 0);
                    if (!tc::mbar_wait_bounded(&bars[kBarEmpty + s], (uint32_t)((u & 1) ^ 1), kWaitNs, s_abort)) {
                        stop = true;
                        break;
                    }
                    unsigned char* A = smem + s * kStageBytes + (m >> 3) * 256 + (m & 7) * 16;
#pragma unroll 1
                    for (int h = 0; h < 2; ++h) {
                        double z[16];
                        gen16(z, dcur, dprev, sc, cb, s_cf, 16 * h);
                        if (scaled) {
                            rescale_check(dcur, dprev, sc);
                            scaled = __any_sync(0xffffffffu, sc > 0);
                        }
                        store_unit16(A + h * 128, kAPlane, z);
                    }
                    tc::fence_proxy_async();
                    __syncwarp();
                    if (lane == 0) tc::mbar_arrive(&bars[kBarFull + s]);
                }
                if (stop) break;
            }
            cur = nx;
            si = sn;
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

// Digits of one value pair (re, im of chunk position k = lane, case q) into the shared-memory image
// of a class's digit blocks for one transform: chunk i at i * 3072, plane p at + 512 p, rows
// 2q (re) and 2q + 1 (im) in the B operand's layout.
__device__ __forceinline__ void digits_to_image(unsigned char* img, int i, int q, int lane, double2 v, double2 cs)
{
    const double zr = fma(v.x, cs.x, kMagic), zi = fma(v.y, cs.y, kMagic);
    const unsigned long long br = (unsigned long long)__double_as_longlong(zr);
    const unsigned long long bi = (unsigned long long)__double_as_longlong(zi);
    const int r = 2 * q;
    unsigned char* u = img + i * kDigT + (r >> 3) * 256 + (lane >> 4) * 128 + (r & 7) * 16 + (lane & 15);
#pragma unroll
    for (int p = 0; p < kPlanes; ++p) {   // plane p: byte 5 - p, most significant first
        u[p * 512] = (unsigned char)(br >> (8 * (5 - p))) ^ 0x80;
        u[p * 512 + 16] = (unsigned char)(bi >> (8 * (5 - p))) ^ 0x80;
    }
}

// The image of `nch` chunks (first chunk j0 of the class-major list) to the digit blocks of
// transform t of a group of T: plane p of chunk i to its block at 512 (nt p + h), 512 bytes per
// warp store. All threads of the CTA.
__device__ __forceinline__ void image_to_blocks(const unsigned char* img, double2* const* X, int t, int T, int B,
                                                long long j0, int nch)
{
    const size_t N = (size_t)(2 * B);
    const int t0 = t & ~1, nt = T - t0 < kNT ? T - t0 : kNT, h = t - t0;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int pc = warp; pc < nch * kPlanes; pc += (int)(blockDim.x >> 5)) {
        const int i = pc / kPlanes, p = pc - kPlanes * i;
        const long long j = j0 + i;
        unsigned char* blk = reinterpret_cast<unsigned char*>(X[dig_block_owner(t0, nt, j)] + N * N * N + aux_dig(B)) +
                             dig_block_off(nt, j);
        const uint4 v = reinterpret_cast<const uint4*>(img + i * kDigT + p * 512)[lane];
        reinterpret_cast<uint4*>(blk + 512 * (nt * p + h))[lane] = v;
    }
}

// Column scale entries of (class, case) {scale * 2^47 re, im}, {1 / scale re, im} from the
// column's largest |re|, |im| (the warp's lanes' maxima reduced here).
__device__ __forceinline__ double2 column_scales(double mre, double mim, double2* tab_entry, int lane)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mre = fmax(mre, __shfl_xor_sync(0xffffffffu, mre, o));
        mim = fmax(mim, __shfl_xor_sync(0xffffffffu, mim, o));
    }
    double cr, ci, ir, ii;
    column_scale(mre, cr, ir);
    column_scale(mim, ci, ii);
    if (lane == 0) {
        tab_entry[0] = make_double2(cr, ci);
        tab_entry[1] = make_double2(ir, ii);
    }
    return make_double2(cr, ci);
}

// Forward operand: for every class, the bin columns of its eight cases over beta (chunk position k
// holds beta k, or N - 1 - k for a reversed case; zero past N and for absent cases), their column
// scales into the scale table and their digits into the class's ceil(N / 32) <= NCM digit blocks.
// One CTA of eight warps (warp = case) per (class, transform), gridDim.z = the group's T
// transforms; lane k reads position 32 i + k of its column (coalesced), the digits go through a
// shared-memory image of the blocks and leave as whole 512-byte plane pieces. Dynamic shared
// memory NCM * 3072 bytes.
template <int NCM>
__global__ void __launch_bounds__(256, NCM == 8 ? 4 : 3) split_fwd_prepare_kernel(double2* const* X, int B, int T)
{
    extern __shared__ __align__(16) unsigned char img[];
    const int N = 2 * B, NC = fwd_chunks(N);
    const int cls = blockIdx.x, t = blockIdx.z, q = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int M, Mp;
    class_orders(cls, M, Mp);
    const bool live = q < class_case_count(M, Mp);
    const PairCase p = class_case(M, Mp, live ? q : 0, N);
    const double2* col = X[t] + ((size_t)p.row * N + p.col) * N;
    double2 v[NCM];
    double mre = 0.0, mim = 0.0;
#pragma unroll
    for (int i = 0; i < NCM; ++i) {
        v[i] = make_double2(0.0, 0.0);
        const int k = kKC * i + lane;
        if (i < NC && live && k < N) {
            v[i] = __ldg(col + (p.rev ? N - 1 - k : k));
            mre = fmax(mre, fabs(v[i].x));
            mim = fmax(mim, fabs(v[i].y));
        }
    }
    double2* tab = X[t] + (size_t)N * N * N + (size_t)2 * (8 * cls + q);
    const double2 cs = column_scales(mre, mim, tab, lane);
#pragma unroll
    for (int i = 0; i < NCM; ++i)
        if (i < NC) digits_to_image(img, i, q, lane, v[i], cs);
    __syncthreads();
    image_to_blocks(img, X, t, T, B, (long long)cls * NC, NC);
}

// Inverse operand: for every (class, case) the column G[l] = (2B^2/pi) sign(l) f^l / (row scale of
// l), l = M..B-1 (src/fn_idsoft.cpp:109; zero past B - 1 and for absent cases), its column scales
// into the scale table and its digits into the class's ceil((B - M) / 32) digit blocks. One CTA of
// eight warps (warp = case) per (class, transform), gridDim.z = the group's T transforms; the row
// table must be written first.
__global__ void split_inv_prepare_kernel(double2* const* X, const double2* const* coeffs, int B, int T)
{
    __shared__ __align__(16) unsigned char img[8 * kDigT];
    const int N = 2 * B;
    const int cls = blockIdx.x, t = blockIdx.z, q = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int M, Mp;
    class_orders(cls, M, Mp);
    const int nch = (B - M + kKC - 1) / kKC;
    double2* aux = X[t] + (size_t)N * N * N;
    const double2* rows = aux + aux_rows(B);
    const bool live = q < class_case_count(M, Mp);
    const PairCase p = class_case(M, Mp, live ? q : 0, N);
    const double2* cf = coeffs[t];
    const double norm = (double)(B * 2 * B) / kPi;
    double2 v[8];
    double mre = 0.0, mim = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        v[i] = make_double2(0.0, 0.0);
        const int l = M + kKC * i + lane;
        if (i < nch && live && l < B) {
            const double f = norm * case_sign(p, l, M) * __ldg(&rows[l].y);
            const double2 x = __ldg(cf + coef_index(l, p.m1, p.m2));
            v[i] = make_double2(f * x.x, f * x.y);
            mre = fmax(mre, fabs(v[i].x));
            mim = fmax(mim, fabs(v[i].y));
        }
    }
    const double2 cs = column_scales(mre, mim, aux + (size_t)2 * (8 * cls + q), lane);
#pragma unroll
    for (int i = 0; i < 8; ++i)
        if (i < nch) digits_to_image(img, i, q, lane, v[i], cs);
    __syncthreads();
    image_to_blocks(img, X, t, T, B, inv_chunk_prefix(B, M, Mp), nch);
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
    double2* rows = X[blockIdx.z] + (size_t)N * N * N + aux_rows(B);
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
    return aux_dig(B) + (size_t)(kDigPair / 16) * (size_t)((dig_chunks(B) + 1) / 2);
}

cudaError_t dwt_split_scales(int direction, int B, int T, double2* const* d_ws, const double2* const* d_coeffs,
                             const double* w, cudaStream_t s)
{
    split_rows_kernel<<<dim3(1, 1, (unsigned)T), 256, 0, s>>>(d_ws, w, B, direction == 0 ? 1 : 0);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    dim3 grid((unsigned)num_classes(B), 1, (unsigned)T);
    if (direction == 0)
        if (fwd_chunks(2 * B) <= 8)
            split_fwd_prepare_kernel<8><<<grid, 256, (size_t)fwd_chunks(2 * B) * kDigT, s>>>(d_ws, B, T);
        else
            split_fwd_prepare_kernel<16><<<grid, 256, (size_t)fwd_chunks(2 * B) * kDigT, s>>>(d_ws, B, T);
    else
        split_inv_prepare_kernel<<<grid, 256, 0, s>>>(d_ws, d_coeffs, B, T);
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
        sg.B = B[i];
        sg.N = 2 * B[i];
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
