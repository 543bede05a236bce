// Batched 1D DFT passes over the (alpha, gamma) plane of every beta layer (sm_100a).
//
// Algorithm: mixed-radix Stockham autosort (Govindaraju et al., SC'08 formulation). A stage of
// radix R over n points with Ns = product of the earlier radices maps butterfly j to
//   inputs  x[j + r*n/R] * w_n^(r * (j mod Ns) * n/(Ns R)),   r < R
//   outputs y[(j/Ns)*Ns*R + (j mod Ns) + q*Ns],              q < R
// and the last stage leaves the result in natural order. The first stage reads HBM directly
// into registers and the last stage writes HBM directly from registers; the stages between
// exchange through shared memory (ping-pong buffers). Radices 2, 4, 8, 16, 3, 5 have
// register butterflies; any other prime uses a direct O(R^2) butterfly.
//
// Coalescing: each stage picks its butterfly -> thread map from the stride of the HBM side
// it touches. If consecutive elements of a vector are contiguous in HBM (se == 1) threads run
// along the vector; otherwise threads run across the KB vectors of the tile, whose values are
// contiguous (sv == 1), so KB*16 bytes move per group of KB lanes. That is how the beta <->
// (alpha, gamma) transpose rides inside the first and last stage at no extra HBM traffic.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "fft.cuh"

namespace pfsoft_dev {

namespace {

constexpr double kSqrtHalf = 0.70710678118654752440084436210485;
constexpr double kCosPi8 = 0.92387953251128675612818318939679;   // cos(pi/8)
constexpr double kSinPi8 = 0.38268343236508977172845998403040;   // sin(pi/8)
constexpr double kSin60 = 0.86602540378443864676372317075294;    // sin(pi/3)
constexpr double kC5_1 = 0.30901699437494742410229341718282;     // cos(2pi/5)
constexpr double kC5_2 = -0.80901699437494742410229341718282;    // cos(4pi/5)
constexpr double kS5_1 = 0.95105651629515357211643933337938;     // sin(2pi/5)
constexpr double kS5_2 = 0.58778525229247312916870595463907;     // sin(4pi/5)

template <int SIGN>
__device__ __forceinline__ void dft2(double2* v)
{
    double2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
}

template <int SIGN>
__device__ __forceinline__ void dft4(double2& v0, double2& v1, double2& v2, double2& v3)
{
    double2 a0 = cadd(v0, v2), a1 = csub(v0, v2);
    double2 b0 = cadd(v1, v3), b1 = cmul_i<SIGN>(csub(v1, v3));
    v0 = cadd(a0, b0);
    v2 = csub(a0, b0);
    v1 = cadd(a1, b1);
    v3 = csub(a1, b1);
}

// w8^q = exp(SIGN*2*pi*i*q/8)
template <int SIGN, int Q>
__device__ __forceinline__ double2 rot8(double2 a)
{
    if (Q == 0) return a;
    if (Q == 2) return cmul_i<SIGN>(a);
    if (Q == 1) return make_double2(kSqrtHalf * (a.x - SIGN * a.y), kSqrtHalf * (a.y + SIGN * a.x));
    // Q == 3: (-1 + SIGN i)/sqrt2
    return make_double2(kSqrtHalf * (-a.x - SIGN * a.y), kSqrtHalf * (-a.y + SIGN * a.x));
}

template <int SIGN>
__device__ __forceinline__ void dft8(double2* v)
{
    // even/odd split: E = DFT4(v0 v2 v4 v6), O = DFT4(v1 v3 v5 v7)
    dft4<SIGN>(v[0], v[2], v[4], v[6]);
    dft4<SIGN>(v[1], v[3], v[5], v[7]);
    double2 o1 = rot8<SIGN, 1>(v[3]), o2 = rot8<SIGN, 2>(v[5]), o3 = rot8<SIGN, 3>(v[7]);
    double2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6], o0 = v[1];
    v[0] = cadd(e0, o0);
    v[4] = csub(e0, o0);
    v[1] = cadd(e1, o1);
    v[5] = csub(e1, o1);
    v[2] = cadd(e2, o2);
    v[6] = csub(e2, o2);
    v[3] = cadd(e3, o3);
    v[7] = csub(e3, o3);
}

template <int SIGN>
__device__ __forceinline__ void dft16(double2* v)
{
    double2 e[8], o[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        e[i] = v[2 * i];
        o[i] = v[2 * i + 1];
    }
    dft8<SIGN>(e);
    dft8<SIGN>(o);
    // w16^q = (cos(pi q/8), SIGN sin(pi q/8))
    const double cq[8] = {1.0, kCosPi8, kSqrtHalf, kSinPi8, 0.0, -kSinPi8, -kSqrtHalf, -kCosPi8};
    const double sq[8] = {0.0, kSinPi8, kSqrtHalf, kCosPi8, 1.0, kCosPi8, kSqrtHalf, kSinPi8};
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        double2 t = (q == 0) ? o[0] : make_double2(cq[q] * o[q].x - SIGN * sq[q] * o[q].y,
                                                    cq[q] * o[q].y + SIGN * sq[q] * o[q].x);
        v[q] = cadd(e[q], t);
        v[q + 8] = csub(e[q], t);
    }
}

template <int SIGN>
__device__ __forceinline__ void dft3(double2* v)
{
    double2 t1 = cadd(v[1], v[2]);
    double2 t2 = csub(v[1], v[2]);
    double2 a = make_double2(v[0].x - 0.5 * t1.x, v[0].y - 0.5 * t1.y);
    double2 b = cmul_i<SIGN>(cscale(t2, kSin60));
    v[0] = cadd(v[0], t1);
    v[1] = cadd(a, b);
    v[2] = csub(a, b);
}

template <int SIGN>
__device__ __forceinline__ void dft5(double2* v)
{
    double2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
    double2 t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
    double2 a1 = make_double2(v[0].x + kC5_1 * t1.x + kC5_2 * t2.x, v[0].y + kC5_1 * t1.y + kC5_2 * t2.y);
    double2 a2 = make_double2(v[0].x + kC5_2 * t1.x + kC5_1 * t2.x, v[0].y + kC5_2 * t1.y + kC5_1 * t2.y);
    double2 b1 = cmul_i<SIGN>(make_double2(kS5_1 * t3.x + kS5_2 * t4.x, kS5_1 * t3.y + kS5_2 * t4.y));
    double2 b2 = cmul_i<SIGN>(make_double2(kS5_2 * t3.x - kS5_1 * t4.x, kS5_2 * t3.y - kS5_1 * t4.y));
    v[0] = cadd(v[0], cadd(t1, t2));
    v[1] = cadd(a1, b1);
    v[4] = csub(a1, b1);
    v[2] = cadd(a2, b2);
    v[3] = csub(a2, b2);
}

__device__ __forceinline__ double2 twiddle(const double2* __restrict__ tw, int t, int sign)
{
    double2 w = __ldg(tw + t);
    return sign < 0 ? w : make_double2(w.x, -w.y);
}

// First-stage load of a pass: the read-only path, unless the pass reads what another CTA of the
// same launch wrote (the second pass of fft_fused_kernel), which needs coherent loads.
__device__ __forceinline__ double2 load_src(const FftPassArgs& a, const double2* p)
{
    if (a.coherent) return __ldcg(p);   // L2, where the other CTAs' stores are
    return __ldg(p);
}

// Last-stage store of a pass: evict-first when the pass's output is not reread through L2
// (measured at B = 128: -1.0 % iDSOFT, -0.5 % DSOFT; neutral at B = 256).
__device__ __forceinline__ void store_out(const FftPassArgs& a, double2* p, double2 v)
{
    if (a.stream_out)
        __stcs(p, v);
    else
        *p = v;
}

// smem position of element i of a vector (one pad slot every 16 elements)
__device__ __forceinline__ int spos(int i) { return i + (i >> 4); }

__host__ __device__ __forceinline__ int padded_len(int n) { return n + (n >> 4) + 1; }

template <int SIGN, int R>
__device__ __forceinline__ void run_stage_fixed(const FftPassArgs& a, int s, const double2* gsrc,
                                                double2* gdst, const double2* sin_, double2* sout,
                                                int nv, long long src_base, long long dst_base)
{
    const int n = a.n;
    const int m = n / R;
    const int Ns = a.ns[s];
    const int step = n / (Ns * R);
    const bool first = (s == 0), last = (s == a.nstages - 1);
    const int pl = padded_len(n);
    // thread map: along the vector (j fastest) unless this stage touches HBM with a non-unit
    // element stride, in which case across vectors (kk fastest)
    const bool kk_fast = (first && a.src.se != 1) || (last && a.dst.se != 1);
    const int total = nv * m;
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        int j, kk;
        if (kk_fast) {
            kk = t % nv;
            j = t / nv;
        } else {
            j = t % m;
            kk = t / m;
        }
        double2 v[R];
        if (first) {
            const double2* p = gsrc + src_base + (long long)kk * a.src.sv;
#pragma unroll
            for (int r = 0; r < R; ++r) v[r] = load_src(a, p + (long long)(j + r * m) * a.src.se);
        } else {
            const double2* p = sin_ + kk * pl;
#pragma unroll
            for (int r = 0; r < R; ++r) v[r] = p[spos(j + r * m)];
        }
        const int k = j % Ns;
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) v[r] = cmul(v[r], twiddle(a.twiddle, r * k * step, SIGN));
        }
        if (R == 1) {
        } else if (R == 2) dft2<SIGN>(v);
        else if (R == 4) dft4<SIGN>(v[0], v[1], v[2], v[3]);
        else if (R == 8) dft8<SIGN>(v);
        else if (R == 16) dft16<SIGN>(v);
        else if (R == 3) dft3<SIGN>(v);
        else if (R == 5) dft5<SIGN>(v);
        const int ob = (j / Ns) * Ns * R + k;
        if (last) {
            double2* p = gdst + dst_base + (long long)kk * a.dst.sv;
#pragma unroll
            for (int q = 0; q < R; ++q) store_out(a, p + (long long)(ob + q * Ns) * a.dst.se, cscale(v[q], a.scale));
        } else {
            double2* p = sout + kk * pl;
#pragma unroll
            for (int q = 0; q < R; ++q) p[spos(ob + q * Ns)] = v[q];
        }
    }
}

// One stage of the in-place kernel: each thread owns up to P butterflies of radix R (its
// threadIdx.x + p * blockDim.x), on a single shared buffer. A stage that reads shared memory and
// writes it (a middle stage) loads all of its inputs, waits for the whole CTA, then overwrites
// the buffer with its outputs. All threads reach the barrier.
template <int SIGN, int R, int P>
__device__ __forceinline__ void run_stage_inplace(const FftPassArgs& a, int s, const double2* gsrc,
                                                  double2* gdst, double2* buf, int nv,
                                                  long long src_base, long long dst_base)
{
    const int n = a.n;
    const int m = n / R;
    const int Ns = a.ns[s];
    const int step = n / (Ns * R);
    const bool first = (s == 0), last = (s == a.nstages - 1);
    const int pl = padded_len(n);
    const bool kk_fast = (first && a.src.se != 1) || (last && a.dst.se != 1);
    int j[P], kk[P];
    bool act[P];
    double2 v[P][R];
#pragma unroll
    for (int p = 0; p < P; ++p) {
        const int t = threadIdx.x + p * blockDim.x;
        act[p] = t < nv * m;
        if (kk_fast) {
            kk[p] = t % nv;
            j[p] = t / nv;
        } else {
            j[p] = t % m;
            kk[p] = t / m;
        }
        if (act[p]) {
            if (first) {
                const double2* q = gsrc + src_base + (long long)kk[p] * a.src.sv;
#pragma unroll
                for (int r = 0; r < R; ++r) v[p][r] = load_src(a, q + (long long)(j[p] + r * m) * a.src.se);
            } else {
                const double2* q = buf + kk[p] * pl;
#pragma unroll
                for (int r = 0; r < R; ++r) v[p][r] = q[spos(j[p] + r * m)];
            }
        }
    }
    if (!first && !last) __syncthreads();   // every input read before any output lands
#pragma unroll
    for (int p = 0; p < P; ++p) {
        if (!act[p]) continue;
        const int k = j[p] % Ns;
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) v[p][r] = cmul(v[p][r], twiddle(a.twiddle, r * k * step, SIGN));
        }
        if (R == 2) dft2<SIGN>(v[p]);
        else if (R == 4) dft4<SIGN>(v[p][0], v[p][1], v[p][2], v[p][3]);
        else if (R == 8) dft8<SIGN>(v[p]);
        else if (R == 3) dft3<SIGN>(v[p]);
        else if (R == 5) dft5<SIGN>(v[p]);
        const int ob = (j[p] / Ns) * Ns * R + k;
        if (last) {
            double2* q = gdst + dst_base + (long long)kk[p] * a.dst.sv;
#pragma unroll
            for (int c = 0; c < R; ++c) store_out(a, q + (long long)(ob + c * Ns) * a.dst.se, cscale(v[p][c], a.scale));
        } else {
            double2* q = buf + kk[p] * pl;
#pragma unroll
            for (int c = 0; c < R; ++c) q[spos(ob + c * Ns)] = v[p][c];
        }
    }
}

// In-place passes for the lengths of kInplacePlans: the radices (R3 = 0: three stages) and the
// butterflies per thread of each stage are compile-time, so that no stage's registers are
// reserved for another's radix. One shared buffer (the ping-pong kernel needs two at three or
// more stages) and 64 registers a thread keep four CTAs of 8 warps on each SM. Measured on
// B200, per pass against the ping-pong kernel: n = 512 1.17-1.23 ms (1.51-1.56), n = 384
// 529-560 us (623-650), n = 192 50-54 us (84-90), n = 96 12.6 us (18.7-19.0), n = 32 6.6 us
// (8.1-8.7); at n = 512, 8-vector tiles with two 16-warp CTAs per SM came within 2 %.
template <int SIGN, int R0, int R1, int R2, int R3, int P0, int P1, int P2, int P3>
struct InplaceTile {
    // CTAs per SM of the fused kernel (fft_fused_kernel): its item loop and both passes' arguments
    // do not fit the stand-alone kernel's 64 registers
    static constexpr int kMinBlocks = 2;
    // tile (bx, by) of a pass: vectors bx*kb .., tile index by
    static __device__ __forceinline__ void run(const FftPassArgs& a, int bx, int by, const double2* src, double2* dst,
                                               double2* smem);
};

template <int SIGN, int R0, int R1, int R2, int R3, int P0, int P1, int P2, int P3>
__device__ __forceinline__ void InplaceTile<SIGN, R0, R1, R2, R3, P0, P1, P2, P3>::run(const FftPassArgs& a, int bx, int by,
                                                                                    const double2* src, double2* dst,
                                                                                    double2* smem)
{
    const int v0 = bx * a.kb;
    const int nv = min(a.kb, a.nvec - v0);
    const long long src_base = (long long)v0 * a.src.sv + (long long)by * a.src.sb;
    const long long dst_base = (long long)v0 * a.dst.sv + (long long)by * a.dst.sb;
    if constexpr (R0 == R1 && R1 == R2 && R3 == 0 && P0 == P1 && P1 == P2) {
        // one radix throughout (n = 512): a loop over the runtime stage count, which compiles
        // to fewer spills at 64 registers than the unrolled stages
        for (int s = 0; s < a.nstages; ++s) {
            run_stage_inplace<SIGN, R0, P0>(a, s, src, dst, smem, nv, src_base, dst_base);
            if (s + 1 < a.nstages) __syncthreads();
        }
    } else {
        run_stage_inplace<SIGN, R0, P0>(a, 0, src, dst, smem, nv, src_base, dst_base);
        __syncthreads();
        run_stage_inplace<SIGN, R1, P1>(a, 1, src, dst, smem, nv, src_base, dst_base);
        if constexpr (R2 != 0) {
            __syncthreads();
            run_stage_inplace<SIGN, R2, P2>(a, 2, src, dst, smem, nv, src_base, dst_base);
        }
        if constexpr (R3 != 0) {
            __syncthreads();
            run_stage_inplace<SIGN, R3, P3>(a, 3, src, dst, smem, nv, src_base, dst_base);
        }
    }
}

template <int SIGN, int R0, int R1, int R2, int R3, int P0, int P1, int P2, int P3>
__global__ void __launch_bounds__(256, 4) fft_pass_inplace_kernel(const double2* src, double2* dst,
                                                                  const FftPassArgs a)
{
    extern __shared__ double2 smem[];
    if (a.srcs) {
        src = a.srcs[blockIdx.z];
        dst = a.dsts[blockIdx.z];
    }
    InplaceTile<SIGN, R0, R1, R2, R3, P0, P1, P2, P3>::run(a, blockIdx.x, blockIdx.y, src, dst, smem);
}


// Direct O(R^2) butterfly for any other radix (lengths with a prime factor above 5). The stage's
// outputs, not its butterflies, are spread over the threads: a large prime leaves few butterflies
// per tile (m = n / R of them per vector), while each of the R outputs of a butterfly is an
// independent R-term sum. A stage never writes the buffer it reads.
template <int SIGN>
__device__ void run_stage_generic(const FftPassArgs& a, int s, const double2* gsrc,
                                  double2* gdst, const double2* sin_, double2* sout, int nv,
                                  long long src_base, long long dst_base)
{
    const int n = a.n, R = a.radix[s];
    const int m = n / R;
    const int Ns = a.ns[s];
    const int step = n / (Ns * R);
    const int rstep = n / R;   // exp(SIGN 2 pi i rq/R) = twiddle[(rq mod R) * n/R]
    const bool first = (s == 0), last = (s == a.nstages - 1);
    const int pl = padded_len(n);
    const bool kk_fast = (first && a.src.se != 1) || (last && a.dst.se != 1);
    const int total = nv * m * R;
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        int j, kk, q;
        if (kk_fast) {   // consecutive threads: consecutive vectors (contiguous in HBM)
            kk = t % nv;
            const int u = t / nv;
            q = u % R;
            j = u / R;
        } else {
            q = t % R;
            const int u = t / R;
            j = u % m;
            kk = u / m;
        }
        const int k = j % Ns;
        const int ob = (j / Ns) * Ns * R + k;
        // input r carries the stage twiddle w_n^(r k step) and the DFT twiddle w_R^(r q) =
        // w_n^(r q rstep): one table entry w_n^(r cq mod n), its index advanced by cq per input
        const int cq = (int)(((long long)k * step + (long long)q * rstep) % n);
        double2 acc = first ? load_src(a, gsrc + src_base + (long long)kk * a.src.sv + (long long)j * a.src.se)
                            : sin_[kk * pl + spos(j)];
        int e = 0;
        for (int r = 1; r < R; ++r) {
            double2 x = first ? load_src(a, gsrc + src_base + (long long)kk * a.src.sv + (long long)(j + r * m) * a.src.se)
                              : sin_[kk * pl + spos(j + r * m)];
            e += cq;
            if (e >= n) e -= n;
            if (e) x = cmul(x, twiddle(a.twiddle, e, SIGN));
            acc = cadd(acc, x);
        }
        if (last) gdst[dst_base + (long long)kk * a.dst.sv + (long long)(ob + q * Ns) * a.dst.se] = cscale(acc, a.scale);
        else sout[kk * pl + spos(ob + q * Ns)] = acc;
    }
}

template <int SIGN>
struct PingPongTile {
    static constexpr int kMinBlocks = 2;   // as the stand-alone kernel
    static __device__ __forceinline__ void run(const FftPassArgs& a, int bx, int by, const double2* src, double2* dst,
                                               double2* smem);
};

template <int SIGN>
__device__ __forceinline__ void PingPongTile<SIGN>::run(const FftPassArgs& a, int bx, int by, const double2* src,
                                                        double2* dst, double2* smem)
{
    const int v0 = bx * a.kb;
    const int nv = min(a.kb, a.nvec - v0);
    const long long src_base = (long long)v0 * a.src.sv + (long long)by * a.src.sb;
    const long long dst_base = (long long)v0 * a.dst.sv + (long long)by * a.dst.sb;
    const int pl = padded_len(a.n);
    double2* buf[2] = {smem, smem + a.kb * pl};
    // In-place passes (src == dst) are safe: every CTA reads its whole tile in stage 0 and
    // writes it only in the last stage, after at least one __syncthreads (nstages >= 2), or in
    // the same thread's registers when there is a single stage.
    for (int s = 0; s < a.nstages; ++s) {
        const double2* sin_ = buf[(s + 1) & 1];
        double2* sout = buf[s & 1];
        switch (a.radix[s]) {
            case 16: run_stage_fixed<SIGN, 16>(a, s, src, dst, sin_, sout, nv, src_base, dst_base); break;
            case 8: run_stage_fixed<SIGN, 8>(a, s, src, dst, sin_, sout, nv, src_base, dst_base); break;
            case 4: run_stage_fixed<SIGN, 4>(a, s, src, dst, sin_, sout, nv, src_base, dst_base); break;
            case 2: run_stage_fixed<SIGN, 2>(a, s, src, dst, sin_, sout, nv, src_base, dst_base); break;
            case 1: run_stage_fixed<SIGN, 1>(a, s, src, dst, sin_, sout, nv, src_base, dst_base); break;
            case 3: run_stage_fixed<SIGN, 3>(a, s, src, dst, sin_, sout, nv, src_base, dst_base); break;
            case 5: run_stage_fixed<SIGN, 5>(a, s, src, dst, sin_, sout, nv, src_base, dst_base); break;
            default: run_stage_generic<SIGN>(a, s, src, dst, sin_, sout, nv, src_base, dst_base); break;
        }
        if (s + 1 < a.nstages) __syncthreads();
    }
}

template <int SIGN>
__global__ void __launch_bounds__(256, 2) fft_pass_kernel(const double2* src, double2* dst,
                                                       const FftPassArgs a)
{
    extern __shared__ double2 smem[];
    if (a.srcs) {
        src = a.srcs[blockIdx.z];
        dst = a.dsts[blockIdx.z];
    }
    PingPongTile<SIGN>::run(a, blockIdx.x, blockIdx.y, src, dst, smem);
}

// Both passes of one direction in one persistent launch. The layers (the vector index of both
// passes) are cut into chunks; CTAs take work items in order from a counter: the first pass's
// tiles of chunk 0, then for each chunk c >= 1 the first pass's tiles of chunk c followed by the
// second pass's tiles of chunk c - 1, then the second pass of the last chunk; transforms of a
// batch one after another. A second-pass tile of chunk c starts once all first-pass tiles of that
// chunk have finished (a counter per chunk), so it reads the first pass's output of the chunk
// while it is still in L2 and the workspace makes one HBM round trip instead of two. Every item
// that waits comes after the items it waits for, and every CTA is resident, so the waits end; a
// wait is bounded all the same (2 s), after which the tile runs anyway and the status word is set.
struct FusedArgs {
    FftPassArgs p[2];
    const double2* src[2];   // single transform: each pass's source and destination
    double2* dst[2];
    int cx[2];               // vector tiles of each pass per chunk (chunk / kb)
    int ny[2];               // tiles along the other index of each pass
    int nchunks;             // chunks per transform
    int per_z;               // items per transform
    int total;               // items of the launch
    long long sync_off;      // double2 offset of the counters in each transform's workspace
    double2* ws;             // single transform: its workspace
    int discard;             // drop the second pass's input lines from L2 once read (dead workspace)
};

// Counters of transform z: [0] next item and [1] status (transform 0 only), [2 + c] first-pass
// tiles of chunk c that have finished. The workspace is the second pass's source.
__device__ __forceinline__ int* fused_sync(const FusedArgs& f, int z)
{
    const double2* w = f.p[1].srcs ? f.p[1].srcs[z] : f.ws;
    return reinterpret_cast<int*>(const_cast<double2*>(w) + f.sync_off);
}

__global__ void fused_sync_clear(FusedArgs f, int words)
{
    int* w = fused_sync(f, blockIdx.x);
    for (int i = threadIdx.x; i < words; i += blockDim.x) w[i] = 0;
}

template <int SIGN, class Tile>
__global__ void __launch_bounds__(256, Tile::kMinBlocks) fft_fused_kernel(const __grid_constant__ FusedArgs f)
{
    extern __shared__ double2 smem[];
    __shared__ int s_item;
    int* ctl = fused_sync(f, 0);
    const int T1 = f.cx[0] * f.ny[0], T2 = f.cx[1] * f.ny[1];
    if (threadIdx.x == 0) s_item = atomicAdd(ctl, 1);
    __syncthreads();
    for (;;) {
        const int item = s_item;
        __syncthreads();
        if (item >= f.total) break;
        // the next item is claimed now; thread 0 waits for the counter's answer only after this tile
        int next = 0;
        if (threadIdx.x == 0) next = atomicAdd(ctl, 1);
        const int z = item / f.per_z;
        int j = item - z * f.per_z;
        int pass, c, t;
        if (j < T1) {
            pass = 0;
            c = 0;
            t = j;
        } else {
            j -= T1;
            const int step = 1 + j / (T1 + T2);
            const int r = j - (step - 1) * (T1 + T2);
            if (step < f.nchunks && r < T1) {
                pass = 0;
                c = step;
                t = r;
            } else {
                pass = 1;
                c = step - 1;
                t = step < f.nchunks ? r - T1 : r;
            }
        }
        int* done = fused_sync(f, z) + 2;
        if (pass == 1) {
            if (threadIdx.x == 0) {
                const volatile int* d = done + c;   // polled; the fence below orders what follows
                if (*d < T1) {
                    uint64_t t0;
                    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t0));
                    for (;;) {
                        if (*d >= T1) break;
                        uint64_t t1;
                        asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t1));
                        if (t1 - t0 > 2000000000ull) {
                            atomicExch(ctl + 1, 1);
                            break;
                        }
                        __nanosleep(256);
                    }
                }
                __threadfence();
            }
            __syncthreads();
        }
        // one call site; the arguments are a __grid_constant__ parameter, so indexing them by the
        // pass reads the parameter space instead of copying it to local memory
        const FftPassArgs& a = f.p[pass];
        const double2* src = a.srcs ? a.srcs[z] : f.src[pass];
        double2* dst = a.dsts ? a.dsts[z] : f.dst[pass];
        const int bx = c * f.cx[pass] + t % f.cx[pass], by = t / f.cx[pass];
        Tile::run(a, bx, by, src, dst, smem);
        if (pass == 0) {
            // the CTA's stores are ordered before the barrier; one release by thread 0 publishes
            // them all (the tile counts as done only after every thread's stores)
            __syncthreads();
            if (threadIdx.x == 0) {
                int* d = done + c;
                asm volatile("red.release.gpu.global.add.s32 [%0], 1;" ::"l"(d) : "memory");
            }
        } else if (f.discard) {
            // the second pass of the inverse read its input (the workspace, dead from here on):
            // one 128-byte line of kb consecutive layers per element; drop them from L2 so that
            // the first pass's writes are not written back to HBM
            __syncthreads();
            const FftPassArgs& q = f.p[1];
            for (int e = threadIdx.x; e < q.n; e += blockDim.x) {
                const double2* line = src + (long long)bx * q.kb * q.src.sv + (long long)by * q.src.sb + (long long)e * q.src.se;
                if ((reinterpret_cast<uintptr_t>(line) & 127) == 0)   // whole lines only
                    asm volatile("discard.global.L2 [%0], 128;" ::"l"(line) : "memory");
            }
        }
        if (threadIdx.x == 0) s_item = next;
        __syncthreads();
    }
}

// Bluestein pass: kBluesteinVec vectors per CTA, each loaded, multiplied by its chirp and
// zero-padded to M in shared memory, transformed (radix-2 stages, two per pass over shared memory;
// decimation in frequency: natural order in, bit-reversed out), multiplied by the bit-reversed
// transform of the chirp kernel (1/M
// included), transformed back (decimation in time: bit-reversed in, natural out), multiplied by
// the chirp and stored. The same HBM access pattern as a pass kernel's first and last stages.
constexpr int kBluesteinVec = 4;

template <int SIGN>
__global__ void __launch_bounds__(256) fft_bluestein_kernel(const double2* src, double2* dst, const FftPassArgs a, int logM)
{
    const int M = 1 << logM;
    extern __shared__ double2 smem[];   // [kBluesteinVec][M]
    if (a.srcs) {
        src = a.srcs[blockIdx.z];
        dst = a.dsts[blockIdx.z];
    }
    const int n = a.n, half = M >> 1;
    const double2* wtab = a.bluestein;                                 // exp(-pi i e^2 / n)
    const double2* fh = a.bluestein + n + (SIGN < 0 ? 0 : M);          // bit-reversed, 1/M included
    const double2* tw = a.bluestein + n + 2 * M;                       // exp(-2 pi i t / M), t < M/2
    const int v0 = blockIdx.x * kBluesteinVec;
    const int nv = min(kBluesteinVec, a.nvec - v0);
    const long long sbase = (long long)v0 * a.src.sv + (long long)blockIdx.y * a.src.sb;
    const long long dbase = (long long)v0 * a.dst.sv + (long long)blockIdx.y * a.dst.sb;
    const bool vfast_in = a.src.se != 1, vfast_out = a.dst.se != 1;   // vectors contiguous in HBM
    for (int t = threadIdx.x; t < kBluesteinVec * M; t += blockDim.x) {
        int v, e;
        if (vfast_in) {
            v = t % kBluesteinVec;
            e = t / kBluesteinVec;
        } else {
            e = t & (M - 1);
            v = t >> logM;
        }
        double2 x = make_double2(0.0, 0.0);
        if (v < nv && e < n) {
            double2 w = wtab[e];
            if (SIGN > 0) w.y = -w.y;
            x = cmul(load_src(a, src + sbase + (long long)v * a.src.sv + (long long)e * a.src.se), w);
        }
        smem[v * M + e] = x;
    }
    __syncthreads();
    // forward, decimation in frequency: two radix-2 stages (spans 2^ls and 2^(ls-1)) per pass over
    // shared memory, the same arithmetic as one stage at a time
    int ls = logM - 1;
    for (; ls >= 1; ls -= 2) {
        const int sp = 1 << ls, h = sp >> 1, tA = logM - 1 - ls, tB = logM - ls;
        for (int b = threadIdx.x; b < kBluesteinVec * (M >> 2); b += blockDim.x) {
            const int i = b & (h - 1);
            const int p0 = ((b >> (ls - 1)) << (ls + 1)) + i, p1 = p0 + h, p2 = p0 + sp, p3 = p2 + h;
            const double2 x0 = smem[p0], x1 = smem[p1], x2 = smem[p2], x3 = smem[p3];
            const double2 a0 = cadd(x0, x2), a2 = cmul(csub(x0, x2), tw[i << tA]);
            const double2 a1 = cadd(x1, x3), a3 = cmul(csub(x1, x3), tw[(i + h) << tA]);
            const double2 wb = tw[i << tB];
            smem[p0] = cadd(a0, a1);
            smem[p1] = cmul(csub(a0, a1), wb);
            smem[p2] = cadd(a2, a3);
            smem[p3] = cmul(csub(a2, a3), wb);
        }
        __syncthreads();
    }
    if (ls == 0) {   // an odd number of stages: the last one alone (span 1, twiddle 1)
        for (int b = threadIdx.x; b < kBluesteinVec * half; b += blockDim.x) {
            const int p = b << 1;
            const double2 u = smem[p], x = smem[p + 1];
            smem[p] = cadd(u, x);
            smem[p + 1] = csub(u, x);
        }
        __syncthreads();
    }
    for (int t = threadIdx.x; t < kBluesteinVec * M; t += blockDim.x) smem[t] = cmul(smem[t], fh[t & (M - 1)]);
    __syncthreads();
    // inverse, decimation in time: spans 2^ls and 2^(ls+1) per pass (conjugate twiddles)
    ls = 0;
    for (; ls + 1 < logM; ls += 2) {
        const int sp = 1 << ls, t1 = logM - 1 - ls, t2 = logM - 2 - ls;
        for (int b = threadIdx.x; b < kBluesteinVec * (M >> 2); b += blockDim.x) {
            const int i = b & (sp - 1);
            const int p0 = ((b >> ls) << (ls + 2)) + i, p1 = p0 + sp, p2 = p1 + sp, p3 = p2 + sp;
            double2 w = tw[i << t1];
            w.y = -w.y;
            const double2 x0 = smem[p0], x1 = cmul(smem[p1], w), x2 = smem[p2], x3 = cmul(smem[p3], w);
            const double2 a0 = cadd(x0, x1), a1 = csub(x0, x1), a2 = cadd(x2, x3), a3 = csub(x2, x3);
            double2 w0 = tw[i << t2], w1 = tw[(i + sp) << t2];
            w0.y = -w0.y;
            w1.y = -w1.y;
            const double2 b2 = cmul(a2, w0), b3 = cmul(a3, w1);
            smem[p0] = cadd(a0, b2);
            smem[p2] = csub(a0, b2);
            smem[p1] = cadd(a1, b3);
            smem[p3] = csub(a1, b3);
        }
        __syncthreads();
    }
    if (ls == logM - 1) {   // the last stage alone (span M/2)
        for (int b = threadIdx.x; b < kBluesteinVec * half; b += blockDim.x) {
            const int i = b & (half - 1);
            const int p = ((b >> (logM - 1)) << logM) + i, q = p + half;
            double2 w = tw[i];
            w.y = -w.y;
            const double2 u = smem[p], x = cmul(smem[q], w);
            smem[p] = cadd(u, x);
            smem[q] = csub(u, x);
        }
        __syncthreads();
    }
    for (int t = threadIdx.x; t < kBluesteinVec * n; t += blockDim.x) {
        int v, k;
        if (vfast_out) {
            v = t % kBluesteinVec;
            k = t / kBluesteinVec;
        } else {
            k = t % n;
            v = t / n;
        }
        if (v >= nv) continue;
        double2 w = wtab[k];
        if (SIGN > 0) w.y = -w.y;
        dst[dbase + (long long)v * a.dst.sv + (long long)k * a.dst.se] = cscale(cmul(smem[v * M + k], w), a.scale);
    }
}

// Lengths that run the in-place kernel: tile vectors and radices (0 ends a shorter plan). 384 is
// planned 8.4.4.3 rather than 16.8.3: radix 16 does not fit the kernel's 64 registers. Measured
// and left on the ping-pong kernel: 256 as 8.8.4 (125 against 96 us per pass: its 16.16 plan
// has one exchange and one buffer), 128 as 8.4.4 (23 against 19 us), 64 as 8.8 (equal).
struct InplacePlan {
    int n, kb, nstages;
    int radix[4];
};
constexpr InplacePlan kInplacePlans[] = {
    {512, 4, 3, {8, 8, 8, 0}},
    {384, 4, 4, {8, 4, 4, 3}},
    {192, 8, 3, {8, 8, 3, 0}},
    {96, 8, 3, {8, 4, 3, 0}},
    {32, 8, 2, {8, 4, 0, 0}},
};

const InplacePlan* inplace_plan_for(int n)
{
    for (const InplacePlan& p : kInplacePlans)
        if (p.n == n) return &p;
    return nullptr;
}

// The in-place plan that a pass's arguments follow, if any (the caller may have chosen other
// tiles or radices; those run the ping-pong kernel).
const InplacePlan* inplace_plan_of(const FftPassArgs& a)
{
    const InplacePlan* p = inplace_plan_for(a.n);
    if (!p || a.kb != p->kb || a.nstages != p->nstages) return nullptr;
    for (int s = 0; s < p->nstages; ++s)
        if (a.radix[s] != p->radix[s]) return nullptr;
    return p;
}

}  // namespace

int fft_plan_radices(int n, int* radix, int* ns)
{
    if (n < 1) return 0;
    if (const InplacePlan* ip = inplace_plan_for(n)) {
        int nsv = 1;
        for (int i = 0; i < ip->nstages; ++i) {
            radix[i] = ip->radix[i];
            ns[i] = nsv;
            nsv *= ip->radix[i];
        }
        return ip->nstages;
    }
    int r[64];
    int cnt = 0, rem = n;
    int p2 = 0;
    while (rem % 2 == 0) {
        rem /= 2;
        ++p2;
    }
    // power-of-two part: as few stages as radix 16 allows, bits spread evenly (8.8.8, 16.8)
    if (p2 > 0) {
        const int st = (p2 + 3) / 4;
        for (int i = 0; i < st; ++i) {
            const int bits = p2 / st + (i < p2 % st ? 1 : 0);
            r[cnt++] = 1 << bits;
        }
    }
    while (rem % 3 == 0) { r[cnt++] = 3; rem /= 3; }
    while (rem % 5 == 0) { r[cnt++] = 5; rem /= 5; }
    for (int p = 7; rem > 1; p += 2) {
        while (rem % p == 0) { r[cnt++] = p; rem /= p; }
    }
    if (cnt == 0) r[cnt++] = 1;
    // A lone direct (O(R^2)) stage would read and write the same HBM vector when the pass
    // is in place; a leading radix-1 stage (a plain copy into shared memory) separates them.
    const bool direct = !(r[0] == 1 || r[0] == 2 || r[0] == 3 || r[0] == 4 || r[0] == 5 || r[0] == 8 || r[0] == 16);
    if (cnt == 1 && direct) {
        r[1] = r[0];
        r[0] = 1;
        cnt = 2;
    }
    if (cnt > kFftMaxStages) return 0;
    int nsv = 1;
    for (int i = 0; i < cnt; ++i) {
        radix[i] = r[i];
        ns[i] = nsv;
        nsv *= r[i];
    }
    return cnt;
}

bool fft_needs_bluestein(int n)
{
    if (n < 2 || n > 512) return false;
    int rem = n, big = 1;
    for (int p = 2; p * p <= rem; ++p)
        while (rem % p == 0) {
            big = p;
            rem /= p;
        }
    if (rem > 1) big = rem > big ? rem : big;
    return big > 16;
}

int fft_bluestein_m(int n)
{
    int m = 1;
    while (m < 2 * n - 1) m <<= 1;
    return m;
}

size_t fft_bluestein_elems(int n)
{
    const int M = fft_bluestein_m(n);
    return (size_t)n + 2 * (size_t)M + (size_t)(M / 2);
}

void fft_bluestein_fill(int n, double2* out)
{
    typedef long double ld;
    const ld pi = 3.14159265358979323846264338327950288L;
    const int M = fft_bluestein_m(n);
    int bits = 0;
    while ((1 << bits) < M) ++bits;
    // w_e = exp(-pi i e^2 / n), the exponent reduced mod 2n first
    std::vector<ld> wr(n), wi(n);
    for (int e = 0; e < n; ++e) {
        const long long r = ((long long)e * e) % (2ll * n);
        const ld ang = pi * (ld)r / (ld)n;
        wr[e] = cosl(ang);
        wi[e] = -sinl(ang);
        out[e] = make_double2((double)wr[e], (double)wi[e]);
    }
    std::vector<ld> cr(M), ci(M);   // exp(-2 pi i t / M)
    for (int t = 0; t < M; ++t) {
        cr[t] = cosl(2 * pi * (ld)t / (ld)M);
        ci[t] = -sinl(2 * pi * (ld)t / (ld)M);
    }
    for (int sg = 0; sg < 2; ++sg) {
        // kernel h_d = conj(w(sign)_d), w(-1) = w, w(+1) = conj(w): h = conj(w) for sign -1, w for +1;
        // placed at d and M - d
        std::vector<ld> hr(M, 0), hi(M, 0);
        for (int d = 0; d < n; ++d) {
            const ld re = wr[d], im = sg == 0 ? -wi[d] : wi[d];
            hr[d] = re;
            hi[d] = im;
            if (d > 0) {
                hr[M - d] = re;
                hi[M - d] = im;
            }
        }
        for (int k = 0; k < M; ++k) {   // DFT (exp(-2 pi i jk / M)) / M, stored bit-reversed
            ld sr = 0, si = 0;
            for (int j = 0; j < M; ++j) {
                const int t = (int)(((long long)j * k) & (M - 1));
                sr += hr[j] * cr[t] - hi[j] * ci[t];
                si += hr[j] * ci[t] + hi[j] * cr[t];
            }
            int br = 0;
            for (int b = 0; b < bits; ++b)
                if (k & (1 << b)) br |= 1 << (bits - 1 - b);
            out[n + sg * M + br] = make_double2((double)(sr / M), (double)(si / M));
        }
    }
    for (int t = 0; t < M / 2; ++t) out[n + 2 * M + t] = make_double2((double)cr[t], (double)ci[t]);
}

int fft_tile_vectors(int n)
{
    if (const InplacePlan* ip = inplace_plan_for(n)) return ip->kb;
    const size_t two_buffers = 2 * (size_t)8 * padded_len(n) * sizeof(double2);
    return two_buffers > (size_t)110 * 1024 ? 4 : 8;
}

size_t fft_pass_smem_bytes(const FftPassArgs& a)
{
    const int buffers = inplace_plan_of(a) ? 1 : (a.nstages >= 3 ? 2 : (a.nstages == 2 ? 1 : 0));
    return (size_t)buffers * a.kb * padded_len(a.n) * sizeof(double2);
}

cudaError_t fft_pass_launch(const double2* src, double2* dst, const FftPassArgs& a, int ntiles, int sign,
                            cudaStream_t stream, int nz)
{
    if (a.bluestein && fft_needs_bluestein(a.n)) {
        const int M = fft_bluestein_m(a.n);
        int logM = 0;
        while ((1 << logM) < M) ++logM;
        const size_t sm = (size_t)kBluesteinVec * M * sizeof(double2);
        dim3 grid((a.nvec + kBluesteinVec - 1) / kBluesteinVec, ntiles, nz);
        auto goB = [&](auto kern) {
            if (sm > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            kern<<<grid, 256, sm, stream>>>(src, dst, a, logM);
        };
        sign < 0 ? goB(fft_bluestein_kernel<-1>) : goB(fft_bluestein_kernel<1>);
        return cudaGetLastError();
    }
    const InplacePlan* ip = inplace_plan_of(a);
    // one butterfly per thread in the widest stage, up to 256 threads (the in-place kernels run
    // 256 threads, each with the butterflies per stage their plan gives)
    int widest = 1;
    for (int s = 0; s < a.nstages; ++s) widest = a.n / a.radix[s] > widest ? a.n / a.radix[s] : widest;
    int nthreads = ((a.kb * widest + 31) / 32) * 32;
    if (ip || nthreads > 256) nthreads = 256;
    dim3 grid((a.nvec + a.kb - 1) / a.kb, ntiles, nz);
    const size_t smem = fft_pass_smem_bytes(a);
    FftPassArgs as = a;
    as.stream_out = 1;   // a stand-alone pass: the next one reads its output from HBM
    auto go = [&](auto kern) {
        if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<grid, nthreads, smem, stream>>>(src, dst, as);
    };
    if (ip) {
        // butterflies per thread per stage: ceil(kb * n / R / 256)
        switch (ip->n) {
            case 512: sign < 0 ? go(fft_pass_inplace_kernel<-1, 8, 8, 8, 0, 1, 1, 1, 1>)
                               : go(fft_pass_inplace_kernel<1, 8, 8, 8, 0, 1, 1, 1, 1>); break;
            case 384: sign < 0 ? go(fft_pass_inplace_kernel<-1, 8, 4, 4, 3, 1, 2, 2, 2>)
                               : go(fft_pass_inplace_kernel<1, 8, 4, 4, 3, 1, 2, 2, 2>); break;
            case 192: sign < 0 ? go(fft_pass_inplace_kernel<-1, 8, 8, 3, 0, 1, 1, 2, 1>)
                               : go(fft_pass_inplace_kernel<1, 8, 8, 3, 0, 1, 1, 2, 1>); break;
            case 32: sign < 0 ? go(fft_pass_inplace_kernel<-1, 8, 4, 0, 0, 1, 1, 1, 1>)
                              : go(fft_pass_inplace_kernel<1, 8, 4, 0, 0, 1, 1, 1, 1>); break;
            case 96: sign < 0 ? go(fft_pass_inplace_kernel<-1, 8, 4, 3, 0, 1, 1, 1, 1>)
                              : go(fft_pass_inplace_kernel<1, 8, 4, 3, 0, 1, 1, 1, 1>); break;
            default: return cudaErrorInvalidValue;   // a table entry without a kernel
        }
    } else {
        // the ping-pong kernel indexes two buffers; with a single buffer the second is never used
        sign < 0 ? go(fft_pass_kernel<-1>) : go(fft_pass_kernel<1>);
    }
    return cudaGetLastError();
}

// Fused-pass choice per transform length (index n <= 1024; default off), set by the autotuner.
constexpr int kFusedMaxN = 1024;
signed char g_fft_fused[kFusedMaxN + 1] = {};   // 0 default (on), 1 on, -1 off
bool g_fft_fused_all = false;
bool fft_fused_enabled(int n)
{
    if (n >= 0 && n <= kFusedMaxN && g_fft_fused[n]) return g_fft_fused[n] > 0;
    return g_fft_fused_all;
}
void fft_set_fused(int n, int on)
{
    if (n <= 0) {
        g_fft_fused_all = on != 0;
        for (int i = 0; i <= kFusedMaxN; ++i) g_fft_fused[i] = 0;
    } else if (n <= kFusedMaxN) {
        g_fft_fused[n] = on ? 1 : -1;
    }
}

// Layers per chunk of the fused passes: about 16 MB of workspace per chunk, a multiple of both
// passes' tile vectors that divides the layer count; 0 when the passes cannot be fused.
int fft_fused_chunk(const FftPassArgs& p0, const FftPassArgs& p1)
{
    if ((p0.bluestein || p1.bluestein) && fft_needs_bluestein(p0.n)) return 0;   // the Bluestein pass has no fused form
    if (p0.n != p1.n || p0.nvec != p1.nvec || p0.kb != p1.kb || p0.nstages != p1.nstages || p0.nstages == 0) return 0;
    for (int st = 0; st < p0.nstages; ++st)
        if (p0.radix[st] != p1.radix[st]) return 0;
    const int nvec = p0.nvec, kb = p0.kb;
    const long long layer_bytes = (long long)p0.n * p0.n * (long long)sizeof(double2);
    int want = (int)((16ll << 20) / (layer_bytes > 0 ? layer_bytes : 1));
    if (want < kb) want = kb;
    int best = 0;
    for (int c = kb; c <= nvec; c += kb)
        if (nvec % c == 0 && c <= want) best = c;
    if (best == 0 && nvec % kb == 0) best = kb;
    if (best == 0 || 2 + nvec / best > kFftSyncBytes / (int)sizeof(int)) return 0;
    return best;
}

cudaError_t fft_fused_launch(int sign, const FftPassArgs& p0, const FftPassArgs& p1, int ntiles0, int ntiles1, int nz,
                             const double2* src0, double2* dst0, const double2* src1, double2* dst1, double2* ws,
                             long long sync_off, cudaStream_t stream)
{
    const int chunk = fft_fused_chunk(p0, p1);
    if (chunk == 0) return cudaErrorInvalidValue;
    if (nz > 1 && !(p0.srcs && p0.dsts && p1.srcs && p1.dsts)) return cudaErrorInvalidValue;
    FusedArgs f;
    memset(&f, 0, sizeof(f));
    f.p[0] = p0;
    f.p[1] = p1;
    f.p[1].coherent = 1;   // reads what the first pass's CTAs of this launch wrote
    f.src[0] = src0;
    f.dst[0] = dst0;
    f.src[1] = src1;
    f.dst[1] = dst1;
    f.cx[0] = f.cx[1] = chunk / p0.kb;
    f.ny[0] = ntiles0;
    f.ny[1] = ntiles1;
    f.nchunks = p0.nvec / chunk;
    f.per_z = f.nchunks * (f.cx[0] * f.ny[0] + f.cx[1] * f.ny[1]);
    f.total = f.per_z * nz;
    f.sync_off = sync_off;
    f.ws = ws;
    // inverse (I2 in place, then I1 out of the workspace): the workspace is dead once I1 has read
    // it; its lines can be dropped when one tile's kb layers fill whole 128-byte lines
    f.discard = (sign > 0 && p1.src.sv == 1 && p1.kb * (int)sizeof(double2) == 128 && p1.dst.sv != 1) ? 1 : 0;
    fused_sync_clear<<<nz, 128, 0, stream>>>(f, 2 + f.nchunks);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const InplacePlan* ip = inplace_plan_of(p0);
    int widest = 1;
    for (int st = 0; st < p0.nstages; ++st) widest = p0.n / p0.radix[st] > widest ? p0.n / p0.radix[st] : widest;
    int nthreads = ((p0.kb * widest + 31) / 32) * 32;
    if (ip || nthreads > 256) nthreads = 256;
    const size_t smem = fft_pass_smem_bytes(p0);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    auto go = [&](auto kern) -> cudaError_t {
        if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        int per = 1;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, nthreads, smem) != cudaSuccess || per < 1) per = 1;
        const int blocks = std::min(sms * per, f.total);
        kern<<<blocks, nthreads, smem, stream>>>(f);
        return cudaGetLastError();
    };
    if (ip) {
        switch (ip->n) {
            case 512: return sign < 0 ? go(fft_fused_kernel<-1, InplaceTile<-1, 8, 8, 8, 0, 1, 1, 1, 1>>)
                                      : go(fft_fused_kernel<1, InplaceTile<1, 8, 8, 8, 0, 1, 1, 1, 1>>);
            case 384: return sign < 0 ? go(fft_fused_kernel<-1, InplaceTile<-1, 8, 4, 4, 3, 1, 2, 2, 2>>)
                                      : go(fft_fused_kernel<1, InplaceTile<1, 8, 4, 4, 3, 1, 2, 2, 2>>);
            case 192: return sign < 0 ? go(fft_fused_kernel<-1, InplaceTile<-1, 8, 8, 3, 0, 1, 1, 2, 1>>)
                                      : go(fft_fused_kernel<1, InplaceTile<1, 8, 8, 3, 0, 1, 1, 2, 1>>);
            case 32: return sign < 0 ? go(fft_fused_kernel<-1, InplaceTile<-1, 8, 4, 0, 0, 1, 1, 1, 1>>)
                                     : go(fft_fused_kernel<1, InplaceTile<1, 8, 4, 0, 0, 1, 1, 1, 1>>);
            case 96: return sign < 0 ? go(fft_fused_kernel<-1, InplaceTile<-1, 8, 4, 3, 0, 1, 1, 1, 1>>)
                                     : go(fft_fused_kernel<1, InplaceTile<1, 8, 4, 3, 0, 1, 1, 1, 1>>);
            default: return cudaErrorInvalidValue;
        }
    }
    return sign < 0 ? go(fft_fused_kernel<-1, PingPongTile<-1>>) : go(fft_fused_kernel<1, PingPongTile<1>>);
}

}  // namespace pfsoft_dev
