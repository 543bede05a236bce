// One SO(3) transform sharded over several GPUs (C ABI: pfsoft_shard_*).
//
// Rank r of P owns a slab of beta layers (the FFT passes) and a set of order classes (the DWT);
// shard.hpp builds the plan and the exchange's copy runs. The steps, each on the caller's stream:
//   DSOFT   fft_forward (slab grid -> slab spectrum)
//           exchange: scatter (direct stores into every rank's spectrum: peer pointers over
//                     NVLink), or pack -> the caller's all-to-all -> unpack
//           dwt_forward (this rank's classes; zero elsewhere, so the sum over ranks is the result)
//   iDSOFT  dwt_inverse (this rank's classes' bins of its spectrum)
//           exchange in the inverse direction (into every rank's slab spectrum)
//           fft_inverse (Nyquist bins zeroed, alpha then gamma inverse DFT -> slab grid)
// The caller orders the ranks around the exchange: after a scatter, every rank's stores must be
// complete and visible before any rank's next step reads its buffer (a barrier on the streams).
// The FFT and DWT kernels are the single-transform ones, run on the slab (strided passes) and on
// a class subset (DwtArgs::classes).

#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/pfsoft_b200.h"
#include "common.cuh"
#include "dwt.cuh"
#include "fft.cuh"
#include "shard.hpp"

using namespace pfsoft_dev;
using pfsoft_shard::Run;

namespace pfsoft_dev {
int tables_for(int B, cudaStream_t s, BandTables* out);   // api.cu: cached tables of a bandwidth
}

namespace {

struct DstTable {
    double2* p[pfsoft_shard::kMaxRanks];
};

// Groups of gw lanes (a power of two <= 32) copy one run each: gw consecutive complex values per
// step, so a run of nk values moves as nk * 16 contiguous bytes on both sides.
__global__ void __launch_bounds__(256) shard_copy_kernel(const Run* __restrict__ runs, long long n, int gw,
                                                         const double2* __restrict__ src, const DstTable dst)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long stride = (long long)gridDim.x * blockDim.x / gw;
    const int sub = (int)(t % gw);
    for (long long i = t / gw; i < n; i += stride) {
        const Run r = runs[i];
        const double2* s = src + r.src_off;
        double2* d = dst.p[r.slot] + r.dst_off;
        for (int e = sub; e < r.len; e += gw) d[e] = __ldg(s + e);
    }
}

// Zero the Nyquist bins (row == B or col == B) of a slab spectrum [N][N][nk].
__global__ void zero_nyquist_slab_kernel(double2* X, int B, int nk)
{
    const int N = 2 * B;
    const long long total = (long long)(2 * N - 1) * nk;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const long long v = i / nk;
        const int k = (int)(i - v * nk);
        int row, col;
        if (v < N) {
            row = B;
            col = (int)v;
        } else {
            col = B;
            row = (int)(v - N);
            if (row >= B) ++row;   // (B, B) is covered above
        }
        X[((size_t)row * N + col) * nk + k] = make_double2(0.0, 0.0);
    }
}

int fail(int status, const std::string& msg)
{
    set_last_error(msg.c_str());
    return status;
}

int cuda_fail(cudaError_t e, const char* what)
{
    return fail(PFSOFT_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

FftPassArgs slab_pass(int n, int nvec, const BandTables& t, FftStrides src, FftStrides dst, double scale)
{
    FftPassArgs a;
    memset(&a, 0, sizeof(a));
    a.n = n;
    a.nvec = nvec;
    a.kb = fft_tile_vectors(n);
    a.nstages = fft_plan_radices(n, a.radix, a.ns);
    a.src = src;
    a.dst = dst;
    a.scale = scale;
    a.twiddle = t.twiddle;
    a.bluestein = t.bluestein;
    return a;
}

}  // namespace

struct pfsoft_shard_plan {
    pfsoft_shard::Plan p;
    std::mutex mu;
    bool built[pfsoft_shard::RUN_KINDS] = {};
    std::vector<Run> runs[pfsoft_shard::RUN_KINDS];
    int gw[pfsoft_shard::RUN_KINDS] = {};
    int device = -1;
    Run* d_runs[pfsoft_shard::RUN_KINDS] = {};
    int* d_classes = nullptr;

    const std::vector<Run>& host_runs(int kind)
    {
        if (!built[kind]) {
            runs[kind] = pfsoft_shard::make_runs(p, (pfsoft_shard::RunKind)kind);
            int mx = 1;
            for (const Run& r : runs[kind]) mx = r.len > mx ? r.len : mx;
            int g = 1;
            while (g < mx && g < 32) g <<= 1;
            gw[kind] = g;
            built[kind] = true;
        }
        return runs[kind];
    }

    // Device copies are made on first use, on the device current at that time.
    int bind_device()
    {
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return cuda_fail(e, "shard plan: no device");
        if (device < 0) {
            device = dev;
            const std::vector<int>& cls = p.classes[p.rank];
            if (!cls.empty()) {
                e = cudaMalloc(&d_classes, cls.size() * sizeof(int));
                if (e != cudaSuccess) return fail(PFSOFT_ENOMEM, std::string("shard plan: ") + cudaGetErrorString(e));
                e = cudaMemcpy(d_classes, cls.data(), cls.size() * sizeof(int), cudaMemcpyHostToDevice);
                if (e != cudaSuccess) return cuda_fail(e, "shard plan: class list upload");
            }
        } else if (device != dev) {
            return fail(PFSOFT_EINVAL, "shard plan used on another device than its first use");
        }
        return PFSOFT_OK;
    }

    int device_runs(int kind, const Run** out, long long* n)
    {
        const std::vector<Run>& h = host_runs(kind);
        if (!d_runs[kind] && !h.empty()) {
            cudaError_t e = cudaMalloc(&d_runs[kind], h.size() * sizeof(Run));
            if (e != cudaSuccess) return fail(PFSOFT_ENOMEM, std::string("shard plan: ") + cudaGetErrorString(e));
            e = cudaMemcpy(d_runs[kind], h.data(), h.size() * sizeof(Run), cudaMemcpyHostToDevice);
            if (e != cudaSuccess) return cuda_fail(e, "shard plan: run upload");
        }
        *out = d_runs[kind];
        *n = (long long)h.size();
        return PFSOFT_OK;
    }

    // frees the device tables on the device they were made on, then restores the caller's device
    ~pfsoft_shard_plan()
    {
        if (device < 0) return;
        int cur = -1;
        const bool switched = cudaGetDevice(&cur) == cudaSuccess && cur != device && cudaSetDevice(device) == cudaSuccess;
        for (Run* r : d_runs)
            if (r) cudaFree(r);
        if (d_classes) cudaFree(d_classes);
        if (switched) cudaSetDevice(cur);
    }
};

namespace {

int kind_of(int direction, int step)   // step 0 scatter, 1 pack, 2 unpack
{
    return (direction == PFSOFT_SHARD_FORWARD ? pfsoft_shard::FWD_SCATTER : pfsoft_shard::INV_SCATTER) + step;
}

int run_copy(pfsoft_shard_plan* plan, int kind, const double* src, const DstTable& dst, bool single, cudaStream_t s)
{
    const Run* d = nullptr;
    long long n = 0;
    int rc;
    try {
        rc = plan->device_runs(kind, &d, &n);
    } catch (const std::bad_alloc&) {
        return fail(PFSOFT_ENOMEM, "shard plan: run list allocation");
    }
    if (rc) return rc;
    if (n == 0) return PFSOFT_OK;
    if (!src) return fail(PFSOFT_EINVAL, "null exchange source buffer");
    if (single && !dst.p[0]) return fail(PFSOFT_EINVAL, "null exchange destination buffer");
    const int gw = plan->gw[kind];
    const long long groups_per_block = 256 / gw;
    long long blocks = (n + groups_per_block - 1) / groups_per_block;
    if (blocks > 148 * 16) blocks = 148 * 16;
    shard_copy_kernel<<<(unsigned)blocks, 256, 0, s>>>(d, n, gw, reinterpret_cast<const double2*>(src), dst);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PFSOFT_OK : cuda_fail(e, "shard exchange launch");
}

int begin(pfsoft_shard_plan* plan, std::unique_lock<std::mutex>& lk)
{
    set_last_error("");
    if (!plan) return fail(PFSOFT_EINVAL, "null shard plan");
    lk = std::unique_lock<std::mutex>(plan->mu);
    return plan->bind_device();
}

}  // namespace

extern "C" {

int pfsoft_shard_create(int B, int nranks, int rank, pfsoft_shard_plan** out)
{
    set_last_error("");
    if (!out) return fail(PFSOFT_EINVAL, "null output handle");
    *out = nullptr;
    if (B < 1 || B > 512) return fail(PFSOFT_EINVAL, "bandwidth must be in [1, 512]");
    if (nranks < 1 || nranks > pfsoft_shard::kMaxRanks) return fail(PFSOFT_EINVAL, "nranks must be in [1, 64]");
    if (rank < 0 || rank >= nranks) return fail(PFSOFT_EINVAL, "rank must be in [0, nranks)");
    pfsoft_shard_plan* p = new (std::nothrow) pfsoft_shard_plan;
    if (!p) return fail(PFSOFT_ENOMEM, "shard plan allocation");
    try {
        p->p = pfsoft_shard::make_plan(B, nranks, rank);
    } catch (const std::bad_alloc&) {
        delete p;
        return fail(PFSOFT_ENOMEM, "shard plan allocation");
    }
    *out = p;
    return PFSOFT_OK;
}

void pfsoft_shard_destroy(pfsoft_shard_plan* plan) { delete plan; }

int pfsoft_shard_layers(const pfsoft_shard_plan* plan, int rank, int* first, int* count)
{
    if (!plan || rank < 0 || rank >= plan->p.P) return fail(PFSOFT_EINVAL, "bad plan or rank");
    if (first) *first = plan->p.k0[rank];
    if (count) *count = plan->p.nk[rank];
    return PFSOFT_OK;
}

int pfsoft_shard_classes(const pfsoft_shard_plan* plan, int rank, int* out, int capacity)
{
    if (!plan || rank < 0 || rank >= plan->p.P) return -1;
    const std::vector<int>& c = plan->p.classes[rank];
    if (out)
        for (int i = 0; i < (int)c.size() && i < capacity; ++i) out[i] = c[i];
    return (int)c.size();
}

long long pfsoft_shard_bins(const pfsoft_shard_plan* plan, int rank, int* out, long long capacity)
{
    if (!plan || rank < 0 || rank >= plan->p.P) return -1;
    const std::vector<int>& b = plan->p.bins[rank];
    if (out)
        for (long long i = 0; i < (long long)b.size() && i < capacity; ++i) out[i] = b[i];
    return (long long)b.size();
}

int pfsoft_shard_counts(const pfsoft_shard_plan* plan, int direction, long long* send, long long* recv)
{
    if (!plan || (direction != PFSOFT_SHARD_FORWARD && direction != PFSOFT_SHARD_INVERSE))
        return fail(PFSOFT_EINVAL, "bad plan or direction");
    const pfsoft_shard::Plan& p = plan->p;
    const bool fwd = direction == PFSOFT_SHARD_FORWARD;
    for (int r = 0; r < p.P; ++r) {
        if (send) send[r] = (long long)(fwd ? p.piece(p.rank, r) : p.piece(r, p.rank));
        if (recv) recv[r] = (long long)(fwd ? p.piece(r, p.rank) : p.piece(p.rank, r));
    }
    return PFSOFT_OK;
}

long long pfsoft_shard_runs(pfsoft_shard_plan* plan, int direction, int step, long long* src_off, long long* dst_off,
                            int* slot, int* len, long long capacity)
{
    if (!plan || (direction != PFSOFT_SHARD_FORWARD && direction != PFSOFT_SHARD_INVERSE) || step < 0 || step > 2)
        return -1;
    std::lock_guard<std::mutex> lk(plan->mu);
    const std::vector<Run>* hp = nullptr;
    try {
        hp = &plan->host_runs(kind_of(direction, step));
    } catch (const std::bad_alloc&) {
        return -1;
    }
    const std::vector<Run>& h = *hp;
    for (long long i = 0; i < (long long)h.size() && i < capacity; ++i) {
        if (src_off) src_off[i] = h[i].src_off;
        if (dst_off) dst_off[i] = h[i].dst_off;
        if (slot) slot[i] = h[i].slot;
        if (len) len[i] = h[i].len;
    }
    return (long long)h.size();
}

int pfsoft_shard_fft_forward(pfsoft_shard_plan* plan, const double* d_slab_grid, double* d_slab_spectrum, void* stream)
{
    std::unique_lock<std::mutex> lk;
    int rc = begin(plan, lk);
    if (rc) return rc;
    const pfsoft_shard::Plan& p = plan->p;
    const int nk = p.nk[p.rank];
    if (nk == 0) return PFSOFT_OK;
    if (!d_slab_grid || !d_slab_spectrum) return fail(PFSOFT_EINVAL, "null data pointer");
    if (d_slab_grid == d_slab_spectrum) return fail(PFSOFT_EINVAL, "slab grid and slab spectrum must not alias");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    BandTables t;
    if ((rc = tables_for(p.B, s, &t))) return rc;
    const long long N = p.N, n2 = N * N, K = nk;
    // F1: gamma DFT of each layer row, G[kk][c][e] -> S[e][c][kk]; F2: alpha DFT in place
    FftPassArgs f1 = slab_pass(p.N, nk, t, FftStrides{n2, N, 1}, FftStrides{1, K, N * K}, 1.0);
    FftPassArgs f2 = slab_pass(p.N, nk, t, FftStrides{1, N * K, K}, FftStrides{1, N * K, K}, 1.0);
    if (f1.nstages == 0) return fail(PFSOFT_EINVAL, "FFT length cannot be planned");
    const double2* G = reinterpret_cast<const double2*>(d_slab_grid);
    double2* S = reinterpret_cast<double2*>(d_slab_spectrum);
    cudaError_t e = fft_pass_launch(G, S, f1, p.N, -1, s);
    if (e == cudaSuccess) e = fft_pass_launch(S, S, f2, p.N, -1, s);
    return e == cudaSuccess ? PFSOFT_OK : cuda_fail(e, "shard FFT launch");
}

int pfsoft_shard_fft_inverse(pfsoft_shard_plan* plan, double* d_slab_spectrum, double* d_slab_grid, void* stream)
{
    std::unique_lock<std::mutex> lk;
    int rc = begin(plan, lk);
    if (rc) return rc;
    const pfsoft_shard::Plan& p = plan->p;
    const int nk = p.nk[p.rank];
    if (nk == 0) return PFSOFT_OK;
    if (!d_slab_grid || !d_slab_spectrum) return fail(PFSOFT_EINVAL, "null data pointer");
    if (d_slab_grid == d_slab_spectrum) return fail(PFSOFT_EINVAL, "slab grid and slab spectrum must not alias");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    BandTables t;
    if ((rc = tables_for(p.B, s, &t))) return rc;
    const long long N = p.N, n2 = N * N, K = nk;
    FftPassArgs i2 = slab_pass(p.N, nk, t, FftStrides{1, N * K, K}, FftStrides{1, N * K, K}, 1.0);
    // scaled by 1/(4B^2) as the single-GPU path (src/fn_idsoft.cpp:289)
    FftPassArgs i1 = slab_pass(p.N, nk, t, FftStrides{1, K, N * K}, FftStrides{n2, N, 1}, 1.0 / (4.0 * p.B * p.B));
    if (i1.nstages == 0) return fail(PFSOFT_EINVAL, "FFT length cannot be planned");
    double2* S = reinterpret_cast<double2*>(d_slab_spectrum);
    double2* G = reinterpret_cast<double2*>(d_slab_grid);
    const long long total = (long long)(2 * p.N - 1) * nk;
    const int blocks = (int)((total + 255) / 256 < 1024 ? (total + 255) / 256 : 1024);
    zero_nyquist_slab_kernel<<<blocks, 256, 0, s>>>(S, p.B, nk);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = fft_pass_launch(S, S, i2, p.N, +1, s);
    if (e == cudaSuccess) e = fft_pass_launch(S, G, i1, p.N, +1, s);
    return e == cudaSuccess ? PFSOFT_OK : cuda_fail(e, "shard FFT launch");
}

int pfsoft_shard_dwt_forward(pfsoft_shard_plan* plan, const double* d_spectrum, double* d_coeffs, void* stream)
{
    std::unique_lock<std::mutex> lk;
    int rc = begin(plan, lk);
    if (rc) return rc;
    if (!d_spectrum || !d_coeffs) return fail(PFSOFT_EINVAL, "null data pointer");
    const pfsoft_shard::Plan& p = plan->p;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(d_coeffs, 0, pfsoft_coef_count(p.B) * 2 * sizeof(double), s);
    if (e != cudaSuccess) return cuda_fail(e, "shard coefficient clear");
    const int n = (int)p.classes[p.rank].size();
    if (n == 0) return PFSOFT_OK;
    BandTables t;
    if ((rc = tables_for(p.B, s, &t))) return rc;
    DwtArgs a = dwt_args_for(t);
    a.classes = plan->d_classes;
    a.n_classes = n;
    e = dwt_forward_launch(reinterpret_cast<const double2*>(d_spectrum), reinterpret_cast<double2*>(d_coeffs), a, 0, s);
    return e == cudaSuccess ? PFSOFT_OK : cuda_fail(e, "shard DWT launch");
}

int pfsoft_shard_dwt_inverse(pfsoft_shard_plan* plan, const double* d_coeffs, double* d_spectrum, void* stream)
{
    std::unique_lock<std::mutex> lk;
    int rc = begin(plan, lk);
    if (rc) return rc;
    if (!d_spectrum || !d_coeffs) return fail(PFSOFT_EINVAL, "null data pointer");
    const pfsoft_shard::Plan& p = plan->p;
    const int n = (int)p.classes[p.rank].size();
    if (n == 0) return PFSOFT_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    BandTables t;
    if ((rc = tables_for(p.B, s, &t))) return rc;
    DwtArgs a = dwt_args_for(t);
    a.classes = plan->d_classes;
    a.n_classes = n;
    cudaError_t e = dwt_inverse_launch(reinterpret_cast<const double2*>(d_coeffs), reinterpret_cast<double2*>(d_spectrum), a, 0, s);
    return e == cudaSuccess ? PFSOFT_OK : cuda_fail(e, "shard DWT launch");
}

int pfsoft_shard_scatter(pfsoft_shard_plan* plan, int direction, const double* d_src, double* const* d_dst, void* stream)
{
    std::unique_lock<std::mutex> lk;
    int rc = begin(plan, lk);
    if (rc) return rc;
    if (direction != PFSOFT_SHARD_FORWARD && direction != PFSOFT_SHARD_INVERSE) return fail(PFSOFT_EINVAL, "bad direction");
    if (!d_dst) return fail(PFSOFT_EINVAL, "null destination table");
    DstTable dst;
    memset(&dst, 0, sizeof(dst));
    const pfsoft_shard::Plan& p = plan->p;
    for (int r = 0; r < p.P; ++r) {
        // a rank whose part is empty (no layers, no classes) may pass a null buffer
        const bool used = direction == PFSOFT_SHARD_FORWARD ? p.piece(p.rank, r) > 0 : p.piece(r, p.rank) > 0;
        if (used && !d_dst[r]) return fail(PFSOFT_EINVAL, "null destination buffer of a rank that receives data");
        dst.p[r] = reinterpret_cast<double2*>(d_dst[r]);
    }
    return run_copy(plan, kind_of(direction, 0), d_src, dst, false, static_cast<cudaStream_t>(stream));
}

int pfsoft_shard_pack(pfsoft_shard_plan* plan, int direction, const double* d_src, double* d_send, void* stream)
{
    std::unique_lock<std::mutex> lk;
    int rc = begin(plan, lk);
    if (rc) return rc;
    if (direction != PFSOFT_SHARD_FORWARD && direction != PFSOFT_SHARD_INVERSE) return fail(PFSOFT_EINVAL, "bad direction");
    DstTable dst;
    memset(&dst, 0, sizeof(dst));
    dst.p[0] = reinterpret_cast<double2*>(d_send);
    return run_copy(plan, kind_of(direction, 1), d_src, dst, true, static_cast<cudaStream_t>(stream));
}

int pfsoft_shard_unpack(pfsoft_shard_plan* plan, int direction, const double* d_recv, double* d_dst, void* stream)
{
    std::unique_lock<std::mutex> lk;
    int rc = begin(plan, lk);
    if (rc) return rc;
    if (direction != PFSOFT_SHARD_FORWARD && direction != PFSOFT_SHARD_INVERSE) return fail(PFSOFT_EINVAL, "bad direction");
    DstTable dst;
    memset(&dst, 0, sizeof(dst));
    dst.p[0] = reinterpret_cast<double2*>(d_dst);
    return run_copy(plan, kind_of(direction, 2), d_recv, dst, true, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
