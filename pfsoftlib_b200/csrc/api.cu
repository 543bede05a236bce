// C ABI of the engine (include/pfsoft_b200.h): argument checks, per-device caches of the
// bandwidth tables and scratch buffers, and the stream-ordered launch sequences.
//
//   forward  (src/fn_dsoft.cpp:76)  grid --F1--> X --F2--> X --DWT--> coeffs
//            F1: DFT over gamma (rows) of every (beta, alpha) row, written beta-innermost
//            F2: DFT over alpha of every (gamma-bin, beta) column, in place
//   inverse  (src/fn_idsoft.cpp:72) coeffs --iDWT--> X --I2--> X --I1--> grid (x 1/N^2)

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/pfsoft_b200.h"
#include "common.cuh"
#include "dwt.cuh"
#include "fft.cuh"

using namespace pfsoft_dev;

namespace {

thread_local std::string g_last_error;

int fail(int status, const std::string& msg)
{
    g_last_error = msg;
    return status;
}

int cuda_fail(cudaError_t e, const char* what)
{
    return fail(PFSOFT_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define PF_CUDA(call)                                   \
    do {                                                \
        cudaError_t e_ = (call);                        \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

constexpr int kMaxBandwidth = 512;

// Device buffers and stream of one host-staged call. A device keeps a pool of them, so that calls
// from different host threads run concurrently (one's device-to-host copy overlapping another's
// host-to-device copy on the two copy engines); a call takes a free context or makes one.
struct StagingContext {
    void* h_grid = nullptr;
    void* h_coef = nullptr;
    void* h_ws = nullptr;
    size_t h_grid_bytes = 0, h_coef_bytes = 0, h_ws_bytes = 0;
    cudaStream_t h_stream = nullptr;
    // pageable host buffers go through two pinned bounce chunks (allocated on first use)
    void* bounce[2] = {nullptr, nullptr};
    cudaEvent_t bounce_ev[2] = {nullptr, nullptr};
};

constexpr size_t kBounceBytes = (size_t)16 << 20;

// Host threads that copy the slices of one large memcpy in parallel (the pageable side of a
// bounce-buffer transfer is a host memory copy, which one thread does at a fraction of the
// host's memory bandwidth). The calling thread takes a slice too.
class CopyPool {
  public:
    static CopyPool& get()
    {
        static CopyPool* p = new CopyPool();   // lives until process exit
        return *p;
    }

    void copy(void* dst, const void* src, size_t bytes)
    {
        const int parts = (int)std::min<size_t>((size_t)nthreads_ + 1, std::max<size_t>(1, bytes >> 20));
        if (parts <= 1) {
            std::memcpy(dst, src, bytes);
            return;
        }
        std::unique_lock<std::mutex> call(call_mu_);   // one parallel copy at a time
        const size_t slice = (bytes + parts - 1) / parts;
        {
            std::lock_guard<std::mutex> lk(mu_);
            dst_ = static_cast<char*>(dst);
            src_ = static_cast<const char*>(src);
            bytes_ = bytes;
            slice_ = slice;
            next_ = 1;
            parts_ = parts;
            pending_ = parts - 1;
            ++gen_;
        }
        cv_.notify_all();
        std::memcpy(dst, src, std::min(slice, bytes));   // slice 0 on the calling thread
        std::unique_lock<std::mutex> lk(mu_);
        done_cv_.wait(lk, [&] { return pending_ == 0; });
    }

  private:
    CopyPool()
    {
        const unsigned hw = std::thread::hardware_concurrency();
        nthreads_ = (int)std::max(1u, std::min(7u, hw > 1 ? hw - 1 : 1u));
        for (int i = 0; i < nthreads_; ++i) std::thread([this] { run(); }).detach();
    }

    void run()
    {
        unsigned long long seen = 0;
        std::unique_lock<std::mutex> lk(mu_);
        for (;;) {
            cv_.wait(lk, [&] { return gen_ != seen && next_ < parts_; });
            while (next_ < parts_) {
                const int part = next_++;
                const size_t off = (size_t)part * slice_;
                const size_t n = off < bytes_ ? std::min(slice_, bytes_ - off) : 0;
                char* d = dst_ + off;
                const char* sp = src_ + off;
                lk.unlock();
                if (n) std::memcpy(d, sp, n);
                lk.lock();
                if (--pending_ == 0) done_cv_.notify_all();
            }
            seen = gen_;
        }
    }

    int nthreads_ = 1;
    std::mutex call_mu_, mu_;
    std::condition_variable cv_, done_cv_;
    char* dst_ = nullptr;
    const char* src_ = nullptr;
    size_t bytes_ = 0, slice_ = 0;
    int next_ = 0, parts_ = 0, pending_ = 0;
    unsigned long long gen_ = 0;
};

bool is_pinned(const void* p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

cudaError_t bounce_ready(StagingContext* st)
{
    for (int b = 0; b < 2; ++b) {
        if (!st->bounce[b]) {
            cudaError_t e = cudaHostAlloc(&st->bounce[b], kBounceBytes, cudaHostAllocDefault);
            if (e != cudaSuccess) return e;
        }
        if (!st->bounce_ev[b]) {
            cudaError_t e = cudaEventCreateWithFlags(&st->bounce_ev[b], cudaEventDisableTiming);
            if (e != cudaSuccess) return e;
        }
    }
    return cudaSuccess;
}

// Host-to-device copy, stream ordered: pinned sources go straight to DMA; pageable ones are
// copied by the host threads into the two pinned chunks in turn while the previous chunk's DMA runs.
cudaError_t copy_in(StagingContext* st, void* dev, const void* host, size_t bytes, cudaStream_t s)
{
    if (is_pinned(host)) return cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, s);
    cudaError_t e = bounce_ready(st);
    bool used[2] = {false, false};
    for (size_t off = 0, i = 0; e == cudaSuccess && off < bytes; off += kBounceBytes, ++i) {
        const int b = (int)(i & 1);
        const size_t n = std::min(kBounceBytes, bytes - off);
        if (used[b]) e = cudaEventSynchronize(st->bounce_ev[b]);   // its last DMA has read it
        if (e != cudaSuccess) break;
        CopyPool::get().copy(st->bounce[b], static_cast<const char*>(host) + off, n);
        e = cudaMemcpyAsync(static_cast<char*>(dev) + off, st->bounce[b], n, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaEventRecord(st->bounce_ev[b], s);
        used[b] = true;
    }
    return e;
}

// Device-to-host copy after the work queued on s; returns when the host buffer holds the data.
// Pageable destinations: chunk i's DMA into one pinned chunk overlaps the host threads' copy of
// chunk i-1 out of the other.
cudaError_t copy_out(StagingContext* st, void* host, const void* dev, size_t bytes, cudaStream_t s)
{
    if (is_pinned(host)) {
        cudaError_t e = cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, s);
        return e == cudaSuccess ? cudaStreamSynchronize(s) : e;
    }
    cudaError_t e = bounce_ready(st);
    size_t prev_off = 0, prev_n = 0;
    int prev_b = -1;
    for (size_t off = 0, i = 0; e == cudaSuccess && off < bytes; off += kBounceBytes, ++i) {
        const int b = (int)(i & 1);
        const size_t n = std::min(kBounceBytes, bytes - off);
        e = cudaMemcpyAsync(st->bounce[b], static_cast<const char*>(dev) + off, n, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaEventRecord(st->bounce_ev[b], s);
        if (e == cudaSuccess && prev_b >= 0) {
            e = cudaEventSynchronize(st->bounce_ev[prev_b]);
            if (e == cudaSuccess) CopyPool::get().copy(static_cast<char*>(host) + prev_off, st->bounce[prev_b], prev_n);
        }
        prev_b = b;
        prev_off = off;
        prev_n = n;
    }
    if (e == cudaSuccess && prev_b >= 0) {
        e = cudaEventSynchronize(st->bounce_ev[prev_b]);
        if (e == cudaSuccess) CopyPool::get().copy(static_cast<char*>(host) + prev_off, st->bounce[prev_b], prev_n);
    }
    return e;
}

struct DeviceState {
    std::mutex mu;
    std::map<int, BandTables> tables;
    void* ws = nullptr;          // library-owned workspace (NULL-workspace calls)
    size_t ws_bytes = 0;
    // host-staged calls
    std::mutex host_mu;
    std::vector<StagingContext*> staging_free;
};

// Takes a staging context of the device (a free one, else a new one) and gives it back.
struct StagingLease {
    DeviceState* st;
    StagingContext* ctx;
    explicit StagingLease(DeviceState* s) : st(s), ctx(nullptr)
    {
        std::lock_guard<std::mutex> lk(st->host_mu);
        if (!st->staging_free.empty()) {
            ctx = st->staging_free.back();
            st->staging_free.pop_back();
        } else {
            ctx = new StagingContext();   // lives until process exit
        }
    }
    ~StagingLease()
    {
        std::lock_guard<std::mutex> lk(st->host_mu);
        st->staging_free.push_back(ctx);
    }
};

std::mutex g_devices_mu;
std::map<int, DeviceState*> g_devices;

DeviceState* device_state(int dev)
{
    std::lock_guard<std::mutex> lk(g_devices_mu);
    auto it = g_devices.find(dev);
    if (it != g_devices.end()) return it->second;
    DeviceState* s = new DeviceState();   // lives until process exit
    g_devices[dev] = s;
    return s;
}

// ---- launch accounting and optional per-stage timing ------------------------------------
enum Stage { ST_FFT_FWD_ROWS, ST_FFT_FWD_COLS, ST_DWT_FWD, ST_NYQUIST, ST_DWT_INV, ST_FFT_INV_COLS, ST_FFT_INV_ROWS,
             ST_TABLES, ST_FFT_FWD_FUSED, ST_FFT_INV_FUSED, ST_COUNT };
const char* kStageNames[ST_COUNT] = {"fft_forward_gamma", "fft_forward_alpha", "dwt_forward", "zero_nyquist",
                                     "dwt_inverse", "fft_inverse_alpha", "fft_inverse_gamma", "tables",
                                     "fft_forward_fused", "fft_inverse_fused"};

std::atomic<long long> g_launches{0};

struct Profiler {
    std::mutex mu;
    bool on = false;
    struct Rec { int stage; cudaEvent_t a, b; };
    std::vector<Rec> recs;
    std::vector<cudaEvent_t> pool;
    double ms[ST_COUNT] = {0};
    long long count[ST_COUNT] = {0};

    cudaEvent_t ev()
    {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
} g_prof;

// Brackets one stage launch: counts it, and times it when profiling is on.
struct StageScope {
    int stage;
    cudaStream_t s;
    cudaEvent_t a = nullptr;
    StageScope(int st, cudaStream_t stream) : stage(st), s(stream)
    {
        g_launches.fetch_add(1, std::memory_order_relaxed);
        std::lock_guard<std::mutex> lk(g_prof.mu);
        if (g_prof.on) {
            a = g_prof.ev();
            cudaEventRecord(a, s);
        }
    }
    ~StageScope()
    {
        if (!a) return;
        std::lock_guard<std::mutex> lk(g_prof.mu);
        cudaEvent_t b = g_prof.ev();
        cudaEventRecord(b, s);
        g_prof.recs.push_back({stage, a, b});
    }
};

bool valid_bandwidth(int B) { return B >= 1 && B <= kMaxBandwidth; }

size_t grid_elems(int B)
{
    const size_t N = 2 * (size_t)B;
    return N * N * N;
}

// Tables for bandwidth B on the current device; built on first use.
int get_tables(int B, cudaStream_t stream, BandTables* out)
{
    int dev = 0;
    PF_CUDA(cudaGetDevice(&dev));
    DeviceState* st = device_state(dev);
    std::lock_guard<std::mutex> lk(st->mu);
    auto it = st->tables.find(B);
    if (it != st->tables.end()) {
        *out = it->second;
        return PFSOFT_OK;
    }
    void* mem = nullptr;
    cudaError_t e = cudaMalloc(&mem, tables_bytes(B));
    if (e != cudaSuccess) return fail(PFSOFT_ENOMEM, std::string("table allocation: ") + cudaGetErrorString(e));
    BandTables t;
    {
        StageScope sc(ST_TABLES, stream);
        e = tables_build(B, mem, &t, stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e == cudaSuccess && fft_needs_bluestein(2 * B)) {
        // lengths with a large prime factor: the FFT's Bluestein table, computed on the host
        std::vector<double2> h(fft_bluestein_elems(2 * B));
        fft_bluestein_fill(2 * B, h.data());
        void* bt = nullptr;
        e = cudaMalloc(&bt, h.size() * sizeof(double2));
        if (e == cudaSuccess) e = cudaMemcpy(bt, h.data(), h.size() * sizeof(double2), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) t.bluestein = static_cast<double2*>(bt);
        else if (bt) cudaFree(bt);
    }
    if (e != cudaSuccess) {
        cudaFree(mem);
        return cuda_fail(e, "tables_build");
    }
    st->tables[B] = t;
    *out = t;
    return PFSOFT_OK;
}

}  // namespace

namespace pfsoft_dev {
void set_last_error(const char* msg) { g_last_error = msg; }
int tables_for(int B, cudaStream_t s, BandTables* out);
}  // namespace pfsoft_dev

namespace {

// Library-owned workspace of at least `bytes` on the current device.
int get_workspace(size_t bytes, void** ws)
{
    int dev = 0;
    PF_CUDA(cudaGetDevice(&dev));
    DeviceState* st = device_state(dev);
    std::lock_guard<std::mutex> lk(st->mu);
    if (st->ws_bytes < bytes) {
        if (st->ws) {
            cudaDeviceSynchronize();
            cudaFree(st->ws);
            st->ws = nullptr;
            st->ws_bytes = 0;
        }
        cudaError_t e = cudaMalloc(&st->ws, bytes);
        if (e != cudaSuccess) return fail(PFSOFT_ENOMEM, std::string("workspace allocation: ") + cudaGetErrorString(e));
        st->ws_bytes = bytes;
    }
    *ws = st->ws;
    return PFSOFT_OK;
}

FftPassArgs pass_args(int n, int nvec, const BandTables& t, FftStrides src, FftStrides dst, double scale)
{
    FftPassArgs a;
    memset(&a, 0, sizeof(a));   // srcs/dsts null: single transform
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

DwtArgs dwt_args(const BandTables& t) { return dwt_args_for(t); }

int check_transform_args(const void* a, const void* b, int B, void*& ws, size_t ws_bytes)
{
    if (!valid_bandwidth(B)) return fail(PFSOFT_EINVAL, "bandwidth must be in [1, 512]");
    if (!a || !b) return fail(PFSOFT_EINVAL, "null data pointer");
    const size_t need = grid_elems(B) * sizeof(double2) + kFftSyncBytes;
    if (ws) {
        if (ws_bytes < need) return fail(PFSOFT_EINVAL, "workspace smaller than pfsoft_workspace_bytes(B)");
        if ((reinterpret_cast<uintptr_t>(ws) & 15) != 0) return fail(PFSOFT_EINVAL, "workspace not 16-byte aligned");
        return PFSOFT_OK;
    }
    return get_workspace(need, &ws);
}

int run_dsoft(const double* d_grid, int B, double* d_coeffs, void* ws, cudaStream_t s)
{
    BandTables t;
    int rc = get_tables(B, s, &t);
    if (rc) return rc;
    const int N = 2 * B;
    const long long n = N, n2 = n * n;
    const double2* G = reinterpret_cast<const double2*>(d_grid);
    double2* X = static_cast<double2*>(ws);
    // F1: vectors = layers k, tile = column c, elements = rows r; G[k][c][r] -> X[r][c][k]
    FftPassArgs f1 = pass_args(N, N, t, FftStrides{n2, n, 1}, FftStrides{1, n, n2}, 1.0);
    // F2: vectors = layers k, tile = gamma bin r, elements = column c; in place on X
    FftPassArgs f2 = pass_args(N, N, t, FftStrides{1, n2, n}, FftStrides{1, n2, n}, 1.0);
    if (f1.nstages == 0) return fail(PFSOFT_EINVAL, "FFT length cannot be planned");
    if (fft_fused_enabled(N) && fft_fused_chunk(f1, f2)) {
        // both passes in one launch; the counters sit past the spectrum in the workspace
        StageScope sc(ST_FFT_FWD_FUSED, s);
        PF_CUDA(fft_fused_launch(-1, f1, f2, N, N, 1, G, X, X, X, X, (long long)grid_elems(B), s));
    } else {
        {
            StageScope sc(ST_FFT_FWD_ROWS, s);
            PF_CUDA(fft_pass_launch(G, X, f1, N, -1, s));
        }
        {
            StageScope sc(ST_FFT_FWD_COLS, s);
            PF_CUDA(fft_pass_launch(X, X, f2, N, -1, s));
        }
    }
    DwtArgs a = dwt_args(t);
    {
        StageScope sc(ST_DWT_FWD, s);
        PF_CUDA(dwt_forward_launch(X, reinterpret_cast<double2*>(d_coeffs), a, 0, s));
    }
    return PFSOFT_OK;
}

int run_idsoft(const double* d_coeffs, int B, double* d_grid, void* ws, cudaStream_t s)
{
    BandTables t;
    int rc = get_tables(B, s, &t);
    if (rc) return rc;
    const int N = 2 * B;
    const long long n = N, n2 = n * n;
    double2* X = static_cast<double2*>(ws);
    double2* G = reinterpret_cast<double2*>(d_grid);
    DwtArgs a = dwt_args(t);
    a.zero_nyquist = 1;   // the Nyquist bins, which no order class writes, zeroed in the DWT's tail
    {
        StageScope sc(ST_DWT_INV, s);
        PF_CUDA(dwt_inverse_launch(reinterpret_cast<const double2*>(d_coeffs), X, a, 0, s));
    }
    // I2: inverse DFT over alpha, in place on X
    FftPassArgs i2 = pass_args(N, N, t, FftStrides{1, n2, n}, FftStrides{1, n2, n}, 1.0);
    // I1: inverse DFT over gamma, X[r][c][k] -> G[k][c][r], scaled by 1/(4B^2) (src/fn_idsoft.cpp:289)
    FftPassArgs i1 = pass_args(N, N, t, FftStrides{1, n, n2}, FftStrides{n2, n, 1}, 1.0 / (4.0 * B * B));
    if (i1.nstages == 0) return fail(PFSOFT_EINVAL, "FFT length cannot be planned");
    if (fft_fused_enabled(N) && fft_fused_chunk(i2, i1)) {
        StageScope sc(ST_FFT_INV_FUSED, s);
        PF_CUDA(fft_fused_launch(+1, i2, i1, N, N, 1, X, X, X, G, X, (long long)grid_elems(B), s));
    } else {
        {
            StageScope sc(ST_FFT_INV_COLS, s);
            PF_CUDA(fft_pass_launch(X, X, i2, N, +1, s));
        }
        {
            StageScope sc(ST_FFT_INV_ROWS, s);
            PF_CUDA(fft_pass_launch(X, G, i1, N, +1, s));
        }
    }
    return PFSOFT_OK;
}

// ---- small kernels for the DWT helper API ---------------------------------------------------

__global__ void copy_weights_kernel(const double* w, double* out, int N)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) out[k] = w[k];
}

// One thread per beta column; the reference's seed cases for any signs of (M, Mp)
// (fn_dwt.hpp:112-163) and its recurrence (:167-199).
__global__ void wigner_matrix_kernel(int B, int M, int Mp, const double* w, const double* cosb, const double* sinh,
                                     const double* cosh, double* out)
{
    const int N = 2 * B;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= N) return;
    const int aM = M < 0 ? -M : M, aMp = Mp < 0 ? -Mp : Mp;
    const int J = aM > aMp ? aM : aMp, Jmin = aM < aMp ? aM : aMp;
    double nf = sqrt((2.0 * J + 1.0) / 2.0);
    for (int i = 0; i < J - Jmin; ++i) nf *= sqrt((2.0 * J - i) / (i + 1.0));
    int cp, sp;
    if (J == aM && M >= 0) { cp = J + Mp; sp = J - Mp; }
    else if (J == aM)      { cp = J - Mp; sp = J + Mp; }
    else if (Mp >= 0)      { cp = J + M;  sp = J - M;  }
    else                   { cp = J - M;  sp = J + M;  }
    const double scale_w = w ? w[k] : 1.0;
    // extended-exponent seed (as in the DWT kernels)
    int xe;
    double ms = 1.0, mc = 1.0;
    int es = 0, ec = 0;
    {
        double xm = frexp(sinh[k], &xe);
        int p = sp;
        while (p) {
            if (p & 1) { int t2; ms = frexp(ms * xm, &t2); es += xe + t2; }
            p >>= 1;
            if (p) { int t2; xm = frexp(xm * xm, &t2); xe = 2 * xe + t2; }
        }
        xm = frexp(cosh[k], &xe);
        p = cp;
        while (p) {
            if (p & 1) { int t2; mc = frexp(mc * xm, &t2); ec += xe + t2; }
            p >>= 1;
            if (p) { int t2; xm = frexp(xm * xm, &t2); xe = 2 * xe + t2; }
        }
    }
    int ev;
    const double v = frexp(nf * scale_w * ms * mc, &ev);
    const int E = ev + es + ec;
    int sc = 0;
    double dcur;
    if (E >= -900) {
        dcur = -ldexp(v, E);
    } else {
        sc = (-900 - E + 599) / 600;
        dcur = -ldexp(v, E + 600 * sc);
    }
    double dprev = 0.0;
    const double cb = cosb[k];
    for (int l = J; l < B; ++l) {
        out[(size_t)(l - J) * N + k] = sc ? ldexp(dcur, -600 * sc) : dcur;
        if (l + 1 >= B) break;
        const double idx = (double)l;
        const double nrm = sqrt((2.0 * idx + 3.0) / (2.0 * idx + 1.0));
        const double nom = (idx + 1.0) * (2.0 * idx + 1.0);
        const double den = 1.0 / sqrt(((idx + 1) * (idx + 1) - (double)M * M) * ((idx + 1) * (idx + 1) - (double)Mp * Mp));
        const double f1 = nrm * nom * den;
        double c1 = 0.0, f2 = 0.0;
        if (l != 0) {
            const double t1 = sqrt((2.0 * idx + 3.0) / (2.0 * idx - 1.0)) * (idx + 1.0) / idx;
            const double t2 = sqrt((idx * idx - (double)M * M) * (idx * idx - (double)Mp * Mp));
            c1 = -t1 * t2 * den;
            f2 = -(double)M * Mp / (idx * (idx + 1.0));
        }
        const double nx = fma(c1, dprev, (dcur * f1) * (f2 + cb));
        dprev = dcur;
        dcur = nx;
        if (sc && fabs(dcur) >= 0x1p300) {
            dcur *= 0x1p-600;
            dprev *= 0x1p-600;
            --sc;
        }
    }
}

}  // namespace

namespace pfsoft_dev {
// Cached tables of a bandwidth on the current device (used by the batch plans).
int tables_for(int B, cudaStream_t s, BandTables* out) { return get_tables(B, s, out); }
}  // namespace pfsoft_dev

extern "C" {

const char* pfsoft_status_string(int status)
{
    switch (status) {
        case PFSOFT_OK: return "ok";
        case PFSOFT_EINVAL: return "invalid argument";
        case PFSOFT_ENOMEM: return "out of memory";
        case PFSOFT_ETIMEOUT: return "timed out";
        case PFSOFT_ECUDA: return "CUDA error";
        case PFSOFT_EBUSY: return "busy";
        case PFSOFT_ECANCELED: return "cancelled";
        default: return "unknown status";
    }
}

const char* pfsoft_last_error(void) { return g_last_error.c_str(); }

int pfsoft_version(void) { return 100; }

size_t pfsoft_coef_count(int B) { return B < 1 ? 0 : coef_offset(B); }

size_t pfsoft_grid_bytes(int B) { return B < 1 ? 0 : grid_elems(B) * sizeof(double2); }

size_t pfsoft_workspace_bytes(int B) { return B < 1 ? 0 : grid_elems(B) * sizeof(double2) + kFftSyncBytes; }

int pfsoft_cuda_dsoft(const double* d_grid, int B, double* d_coeffs, void* d_workspace, size_t workspace_bytes,
                      void* stream)
{
    g_last_error.clear();
    int rc = check_transform_args(d_grid, d_coeffs, B, d_workspace, workspace_bytes);
    if (rc) return rc;
    return run_dsoft(d_grid, B, d_coeffs, d_workspace, static_cast<cudaStream_t>(stream));
}

int pfsoft_cuda_idsoft(const double* d_coeffs, int B, double* d_grid, void* d_workspace, size_t workspace_bytes,
                       void* stream)
{
    g_last_error.clear();
    int rc = check_transform_args(d_coeffs, d_grid, B, d_workspace, workspace_bytes);
    if (rc) return rc;
    return run_idsoft(d_coeffs, B, d_grid, d_workspace, static_cast<cudaStream_t>(stream));
}

static int host_staged(int B, bool forward, const double* in, double* out)
{
    g_last_error.clear();
    if (!valid_bandwidth(B)) return fail(PFSOFT_EINVAL, "bandwidth must be in [1, 512]");
    if (!in || !out) return fail(PFSOFT_EINVAL, "null host pointer");
    int dev = 0;
    PF_CUDA(cudaGetDevice(&dev));
    StagingLease lease(device_state(dev));
    StagingContext* st = lease.ctx;
    const size_t gb = grid_elems(B) * sizeof(double2);
    const size_t cb = coef_offset(B) * sizeof(double2);
    if (!st->h_stream) PF_CUDA(cudaStreamCreateWithFlags(&st->h_stream, cudaStreamNonBlocking));
    auto grow = [](void** p, size_t* have, size_t need) -> cudaError_t {
        if (*have >= need) return cudaSuccess;
        if (*p) cudaFree(*p);
        *p = nullptr;
        *have = 0;
        cudaError_t e = cudaMalloc(p, need);
        if (e == cudaSuccess) *have = need;
        return e;
    };
    cudaError_t e = grow(&st->h_grid, &st->h_grid_bytes, gb);
    if (e == cudaSuccess) e = grow(&st->h_coef, &st->h_coef_bytes, cb);
    if (e == cudaSuccess) e = grow(&st->h_ws, &st->h_ws_bytes, gb + kFftSyncBytes);
    if (e != cudaSuccess) return fail(PFSOFT_ENOMEM, std::string("staging allocation: ") + cudaGetErrorString(e));
    cudaStream_t s = st->h_stream;
    int rc;
    if (forward) {
        PF_CUDA(copy_in(st, st->h_grid, in, gb, s));
        rc = run_dsoft(static_cast<const double*>(st->h_grid), B, static_cast<double*>(st->h_coef), st->h_ws, s);
        if (rc) return rc;
        PF_CUDA(copy_out(st, out, st->h_coef, cb, s));
    } else {
        PF_CUDA(copy_in(st, st->h_coef, in, cb, s));
        rc = run_idsoft(static_cast<const double*>(st->h_coef), B, static_cast<double*>(st->h_grid), st->h_ws, s);
        if (rc) return rc;
        PF_CUDA(copy_out(st, out, st->h_grid, gb, s));
    }
    PF_CUDA(cudaStreamSynchronize(s));
    return PFSOFT_OK;
}

int pfsoft_dsoft_host(const double* h_grid, int B, double* h_coeffs) { return host_staged(B, true, h_grid, h_coeffs); }

int pfsoft_idsoft_host(const double* h_coeffs, int B, double* h_grid) { return host_staged(B, false, h_coeffs, h_grid); }

static int layer_wise(int cols, int rows, int lays, double* d_arr, double scale, void* stream, int sign)
{
    g_last_error.clear();
    if (cols < 1 || rows < 1 || lays < 1) return fail(PFSOFT_EINVAL, "grid dimensions must be positive");
    if (cols > 65535 || rows > 65535) return fail(PFSOFT_EINVAL, "layer dimensions above 65535");
    if (!d_arr) return fail(PFSOFT_EINVAL, "null data pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // twiddle tables for both lengths: reuse the bandwidth tables when the length is even
    // and within range, else build a temporary table
    double2* G = reinterpret_cast<double2*>(d_arr);
    const long long r = rows, c = cols, layer = r * c;
    const int lens[2] = {rows, cols};
    for (int pass = 0; pass < 2; ++pass) {
        const int n = lens[pass];
        const double2* tw = nullptr;
        void* tmp = nullptr;
        const double2* blu = nullptr;
        void* tmp_b = nullptr;
        if (n % 2 == 0 && valid_bandwidth(n / 2)) {
            BandTables t;
            int rc = get_tables(n / 2, s, &t);
            if (rc) return rc;
            tw = t.twiddle;
            blu = t.bluestein;
        } else {
            // odd length: a private table (rare); freed after the stream drains
            std::vector<double2> h(n);
            for (int i = 0; i < n; ++i) {
                const long double a = 6.283185307179586476925286766559005768L * (long double)i / (long double)n;
                h[i] = make_double2((double)cosl(a), -(double)sinl(a));
            }
            PF_CUDA(cudaMalloc(&tmp, n * sizeof(double2)));
            PF_CUDA(cudaMemcpyAsync(tmp, h.data(), n * sizeof(double2), cudaMemcpyHostToDevice, s));
            PF_CUDA(cudaStreamSynchronize(s));
            tw = static_cast<const double2*>(tmp);
            if (fft_needs_bluestein(n)) {
                std::vector<double2> hb(fft_bluestein_elems(n));
                fft_bluestein_fill(n, hb.data());
                PF_CUDA(cudaMalloc(&tmp_b, hb.size() * sizeof(double2)));
                PF_CUDA(cudaMemcpy(tmp_b, hb.data(), hb.size() * sizeof(double2), cudaMemcpyHostToDevice));
                blu = static_cast<const double2*>(tmp_b);
            }
        }
        FftPassArgs a;
        memset(&a, 0, sizeof(a));
        a.n = n;
        a.kb = fft_tile_vectors(n);
        a.nstages = fft_plan_radices(n, a.radix, a.ns);
        a.twiddle = tw;
        a.bluestein = blu;
        a.scale = pass == 1 ? scale : 1.0;
        int ntiles;
        if (pass == 0) {
            // rows: vectors = layers (stride rows*cols), tile = column index, elements contiguous
            a.nvec = lays;
            a.src = a.dst = FftStrides{layer, r, 1};
            ntiles = cols;
        } else {
            // columns: vectors = row index (contiguous), tile = layer, elements stride rows
            a.nvec = rows;
            a.src = a.dst = FftStrides{1, layer, r};
            ntiles = lays;
        }
        cudaError_t e = cudaSuccess;
        if (a.nstages == 0) e = cudaErrorInvalidValue;
        // grid.y is limited to 65535 tiles: split the launch when needed
        for (int t0 = 0; e == cudaSuccess && t0 < ntiles; t0 += 65535) {
            const int nt = ntiles - t0 < 65535 ? ntiles - t0 : 65535;
            double2* base = G + (long long)t0 * a.src.sb;
            e = fft_pass_launch(base, base, a, nt, sign, s);
        }
        if (tmp || tmp_b) {
            cudaStreamSynchronize(s);
            cudaFree(tmp);
            cudaFree(tmp_b);
        }
        if (e != cudaSuccess) return cuda_fail(e, "fft_pass_launch");
    }
    return PFSOFT_OK;
}

int pfsoft_cuda_layer_wise_dft2(int cols, int rows, int lays, double* d_arr, double scale, void* stream)
{
    return layer_wise(cols, rows, lays, d_arr, scale, stream, -1);
}

int pfsoft_cuda_layer_wise_idft2(int cols, int rows, int lays, double* d_arr, double scale, void* stream)
{
    return layer_wise(cols, rows, lays, d_arr, scale, stream, +1);
}

static int layer_wise_host(int cols, int rows, int lays, double* h_arr, double scale, int sign)
{
    g_last_error.clear();
    if (cols < 1 || rows < 1 || lays < 1) return fail(PFSOFT_EINVAL, "grid dimensions must be positive");
    if (!h_arr) return fail(PFSOFT_EINVAL, "null host pointer");
    int dev = 0;
    PF_CUDA(cudaGetDevice(&dev));
    StagingLease lease(device_state(dev));
    StagingContext* st = lease.ctx;
    const size_t bytes = (size_t)cols * rows * lays * sizeof(double2);
    if (!st->h_stream) PF_CUDA(cudaStreamCreateWithFlags(&st->h_stream, cudaStreamNonBlocking));
    if (st->h_grid_bytes < bytes) {
        if (st->h_grid) cudaFree(st->h_grid);
        st->h_grid = nullptr;
        st->h_grid_bytes = 0;
        cudaError_t e = cudaMalloc(&st->h_grid, bytes);
        if (e != cudaSuccess) return fail(PFSOFT_ENOMEM, std::string("staging allocation: ") + cudaGetErrorString(e));
        st->h_grid_bytes = bytes;
    }
    cudaStream_t s = st->h_stream;
    PF_CUDA(cudaMemcpyAsync(st->h_grid, h_arr, bytes, cudaMemcpyHostToDevice, s));
    int rc = layer_wise(cols, rows, lays, static_cast<double*>(st->h_grid), scale, s, sign);
    if (rc) return rc;
    PF_CUDA(cudaMemcpyAsync(h_arr, st->h_grid, bytes, cudaMemcpyDeviceToHost, s));
    PF_CUDA(cudaStreamSynchronize(s));
    return PFSOFT_OK;
}

int pfsoft_layer_wise_dft2_host(int cols, int rows, int lays, double* h_arr, double scale)
{
    return layer_wise_host(cols, rows, lays, h_arr, scale, -1);
}

int pfsoft_layer_wise_idft2_host(int cols, int rows, int lays, double* h_arr, double scale)
{
    return layer_wise_host(cols, rows, lays, h_arr, scale, +1);
}

int pfsoft_cuda_quadrature_weights(int B, double* d_w, void* stream)
{
    g_last_error.clear();
    if (!valid_bandwidth(B)) return fail(PFSOFT_EINVAL, "bandwidth must be in [1, 512]");
    if (!d_w) return fail(PFSOFT_EINVAL, "null output pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    BandTables t;
    int rc = get_tables(B, s, &t);
    if (rc) return rc;
    copy_weights_kernel<<<(2 * B + 255) / 256, 256, 0, s>>>(t.w, d_w, 2 * B);
    PF_CUDA(cudaGetLastError());
    return PFSOFT_OK;
}

int pfsoft_cuda_wigner_d_matrix(int B, int M, int Mp, int weighted, double* d_out, void* stream)
{
    g_last_error.clear();
    if (!valid_bandwidth(B)) return fail(PFSOFT_EINVAL, "bandwidth must be in [1, 512]");
    if (!d_out) return fail(PFSOFT_EINVAL, "null output pointer");
    if (M <= -B || M >= B || Mp <= -B || Mp >= B) return fail(PFSOFT_EINVAL, "orders must satisfy |M|,|M'| < B");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    BandTables t;
    int rc = get_tables(B, s, &t);
    if (rc) return rc;
    wigner_matrix_kernel<<<(2 * B + 127) / 128, 128, 0, s>>>(B, M, Mp, weighted ? t.w : nullptr, t.cosb, t.sinh,
                                                              t.cosh, d_out);
    PF_CUDA(cudaGetLastError());
    return PFSOFT_OK;
}

long long pfsoft_launch_count(void) { return g_launches.load(); }

int pfsoft_tune_fft_fused(int B, int on)
{
    if (B > kMaxBandwidth) return fail(PFSOFT_EINVAL, "bandwidth must be at most 512");
    fft_set_fused(B <= 0 ? 0 : 2 * B, on);
    return PFSOFT_OK;
}

int pfsoft_tune_dwt_case_split(int direction, int case_split)
{
    if (direction < 0 || direction > 1 || case_split < 0 || case_split > 2) return fail(PFSOFT_EINVAL, "bad tuning value");
    dwt_set_case_split(direction, case_split);
    return PFSOFT_OK;
}

int pfsoft_profile_enable(int on)
{
    std::lock_guard<std::mutex> lk(g_prof.mu);
    g_prof.on = on != 0;
    return PFSOFT_OK;
}

int pfsoft_profile_read(double* ms, long long* launches, int max_stages)
{
    g_last_error.clear();
    std::lock_guard<std::mutex> lk(g_prof.mu);
    for (auto& r : g_prof.recs) {
        float t = 0.f;
        cudaError_t e = cudaEventSynchronize(r.b);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&t, r.a, r.b);
        if (e != cudaSuccess) return cuda_fail(e, "pfsoft_profile_read");
        g_prof.ms[r.stage] += t;
        g_prof.count[r.stage] += 1;
        g_prof.pool.push_back(r.a);
        g_prof.pool.push_back(r.b);
    }
    g_prof.recs.clear();
    const int n = max_stages < ST_COUNT ? max_stages : ST_COUNT;
    for (int i = 0; i < n; ++i) {
        if (ms) ms[i] = g_prof.ms[i];
        if (launches) launches[i] = g_prof.count[i];
        g_prof.ms[i] = 0.0;
        g_prof.count[i] = 0;
    }
    return ST_COUNT;
}

const char* pfsoft_profile_stage_name(int stage) { return (stage >= 0 && stage < ST_COUNT) ? kStageNames[stage] : ""; }

}  // extern "C"
