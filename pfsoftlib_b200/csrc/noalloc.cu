// DSOFT without any device allocation, for callers that cannot call cudaMalloc.
//
// Who needs this: a plugin whose host framework owns the device memory through its own pool
// and caps it, so a raw cudaMalloc fails or fragments that pool; a client under a hard
// per-process device-memory limit (MPS, containers) that must not grow its footprint at call
// time; a latency-critical loop where cudaMalloc/cudaFree would take driver locks and
// cudaFree would synchronise the device. pfsoft_cuda_dsoft needs a spectrum workspace and
// per-bandwidth tables, both allocated on first use; this entry point takes both from one
// file-scope device array instead.
//
// Limit: bandwidth B <= 32 (a 64^3 complex128 spectrum, 4 MiB, plus 320 KiB reserved for the
// tables, of which B = 32 needs about 276 KiB). Every GPU that loads the library holds this
// array until the process exits. All calls on a device share it and it keeps the last call's
// contents; nothing in it has to start at zero (the first FFT pass overwrites the whole spectrum
// before anything reads it, and the tables are rebuilt whenever the bandwidth changes). Calls
// that overlap on the GPU race on it. Once a call has been recorded into a CUDA graph on a
// device, every later call on that device rebuilds the tables (three small kernels): a graph
// replay rewrites the array with its own bandwidth's tables, which the host cannot see.

#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

#include "../../include/pfsoft_b200.h"
#include "common.cuh"
#include "dwt.cuh"
#include "fft.cuh"

using namespace pfsoft_dev;

namespace {

constexpr int kNoAllocMaxB = 32;
constexpr size_t kSpectrumBytes = (size_t)(2 * kNoAllocMaxB) * (2 * kNoAllocMaxB) * (2 * kNoAllocMaxB) * sizeof(double2);
constexpr size_t kTableBytes = 320 * 1024;
constexpr int kMaxDevices = 64;

// The scratch: spectrum first, tables after it. In host code this name is only a handle for
// cudaGetSymbolAddress; the kernels receive the device address it returns.
__device__ __align__(256) unsigned char g_noalloc_scratch[kSpectrumBytes + kTableBytes];

struct NoAllocDevice {
    bool ready;          // symbol address resolved on this device
    bool captured;       // a call was recorded into a graph: the host no longer knows the tables
    unsigned char* base; // device address of g_noalloc_scratch
    int tables_B;        // bandwidth whose tables the array holds (0 = unknown)
    BandTables tables;
};

std::mutex g_mu;                       // guards g_dev (host bookkeeping only)
NoAllocDevice g_dev[kMaxDevices] = {};

int fail(int status, const char* msg)
{
    set_last_error(msg);
    return status;
}

}  // namespace

extern "C" {

int pfsoft_cuda_dsoft_noalloc(const double* d_grid, int B, double* d_coeffs, void* stream)
{
    set_last_error("");
    if (B < 1 || B > kNoAllocMaxB) return fail(PFSOFT_EINVAL, "pfsoft_cuda_dsoft_noalloc: bandwidth must be in [1, 32]");
    if (!d_grid || !d_coeffs) return fail(PFSOFT_EINVAL, "pfsoft_cuda_dsoft_noalloc: null data pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return fail(PFSOFT_ECUDA, "pfsoft_cuda_dsoft_noalloc: cudaGetDevice failed");
    if (dev < 0 || dev >= kMaxDevices) return fail(PFSOFT_EINVAL, "pfsoft_cuda_dsoft_noalloc: device ordinal above 63");

    std::lock_guard<std::mutex> lk(g_mu);
    NoAllocDevice& d = g_dev[dev];
    if (!d.ready) {
        // once per device, with that device current: the array's device address
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return fail(PFSOFT_ECUDA, "pfsoft_cuda_dsoft_noalloc: cudaGetSymbolAddress failed");
        d.base = static_cast<unsigned char*>(p);
        d.ready = true;
        d.tables_B = 0;
    }
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess)
        return fail(PFSOFT_ECUDA, "pfsoft_cuda_dsoft_noalloc: cudaStreamIsCapturing failed");
    if (cap != cudaStreamCaptureStatusNone) d.captured = true;
    if (d.captured || d.tables_B != B) {
        // recorded into the captured work too, so that every replay builds the tables it reads
        if (tables_bytes(B) > kTableBytes) return fail(PFSOFT_EINVAL, "pfsoft_cuda_dsoft_noalloc: tables exceed the reserve");
        if (tables_build(B, d.base + kSpectrumBytes, &d.tables, s) != cudaSuccess) {
            d.tables_B = 0;
            return fail(PFSOFT_ECUDA, "pfsoft_cuda_dsoft_noalloc: table kernels failed to launch");
        }
        d.tables_B = d.captured ? 0 : B;
    }
    const BandTables& t = d.tables;
    const int N = 2 * B;
    const long long n = N, n2 = n * n;
    double2* X = reinterpret_cast<double2*>(d.base);

    // the same three stages as pfsoft_cuda_dsoft: gamma DFT into the beta-innermost spectrum,
    // alpha DFT in place, discrete Wigner transform
    FftPassArgs f;
    memset(&f, 0, sizeof(f));
    f.n = N;
    f.nvec = N;
    f.kb = fft_tile_vectors(N);
    f.nstages = fft_plan_radices(N, f.radix, f.ns);
    f.scale = 1.0;
    f.twiddle = t.twiddle;
    if (f.nstages == 0) return fail(PFSOFT_EINVAL, "pfsoft_cuda_dsoft_noalloc: FFT length cannot be planned");
    FftPassArgs f1 = f, f2 = f;
    f1.src = FftStrides{n2, n, 1};
    f1.dst = FftStrides{1, n, n2};
    f2.src = f2.dst = FftStrides{1, n2, n};
    if (fft_pass_launch(reinterpret_cast<const double2*>(d_grid), X, f1, N, -1, s) != cudaSuccess ||
        fft_pass_launch(X, X, f2, N, -1, s) != cudaSuccess)
        return fail(PFSOFT_ECUDA, "pfsoft_cuda_dsoft_noalloc: FFT launch failed");
    const DwtArgs a = dwt_args_for(t);
    if (dwt_forward_launch(X, reinterpret_cast<double2*>(d_coeffs), a, 0, s) != cudaSuccess)
        return fail(PFSOFT_ECUDA, "pfsoft_cuda_dsoft_noalloc: DWT launch failed");
    return PFSOFT_OK;
}

}  // extern "C"
