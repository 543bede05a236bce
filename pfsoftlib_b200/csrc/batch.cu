// Batched SO(3) transforms over many bandwidths (C ABI: pfsoft_batch_*).
//
// A batch plan groups its transforms by bandwidth. One forward execution is
//   per group:  F1 (gamma DFT -> beta-innermost spectrum), F2 (alpha DFT)   [one launch each,
//               gridDim.z = transforms of the group]
//   all groups: one persistent DWT launch over every (group, order class, transform block)
//               item, longest first (dwt_batch.cu)
// and the inverse runs the mirror image. FP64 groups above B = 128 run the per-transform DWT
// kernels; with PFSOFT_BATCH_SPLIT every group up to B = 256 shares one split-precision launch.
// The whole sequence is captured once into a CUDA graph; the device tables of grid and
// coefficient pointers that the kernels read are refreshed before each replay, so one graph
// serves any buffers.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/pfsoft_b200.h"
#include "common.cuh"
#include "dwt.cuh"
#include "fft.cuh"

using namespace pfsoft_dev;

namespace pfsoft_dev {
int tables_for(int B, cudaStream_t s, BandTables* out);   // api.cu: cached tables of a bandwidth
}

namespace {

constexpr int kBatchMaxFused = 128;   // largest bandwidth of the fused DWT launch (N <= 256)

// Autotuner's split-precision choice per bandwidth (0 default = split where supported, 1 split,
// -1 FP64), read when a PFSOFT_BATCH_SPLIT plan is created.
signed char g_split_choice[513] = {};
bool g_split_all = true;

bool split_wanted(int B)
{
    if (B >= 1 && B <= 512 && g_split_choice[B]) return g_split_choice[B] > 0;
    return g_split_all;
}

__global__ void zero_nyquist_batched(double2* const* X, int B)
{
    double2* x = X[blockIdx.z];
    const int N = 2 * B;
    const long long total = (long long)(2 * N - 1) * N;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const long long v = i / N;
        const int k = (int)(i - v * N);
        int row, col;
        if (v < N) {
            row = B;
            col = (int)v;
        } else {
            col = B;
            row = (int)(v - N);
            if (row >= B) ++row;
        }
        x[((size_t)row * N + col) * N + k] = make_double2(0.0, 0.0);
    }
}

int fail(int status, const std::string& msg)
{
    set_last_error(msg.c_str());
    return status;
}

}  // namespace


namespace pfsoft_dev {

// FFT pass of one same-bandwidth group: forward F1 (gamma DFT, grid -> beta-innermost spectrum)
// and F2 (alpha DFT in place), inverse I2 (alpha, in place) and I1 (gamma, spectrum -> grid,
// scaled 1/(4B^2)). grids / ws are device tables with one pointer per transform.
FftPassArgs group_pass_args(int dir, bool first, const BandTables& t, double2** grids, double2** ws)
{
    const long long n = t.N, n2 = n * n;
    FftPassArgs a;
    memset(&a, 0, sizeof(a));
    a.n = t.N;
    a.nvec = t.N;
    a.kb = fft_tile_vectors(t.N);
    a.nstages = fft_plan_radices(t.N, a.radix, a.ns);
    a.twiddle = t.twiddle;
    a.bluestein = t.bluestein;
    a.scale = 1.0;
    if (dir == 0 && first) {          // F1
        a.src = FftStrides{n2, n, 1};
        a.dst = FftStrides{1, n, n2};
        a.srcs = grids;
        a.dsts = ws;
    } else if (dir == 0 || first) {   // F2 / I2, in place
        a.src = a.dst = FftStrides{1, n2, n};
        a.srcs = ws;
        a.dsts = ws;
    } else {                          // I1
        a.src = FftStrides{1, n, n2};
        a.dst = FftStrides{n2, n, 1};
        a.srcs = ws;
        a.dsts = grids;
        a.scale = 1.0 / (4.0 * t.B * t.B);
    }
    return a;
}

cudaError_t zero_nyquist_launch(double2** ws, int B, int T, cudaStream_t s)
{
    const int N = 2 * B;
    const long long total = (long long)(2 * N - 1) * N;
    dim3 grid((unsigned)std::min<long long>((total + 255) / 256, 1024), 1, (unsigned)T);
    zero_nyquist_batched<<<grid, 256, 0, s>>>(ws, B);
    return cudaGetLastError();
}

// Per-transform DWT launches of a group (bandwidths above the fused launch); X / coeffs are host
// arrays of the device pointers.
cudaError_t dwt_per_transform(int dir, const BandTables& t, int T, double2* const* X, double2* const* coeffs,
                              cudaStream_t s)
{
    const DwtArgs a = dwt_args_for(t);
    for (int i = 0; i < T; ++i) {
        cudaError_t e = dir == 0 ? dwt_forward_launch(X[i], coeffs[i], a, 0, s) : dwt_inverse_launch(coeffs[i], X[i], a, 0, s);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// One same-bandwidth group of T transforms in direction dir (0 forward, 1 inverse) on stream s.
// d_grids / d_coefs / d_ws are device tables of T pointers; d_group describes the group for the
// fused DWT and d_items lists its items (group_items); *d_counter is reset here. Bandwidths
// above the fused launch use the per-transform kernels with the host copies h_coef / h_ws.
int launch_group(int dir, const BandTables& t, int T, double2** d_grids, double2** d_ws, const DwtGroup* d_group,
                 const DwtItem* d_items, int n_items, int* d_counter, int tpc, double2* const* h_coef,
                 double2* const* h_ws, cudaStream_t s)
{
    const int sign = dir == 0 ? -1 : +1;
    auto pass = [&](bool first) {
        return fft_pass_launch(nullptr, nullptr, group_pass_args(dir, first, t, d_grids, d_ws), t.N, sign, s, T);
    };
    // both passes of the direction: one fused launch (counters past each spectrum) or two
    auto passes = [&]() -> cudaError_t {
        const FftPassArgs a = group_pass_args(dir, true, t, d_grids, d_ws), b = group_pass_args(dir, false, t, d_grids, d_ws);
        if (fft_fused_enabled(t.N) && fft_fused_chunk(a, b))
            return fft_fused_launch(sign, a, b, t.N, t.N, T, nullptr, nullptr, nullptr, nullptr, nullptr,
                                    (long long)t.N * t.N * t.N, s);
        cudaError_t e = pass(true);
        return e == cudaSuccess ? pass(false) : e;
    };
    auto dwt = [&]() -> cudaError_t {
        if (t.B > kBatchMaxFused) return dwt_per_transform(dir, t, T, h_ws, h_coef, s);
        cudaError_t e = cudaMemsetAsync(d_counter, 0, sizeof(int), s);
        if (e != cudaSuccess) return e;
        return dwt_batch_launch(dir, d_group, d_items, n_items, d_counter, tpc, t.N <= 64 ? 64 : (t.N <= 128 ? 128 : 256), s);
    };
    cudaError_t e;
    if (dir == 0) {
        e = passes();
        if (e == cudaSuccess) e = dwt();
    } else {
        e = zero_nyquist_launch(d_ws, t.B, T, s);
        if (e == cudaSuccess) e = dwt();
        if (e == cudaSuccess) e = passes();
    }
    if (e != cudaSuccess) return fail(PFSOFT_ECUDA, std::string("group launch: ") + cudaGetErrorString(e));
    return PFSOFT_OK;
}

// Fused-DWT work items of one group of T transforms at bandwidth B, longest first.
void group_items(int B, int T, int tpc, std::vector<DwtItem>& out)
{
    std::vector<std::pair<double, DwtItem> > v;
    for (int c = 0; c < num_classes(B); ++c) {
        int M, Mp;
        class_orders(c, M, Mp);
        for (int t0 = 0; t0 < T; t0 += tpc) {
            DwtItem it;
            it.group = 0;
            it.cls = c;
            it.t0 = t0;
            it.nt = std::min(tpc, T - t0);
            v.push_back(std::make_pair((double)(B - M) * it.nt + 64.0, it));
        }
    }
    std::stable_sort(v.begin(), v.end(), [](const std::pair<double, DwtItem>& a, const std::pair<double, DwtItem>& b) {
        return a.first > b.first;
    });
    out.clear();
    for (auto& p : v) out.push_back(p.second);
}

}  // namespace pfsoft_dev

struct pfsoft_batch {
    struct Group {
        int B = 0, N = 0;
        std::vector<int> members;   // transform indices in the caller's order
        BandTables tables;
        size_t ptr_base = 0;        // offset of this group's entries in the pointer tables
        bool split = false;         // DWT on the split-precision tensor-core kernel
    };
    int count = 0;
    int tpc = 1;
    int nmax = 0;
    bool use_graph = true;
    std::vector<Group> groups;
    // device: pointer tables [3][count] (grid, coeffs, workspace) in group order
    double2** d_ptr = nullptr;
    double2** h_ptr = nullptr;   // pinned staging of the same
    DwtGroup* d_groups_fwd = nullptr;
    DwtGroup* d_groups_inv = nullptr;
    DwtItem* d_items = nullptr;
    int n_items = 0;
    int* d_counter = nullptr;
    // split-precision DWT (PFSOFT_BATCH_SPLIT): segments of the groups it takes (one per group),
    // their item counts, and the sticky status of its bounded waits
    void* d_split_fwd = nullptr;
    void* d_split_inv = nullptr;
    int n_split_fwd = 0, n_split_inv = 0;
    int n_split_seg = 0;
    int* d_split = nullptr;   // [0] counter, [1] status
    void* ws = nullptr;
    size_t ws_bytes = 0;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    cudaEvent_t uploaded = nullptr;   // the last pointer upload has read h_ptr
    std::mutex mu;

    double2** grid_ptrs() const { return d_ptr; }
    double2** coef_ptrs() const { return d_ptr + count; }
    double2** ws_ptrs() const { return d_ptr + 2 * (size_t)count; }
};

namespace {

// Sequence of one direction on stream s (captured into a graph, or run directly).
int enqueue(pfsoft_batch* b, int dir, cudaStream_t s)
{
    const int sign = dir == 0 ? -1 : +1;
    auto fft_group = [&](const pfsoft_batch::Group& g, bool first_pass) -> cudaError_t {
        FftPassArgs a = group_pass_args(dir, first_pass, g.tables, b->grid_ptrs() + g.ptr_base, b->ws_ptrs() + g.ptr_base);
        return fft_pass_launch(nullptr, nullptr, a, g.N, sign, s, (int)g.members.size());
    };
    // both passes of a group: one fused launch when the plan allows, else the two passes
    auto fft_both = [&](const pfsoft_batch::Group& g) -> cudaError_t {
        const FftPassArgs a = group_pass_args(dir, true, g.tables, b->grid_ptrs() + g.ptr_base, b->ws_ptrs() + g.ptr_base);
        const FftPassArgs c = group_pass_args(dir, false, g.tables, b->grid_ptrs() + g.ptr_base, b->ws_ptrs() + g.ptr_base);
        if (fft_fused_enabled(g.N) && fft_fused_chunk(a, c))
            return fft_fused_launch(sign, a, c, g.N, g.N, (int)g.members.size(), nullptr, nullptr, nullptr, nullptr, nullptr,
                                    (long long)g.N * g.N * g.N + (g.split ? (long long)dwt_split_aux_elems(g.B) : 0), s);
        cudaError_t e = fft_group(g, true);
        return e == cudaSuccess ? fft_group(g, false) : e;
    };
    auto dwt_large = [&](const pfsoft_batch::Group& g) -> cudaError_t {
        const size_t c = (size_t)b->count;
        return dwt_per_transform(dir, g.tables, (int)g.members.size(), b->h_ptr + 2 * c + g.ptr_base,
                                 b->h_ptr + c + g.ptr_base, s);
    };
    cudaError_t e = cudaSuccess;
    if (dir == 0) {
        for (const auto& g : b->groups)
            if (e == cudaSuccess) e = fft_both(g);
        if (e == cudaSuccess && b->n_items > 0) {
            e = cudaMemsetAsync(b->d_counter, 0, sizeof(int), s);
            if (e == cudaSuccess) e = dwt_batch_launch(0, b->d_groups_fwd, b->d_items, b->n_items, b->d_counter, b->tpc, b->nmax, s);
        }
        for (const auto& g : b->groups)
            if (e == cudaSuccess && g.split)
                e = dwt_split_scales(0, g.B, (int)g.members.size(), b->ws_ptrs() + g.ptr_base, b->coef_ptrs() + g.ptr_base, g.tables.w, s);
        if (e == cudaSuccess && b->n_split_fwd > 0) {
            e = cudaMemsetAsync(b->d_split, 0, sizeof(int), s);
            if (e == cudaSuccess)
                e = dwt_split_launch(0, b->d_groups_fwd, b->d_split_fwd, b->n_split_seg, b->n_split_fwd, b->d_split + 1, s);
        }
        for (const auto& g : b->groups)
            if (e == cudaSuccess && g.B > kBatchMaxFused && !g.split) e = dwt_large(g);
    } else {
        for (const auto& g : b->groups)
            if (e == cudaSuccess) e = zero_nyquist_launch(b->ws_ptrs() + g.ptr_base, g.B, (int)g.members.size(), s);
        if (e == cudaSuccess && b->n_items > 0) {
            e = cudaMemsetAsync(b->d_counter, 0, sizeof(int), s);
            if (e == cudaSuccess) e = dwt_batch_launch(1, b->d_groups_inv, b->d_items, b->n_items, b->d_counter, b->tpc, b->nmax, s);
        }
        for (const auto& g : b->groups)
            if (e == cudaSuccess && g.split)
                e = dwt_split_scales(1, g.B, (int)g.members.size(), b->ws_ptrs() + g.ptr_base, b->coef_ptrs() + g.ptr_base, g.tables.w, s);
        if (e == cudaSuccess && b->n_split_inv > 0) {
            e = cudaMemsetAsync(b->d_split, 0, sizeof(int), s);
            if (e == cudaSuccess)
                e = dwt_split_launch(1, b->d_groups_inv, b->d_split_inv, b->n_split_seg, b->n_split_inv, b->d_split + 1, s);
        }
        for (const auto& g : b->groups)
            if (e == cudaSuccess && g.B > kBatchMaxFused && !g.split) e = dwt_large(g);
        for (const auto& g : b->groups)
            if (e == cudaSuccess) e = fft_both(g);
    }
    if (e != cudaSuccess) return fail(PFSOFT_ECUDA, std::string("batch launch: ") + cudaGetErrorString(e));
    return PFSOFT_OK;
}

void free_batch(pfsoft_batch* b)
{
    for (auto& g : b->graph)
        if (g) cudaGraphExecDestroy(g);
    if (b->uploaded) cudaEventDestroy(b->uploaded);
    cudaFree(b->d_ptr);
    cudaFreeHost(b->h_ptr);
    cudaFree(b->d_groups_fwd);
    cudaFree(b->d_groups_inv);
    cudaFree(b->d_items);
    cudaFree(b->d_counter);
    cudaFree(b->d_split_fwd);
    cudaFree(b->d_split_inv);
    cudaFree(b->d_split);
    cudaFree(b->ws);
    delete b;
}

}  // namespace

extern "C" {

int pfsoft_batch_create(const int* bandwidths, int count, int transforms_per_cta, int flags, pfsoft_batch** out)
{
    set_last_error("");
    if (!out) return fail(PFSOFT_EINVAL, "null output handle");
    *out = nullptr;
    if (!bandwidths || count < 1) return fail(PFSOFT_EINVAL, "batch needs at least one bandwidth");
    if (transforms_per_cta != 0 && transforms_per_cta != 1 && transforms_per_cta != 2 && transforms_per_cta != 4)
        return fail(PFSOFT_EINVAL, "transforms_per_cta must be 0 (auto), 1, 2 or 4");
    for (int i = 0; i < count; ++i)
        if (bandwidths[i] < 1 || bandwidths[i] > 512) return fail(PFSOFT_EINVAL, "bandwidth must be in [1, 512]");
    pfsoft_batch* b = new pfsoft_batch();
    b->count = count;
    b->use_graph = (flags & 1) == 0;
    std::map<int, std::vector<int> > by_b;
    for (int i = 0; i < count; ++i) by_b[bandwidths[i]].push_back(i);
    size_t base = 0, ws_total = 0;
    std::vector<size_t> ws_off(count);
    for (auto& kv : by_b) {
        pfsoft_batch::Group g;
        g.B = kv.first;
        g.N = 2 * kv.first;
        g.members = kv.second;
        g.ptr_base = base;
        base += g.members.size();
        g.split = (flags & PFSOFT_BATCH_SPLIT) && dwt_split_supported(g.B) && split_wanted(g.B);
        for (int t : g.members) {
            ws_off[t] = ws_total;
            ws_total += ((((size_t)g.N * g.N * g.N + (g.split ? dwt_split_aux_elems(g.B) : 0)) * sizeof(double2) + kFftSyncBytes
                          + 255) & ~(size_t)255);   // each workspace 256-byte aligned
        }
        int rc = tables_for(g.B, nullptr, &g.tables);
        if (rc) {
            free_batch(b);
            return rc;
        }
        if (g.B <= kBatchMaxFused && !g.split) b->nmax = std::max(b->nmax, g.N);
        b->groups.push_back(g);
    }
    b->tpc = transforms_per_cta ? transforms_per_cta : dwt_batch_transforms_per_cta(std::max(b->nmax, 2));
    // work items, longest first: (B - M) degrees x N columns of beta x transforms
    std::vector<DwtItem> items;
    std::vector<double> cost;
    std::vector<DwtGroup> dg_f, dg_i;
    int gi_fused = 0;
    std::vector<int> fused_index(b->groups.size(), -1);
    std::vector<int> split_group, split_B, split_T;   // the split groups: index in d_groups, B, T
    for (size_t gi = 0; gi < b->groups.size(); ++gi) {
        const auto& g = b->groups[gi];
        if (g.B > kBatchMaxFused && !g.split) continue;
        fused_index[gi] = gi_fused++;
        const int T = (int)g.members.size();
        if (g.split) {
            split_group.push_back(fused_index[gi]);
            split_B.push_back(g.B);
            split_T.push_back(T);
            continue;
        }
        for (int c = 0; c < num_classes(g.B); ++c) {
            int M, Mp;
            class_orders(c, M, Mp);
            for (int t0 = 0; t0 < T; t0 += b->tpc) {
                DwtItem it;
                it.group = fused_index[gi];
                it.cls = c;
                it.t0 = t0;
                it.nt = std::min(b->tpc, T - t0);
                items.push_back(it);
                cost.push_back((double)(g.B - M) * g.N * it.nt + 64.0 * g.N);
            }
        }
    }
    std::vector<unsigned char> split_f, split_i;   // forward / inverse segments
    const int n_split_f = dwt_split_segments(0, split_group, split_B, split_T, split_f);
    const int n_split_i = dwt_split_segments(1, split_group, split_B, split_T, split_i);
    std::vector<int> order(items.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost[x] > cost[y]; });
    std::vector<DwtItem> sorted(items.size());
    for (size_t i = 0; i < order.size(); ++i) sorted[i] = items[order[i]];
    b->n_items = (int)sorted.size();

    cudaError_t e = cudaMalloc(&b->d_ptr, 3 * (size_t)count * sizeof(double2*));
    if (e == cudaSuccess) e = cudaHostAlloc(&b->h_ptr, 3 * (size_t)count * sizeof(double2*), cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_counter, sizeof(int));
    if (e == cudaSuccess && !sorted.empty()) e = cudaMalloc(&b->d_items, sorted.size() * sizeof(DwtItem));
    if (e == cudaSuccess) e = cudaMalloc(&b->ws, ws_total);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->uploaded, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_split, 2 * sizeof(int));
    if (e == cudaSuccess && n_split_f > 0) e = cudaMalloc(&b->d_split_fwd, split_f.size());
    if (e == cudaSuccess && n_split_i > 0) e = cudaMalloc(&b->d_split_inv, split_i.size());
    if (e != cudaSuccess) {
        free_batch(b);
        return fail(PFSOFT_ENOMEM, std::string("batch allocation: ") + cudaGetErrorString(e));
    }
    b->n_split_fwd = n_split_f;
    b->n_split_inv = n_split_i;
    b->n_split_seg = (int)split_group.size();
    e = cudaMemset(b->d_split, 0, 2 * sizeof(int));
    if (e == cudaSuccess && (n_split_f > 0 || n_split_i > 0)) e = dwt_split_prepare();
    if (e == cudaSuccess && n_split_f > 0) e = cudaMemcpy(b->d_split_fwd, split_f.data(), split_f.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && n_split_i > 0) e = cudaMemcpy(b->d_split_inv, split_i.data(), split_i.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        free_batch(b);
        return fail(PFSOFT_ECUDA, std::string("batch setup: ") + cudaGetErrorString(e));
    }
    b->ws_bytes = ws_total;
    std::memset(b->h_ptr, 0, 3 * (size_t)count * sizeof(double2*));
    for (const auto& g : b->groups)
        for (size_t i = 0; i < g.members.size(); ++i)
            b->h_ptr[2 * (size_t)count + g.ptr_base + i] =
                reinterpret_cast<double2*>(static_cast<char*>(b->ws) + ws_off[g.members[i]]);
    // the fused FFT counters start cleared (a group whose FFT runs as two passes never writes them)
    for (const auto& g : b->groups) {
        const size_t sync = ((size_t)g.N * g.N * g.N + (g.split ? dwt_split_aux_elems(g.B) : 0)) * sizeof(double2);
        for (size_t i = 0; i < g.members.size() && e == cudaSuccess; ++i)
            e = cudaMemset(static_cast<char*>(b->ws) + ws_off[g.members[i]] + sync, 0, kFftSyncBytes);
    }
    if (e != cudaSuccess) {
        free_batch(b);
        return fail(PFSOFT_ECUDA, std::string("batch setup: ") + cudaGetErrorString(e));
    }
    // group descriptors for the fused DWT (pointer tables inside the device array)
    for (size_t gi = 0; gi < b->groups.size(); ++gi) {
        const auto& g = b->groups[gi];
        if (fused_index[gi] < 0) continue;
        DwtGroup d;
        d.B = g.B;
        d.N = g.N;
        d.T = (int)g.members.size();
        d.cosb = g.tables.cosb;
        d.w = g.tables.w;
        d.normf = g.tables.normf;
        d.pw_sin = g.tables.pw_sin;
        d.pw_cos = g.tables.pw_cos;
        d.rc_cf = g.tables.rc_cf;
        d.rc_f1 = g.tables.rc_f1;
        d.X = b->ws_ptrs() + g.ptr_base;
        d.coeffs = b->coef_ptrs() + g.ptr_base;
        dg_f.push_back(d);
        dg_i.push_back(d);
    }
    if (!dg_f.empty()) {
        e = cudaMalloc(&b->d_groups_fwd, dg_f.size() * sizeof(DwtGroup));
        if (e == cudaSuccess) e = cudaMalloc(&b->d_groups_inv, dg_i.size() * sizeof(DwtGroup));
        if (e == cudaSuccess) e = cudaMemcpy(b->d_groups_fwd, dg_f.data(), dg_f.size() * sizeof(DwtGroup), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(b->d_groups_inv, dg_i.data(), dg_i.size() * sizeof(DwtGroup), cudaMemcpyHostToDevice);
        if (e == cudaSuccess && !sorted.empty())
            e = cudaMemcpy(b->d_items, sorted.data(), sorted.size() * sizeof(DwtItem), cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = cudaMemcpy(b->d_ptr, b->h_ptr, 3 * (size_t)count * sizeof(double2*), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        free_batch(b);
        return fail(PFSOFT_ECUDA, std::string("batch setup: ") + cudaGetErrorString(e));
    }
    *out = b;
    return PFSOFT_OK;
}

int pfsoft_batch_destroy(pfsoft_batch* b)
{
    if (!b) return PFSOFT_OK;
    cudaDeviceSynchronize();
    free_batch(b);
    return PFSOFT_OK;
}

size_t pfsoft_batch_workspace_bytes(const pfsoft_batch* b) { return b ? b->ws_bytes : 0; }

int pfsoft_batch_transforms_per_cta(const pfsoft_batch* b) { return b ? b->tpc : 0; }

int pfsoft_split_supported(int B) { return dwt_split_supported(B) ? 1 : 0; }

int pfsoft_tune_split_bandwidth(int B, int use_split)
{
    if (B > 512) return fail(PFSOFT_EINVAL, "bandwidth must be at most 512");
    if (B <= 0) {
        g_split_all = use_split != 0;
        for (auto& v : g_split_choice) v = 0;
    } else {
        g_split_choice[B] = use_split ? 1 : -1;
    }
    return PFSOFT_OK;
}

int pfsoft_test_split_wait_ns(unsigned long long wait_ns)
{
    dwt_split_set_fail_ns(wait_ns);
    return PFSOFT_OK;
}

int pfsoft_batch_status(pfsoft_batch* b)
{
    if (!b) return fail(PFSOFT_EINVAL, "null batch");
    int st[2] = {0, 0};
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(st, b->d_split, sizeof(st), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail(PFSOFT_ECUDA, std::string("batch status: ") + cudaGetErrorString(e));
    if (st[1]) return fail(PFSOFT_ETIMEOUT, "a bounded wait in the split-precision DWT ran out");
    // the fused FFT launches' status word (counters past the first transform's spectrum of each
    // group, cleared by every launch): a bounded wait of the last execution ran out
    for (const auto& g : b->groups) {
        const char* ws = reinterpret_cast<const char*>(b->h_ptr[2 * (size_t)b->count + g.ptr_base]);
        const size_t off = ((size_t)g.N * g.N * g.N + (g.split ? dwt_split_aux_elems(g.B) : 0)) * sizeof(double2);
        int word = 0;
        e = cudaMemcpy(&word, ws + off + sizeof(int), sizeof(int), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return fail(PFSOFT_ECUDA, std::string("batch status: ") + cudaGetErrorString(e));
        if (word) return fail(PFSOFT_ETIMEOUT, "a bounded wait in the fused FFT launch ran out");
    }
    return PFSOFT_OK;
}

static int batch_run(pfsoft_batch* b, int dir, const double* const* in, double* const* out, void* stream)
{
    set_last_error("");
    if (!b) return fail(PFSOFT_EINVAL, "null batch");
    if (!in || !out) return fail(PFSOFT_EINVAL, "null pointer table");
    std::lock_guard<std::mutex> lk(b->mu);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the previous call's upload must have read the staging table before it is rewritten
    cudaError_t e = cudaEventSynchronize(b->uploaded);
    if (e != cudaSuccess) return fail(PFSOFT_ECUDA, std::string("pointer upload wait: ") + cudaGetErrorString(e));
    // pointer tables in group order (forward: in = grids, out = coeffs; inverse: swapped)
    for (const auto& g : b->groups)
        for (size_t i = 0; i < g.members.size(); ++i) {
            const int t = g.members[i];
            if (!in[t] || !out[t]) return fail(PFSOFT_EINVAL, "null buffer in the pointer table");
            double2* grid = reinterpret_cast<double2*>(const_cast<double*>(dir == 0 ? in[t] : out[t]));
            double2* coef = reinterpret_cast<double2*>(const_cast<double*>(dir == 0 ? out[t] : in[t]));
            b->h_ptr[g.ptr_base + i] = grid;
            b->h_ptr[b->count + g.ptr_base + i] = coef;
        }
    e = cudaMemcpyAsync(b->d_ptr, b->h_ptr, 2 * (size_t)b->count * sizeof(double2*), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaEventRecord(b->uploaded, s);
    if (e != cudaSuccess) return fail(PFSOFT_ECUDA, std::string("pointer upload: ") + cudaGetErrorString(e));
    bool large = false;
    for (const auto& g : b->groups) large |= g.B > kBatchMaxFused && !g.split;
    // groups above the fused limit take their per-transform pointers at enqueue time, so they
    // are launched directly; everything else replays one captured graph
    if (!b->use_graph || large) {
        // the host-side pointer table must stay valid until the launches are enqueued
        return enqueue(b, dir, s);
    }
    if (!b->graph[dir]) {
        cudaStream_t cs;
        e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
        if (e != cudaSuccess) return fail(PFSOFT_ECUDA, "capture stream");
        cudaGraph_t graph = nullptr;
        e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        int rc = PFSOFT_OK;
        if (e == cudaSuccess) rc = enqueue(b, dir, cs);
        cudaError_t e2 = cudaStreamEndCapture(cs, &graph);
        if (e == cudaSuccess) e = e2;
        if (e == cudaSuccess && rc == PFSOFT_OK) e = cudaGraphInstantiate(&b->graph[dir], graph, 0);
        if (graph) cudaGraphDestroy(graph);
        cudaStreamDestroy(cs);
        if (rc != PFSOFT_OK) return rc;
        if (e != cudaSuccess) return fail(PFSOFT_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    }
    e = cudaGraphLaunch(b->graph[dir], s);
    if (e != cudaSuccess) return fail(PFSOFT_ECUDA, std::string("graph launch: ") + cudaGetErrorString(e));
    return PFSOFT_OK;
}

int pfsoft_batch_dsoft(pfsoft_batch* b, const double* const* d_grids, double* const* d_coeffs, void* stream)
{
    return batch_run(b, 0, d_grids, d_coeffs, stream);
}

int pfsoft_batch_idsoft(pfsoft_batch* b, const double* const* d_coeffs, double* const* d_grids, void* stream)
{
    return batch_run(b, 1, d_coeffs, d_grids, stream);
}

}  // extern "C"
