// Transform server (C ABI: pfsoft_server_*): a persistent request loop with continuous batching.
//
// Requests (DSOFT or iDSOFT of one caller-owned device grid / coefficient buffer) enter a FIFO
// queue. A scheduler thread forms batches of equal direction and bandwidth (serving.hpp: the
// arena the HBM budget is counted against, and the batch former), and launches each batch on a
// free stream as one group: batched FFT passes (gridDim.z = transforms) and one fused DWT launch
// (dwt_batch.cu) over the batch's (order class, transform block) items. In split mode
// (PFSOFT_SERVER_SPLIT) a batch takes requests of one direction and any bandwidths up to 256: FFT
// passes per bandwidth group, then ONE split-precision DWT launch (dwt_split.cu) over every
// group's items. Completion is stamped by
// a host function queued behind the batch on its stream; the scheduler then returns the batch's
// arena range, frees the stream, and launches whatever waits -- batches of later requests run
// while earlier ones are still on the device.
//
// Locking: one mutex guards the queue, the request table and the statistics. No CUDA call is made
// while it is held, because the completion host function takes it and CUDA may wait for that
// function inside a launch.

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/pfsoft_b200.h"
#include "common.cuh"
#include "dwt.cuh"
#include "fft.cuh"
#include "serving.hpp"

using namespace pfsoft_dev;

namespace pfsoft_dev {
int tables_for(int B, cudaStream_t s, BandTables* out);   // api.cu
int launch_group(int dir, const BandTables& t, int T, double2** d_grids, double2** d_ws, const DwtGroup* d_group,
                 const DwtItem* d_items, int n_items, int* d_counter, int tpc, double2* const* h_coef,
                 double2* const* h_ws, cudaStream_t s);   // batch.cu
void group_items(int B, int T, int tpc, std::vector<DwtItem>& out);   // batch.cu
FftPassArgs group_pass_args(int dir, bool first, const BandTables& t, double2** grids, double2** ws);   // batch.cu
cudaError_t zero_nyquist_launch(double2** ws, int B, int T, cudaStream_t s);   // batch.cu
}  // namespace pfsoft_dev

namespace {

constexpr size_t kStageHeader = 128;   // DwtGroup, padded; pointer tables follow
constexpr int kMaxBatchLimit = 256;
constexpr int kMaxStreams = 16;
constexpr size_t kLatencyWindow = (size_t)1 << 20;   // latency samples kept (the most recent)

double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int fail(int status, const std::string& msg)
{
    set_last_error(msg.c_str());
    return status;
}

struct Batch;

struct Slot {
    cudaStream_t stream = nullptr;
    unsigned char* h_stage = nullptr;   // pinned: DwtGroup(s), [segments], then grid / coefficient / spectrum tables
    unsigned char* d_stage = nullptr;
    int* d_counter = nullptr;
    int* h_status = nullptr;            // split mode: mapped host flag a timed-out bounded wait sets
    int* d_status = nullptr;            // its device alias
    Batch* batch = nullptr;             // the batch on the device, or null
};

enum { kQueued = 0, kRunning = 1, kFinished = 2 };

struct Request {
    int dir = 0, B = 0;
    const double* in = nullptr;
    double* out = nullptr;
    cudaEvent_t ready = nullptr;   // input complete on the caller's stream (or null)
    double t_submit = 0, t_done = 0;
    int state = kQueued;
    int status = PFSOFT_OK;
};

struct Batch {
    pfsoft_server* srv = nullptr;
    int slot = -1;
    pfsoft_serving::BatchPlan plan;
    double t_done = 0;
    int status = PFSOFT_OK;
};

// transforms per CTA of the fused DWT for a batch of k transforms at bandwidth B
int tpc_for(int B, int k)
{
    const int N = 2 * B;
    int t = dwt_batch_transforms_per_cta(N <= 64 ? 64 : (N <= 128 ? 128 : 256));
    while (t > 1 && t > k) t >>= 1;
    return t;
}

}  // namespace

struct pfsoft_server {
    int device = 0;
    int max_batch = 16;
    bool split = false;          // PFSOFT_SERVER_SPLIT
    size_t stage_bytes = 0;
    cudaStream_t table_stream = nullptr;   // builds a bandwidth's tables at submission
    std::vector<Slot> slots;
    void* arena_base = nullptr;
    pfsoft_serving::Arena arena;
    pfsoft_serving::Scheduler sched;
    std::unordered_map<long long, Request> reqs;
    long long next_id = 1;
    std::vector<Batch*> finished;   // done on the device, not yet reaped
    std::vector<cudaEvent_t> dead_events;   // of cancelled requests; destroyed without the mutex
    // fused-DWT item lists per (B, k): scheduler thread only
    std::map<std::pair<int, int>, std::pair<DwtItem*, int> > items;
    std::mutex mu;
    std::condition_variable cv;
    bool stop = false, paused = false;
    int running = 0;   // batches on the device
    std::thread worker;
    // statistics since the last reset
    long long submitted = 0, completed = 0, cancelled = 0, rejected = 0, failed = 0, batches = 0, batched = 0;
    std::vector<double> lat_ms;   // ring of the last kLatencyWindow latencies
    size_t lat_next = 0;
    double t_first = -1, t_last = 0;
    int max_concurrent = 0;
};

namespace {

void CUDART_CB on_batch_done(void* p)   // host function: no CUDA calls in here
{
    Batch* b = static_cast<Batch*>(p);
    b->t_done = now_s();
    pfsoft_server* s = b->srv;
    int* flag = s->slots[b->slot].h_status;
    if (flag && *reinterpret_cast<volatile int*>(flag)) {   // the slot's next batch starts after the reap
        b->status = PFSOFT_ETIMEOUT;
        *reinterpret_cast<volatile int*>(flag) = 0;
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->finished.push_back(b);
    }
    s->cv.notify_all();
}

// Device item list of a (B, k) batch, built on first use.
int items_for(pfsoft_server* s, int B, int k, int tpc, const DwtItem** d_items, int* n)
{
    auto key = std::make_pair(B, k);
    auto it = s->items.find(key);
    if (it == s->items.end()) {
        std::vector<DwtItem> v;
        group_items(B, k, tpc, v);
        DwtItem* d = nullptr;
        cudaError_t e = cudaMalloc(&d, v.size() * sizeof(DwtItem));
        if (e == cudaSuccess) e = cudaMemcpy(d, v.data(), v.size() * sizeof(DwtItem), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            cudaFree(d);
            return fail(PFSOFT_ECUDA, std::string("server item list: ") + cudaGetErrorString(e));
        }
        it = s->items.emplace(key, std::make_pair(d, (int)v.size())).first;
    }
    *d_items = it->second.first;
    *n = it->second.second;
    return PFSOFT_OK;
}

// Split mode: batch b's requests grouped by bandwidth; FFT passes per group and one
// split-precision DWT launch over all groups (scheduler thread, mutex not held). Stage layout:
// DwtGroup[cap], segments[cap], then the grid / coefficient / spectrum pointer tables, members of
// a group contiguous.
int launch_split_batch(pfsoft_server* s, Batch* b, const std::vector<Request>& io)
{
    Slot& sl = s->slots[b->slot];
    const int dir = b->plan.dir, k = (int)b->plan.ids.size();
    const size_t cap = (size_t)s->max_batch;
    std::map<int, std::vector<int>, std::greater<int> > byB;
    for (int i = 0; i < k; ++i) byB[b->plan.Bs[i]].push_back(i);
    const size_t groups_bytes = cap * sizeof(DwtGroup), segs_bytes = cap * dwt_split_seg_bytes();
    const size_t tab_off = (groups_bytes + segs_bytes + 255) & ~size_t(255);
    double2** h_tab = reinterpret_cast<double2**>(sl.h_stage + tab_off);
    double2** d_tab = reinterpret_cast<double2**>(sl.d_stage + tab_off);
    DwtGroup* h_groups = reinterpret_cast<DwtGroup*>(sl.h_stage);
    const DwtGroup* d_groups = reinterpret_cast<const DwtGroup*>(sl.d_stage);
    std::vector<BandTables> tabs;
    std::vector<int> gidx, gB, gT, gbase;
    int pos = 0;
    for (const auto& kv : byB) {
        BandTables t;
        const int rc = tables_for(kv.first, sl.stream, &t);
        if (rc) return rc;
        const int g = (int)tabs.size();
        for (size_t m = 0; m < kv.second.size(); ++m) {
            const Request& r = io[kv.second[m]];
            const int p = pos + (int)m;
            h_tab[p] = reinterpret_cast<double2*>(const_cast<double*>(dir == 0 ? r.in : r.out));
            h_tab[cap + p] = reinterpret_cast<double2*>(const_cast<double*>(dir == 0 ? r.out : r.in));
            h_tab[2 * cap + p] = reinterpret_cast<double2*>(static_cast<char*>(s->arena_base) + b->plan.offset +
                                                              b->plan.offs[kv.second[m]]);
        }
        DwtGroup d;
        d.B = t.B;
        d.N = t.N;
        d.T = (int)kv.second.size();
        d.cosb = t.cosb;
        d.w = t.w;
        d.normf = t.normf;
        d.pw_sin = t.pw_sin;
        d.pw_cos = t.pw_cos;
        d.rc_cf = t.rc_cf;
        d.rc_f1 = t.rc_f1;
        d.X = d_tab + 2 * cap + pos;
        d.coeffs = d_tab + cap + pos;
        h_groups[g] = d;
        tabs.push_back(t);
        gidx.push_back(g);
        gB.push_back(t.B);
        gT.push_back(d.T);
        gbase.push_back(pos);
        pos += d.T;
    }
    std::vector<unsigned char> segs;
    const int n_items = dwt_split_segments(dir, gidx, gB, gT, segs);
    std::memcpy(sl.h_stage + groups_bytes, segs.data(), segs.size());
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < k && e == cudaSuccess; ++i)
        if (io[i].ready) e = cudaStreamWaitEvent(sl.stream, io[i].ready, 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(sl.d_stage, sl.h_stage, s->stage_bytes, cudaMemcpyHostToDevice, sl.stream);
    const int sign = dir == 0 ? -1 : +1;
    auto fft = [&](size_t g) -> cudaError_t {
        const FftPassArgs a = group_pass_args(dir, true, tabs[g], d_tab + gbase[g], d_tab + 2 * cap + gbase[g]);
        const FftPassArgs c = group_pass_args(dir, false, tabs[g], d_tab + gbase[g], d_tab + 2 * cap + gbase[g]);
        const int N = tabs[g].N;
        if (fft_fused_enabled(N) && fft_fused_chunk(a, c))
            return fft_fused_launch(sign, a, c, N, N, gT[g], nullptr, nullptr, nullptr, nullptr, nullptr,
                                    (long long)N * N * N + (long long)dwt_split_aux_elems(gB[g]), sl.stream);
        cudaError_t e2 = fft_pass_launch(nullptr, nullptr, a, N, sign, sl.stream, gT[g]);
        return e2 == cudaSuccess ? fft_pass_launch(nullptr, nullptr, c, N, sign, sl.stream, gT[g]) : e2;
    };
    for (size_t g = 0; g < tabs.size() && e == cudaSuccess; ++g) {
        double2** ws = d_tab + 2 * cap + gbase[g];
        double2** cf = d_tab + cap + gbase[g];
        if (dir == 0) {
            e = fft(g);
        } else {
            e = zero_nyquist_launch(ws, gB[g], gT[g], sl.stream);
        }
        if (e == cudaSuccess) e = dwt_split_scales(dir, gB[g], gT[g], ws, cf, tabs[g].w, sl.stream);
    }
    if (e == cudaSuccess)
        e = dwt_split_launch(dir, d_groups, sl.d_stage + groups_bytes, (int)tabs.size(), n_items, sl.d_status, sl.stream);
    for (size_t g = 0; dir == 1 && g < tabs.size() && e == cudaSuccess; ++g) e = fft(g);
    if (e == cudaSuccess) e = cudaLaunchHostFunc(sl.stream, on_batch_done, b);
    if (e != cudaSuccess) return fail(PFSOFT_ECUDA, std::string("server split batch: ") + cudaGetErrorString(e));
    return PFSOFT_OK;
}

// Launches batch b on its slot (scheduler thread, mutex not held).
int launch_batch(pfsoft_server* s, Batch* b, const std::vector<Request>& io)
{
    if (s->split) return launch_split_batch(s, b, io);
    Slot& sl = s->slots[b->slot];
    const int B = b->plan.B, k = (int)b->plan.ids.size(), dir = b->plan.dir;
    BandTables t;
    int rc = tables_for(B, sl.stream, &t);
    if (rc) return rc;
    const int tpc = tpc_for(B, k);
    const DwtItem* d_items = nullptr;
    int n_items = 0;
    if (B <= 128) {
        rc = items_for(s, B, k, tpc, &d_items, &n_items);
        if (rc) return rc;
    }
    const size_t cap = (size_t)s->max_batch;
    double2** h_tab = reinterpret_cast<double2**>(sl.h_stage + kStageHeader);
    double2** d_tab = reinterpret_cast<double2**>(sl.d_stage + kStageHeader);
    double2** h_grid = h_tab;
    double2** h_coef = h_tab + cap;
    double2** h_ws = h_tab + 2 * cap;
    for (int i = 0; i < k; ++i) {
        const double* in = io[i].in;
        double* out = io[i].out;
        h_grid[i] = reinterpret_cast<double2*>(const_cast<double*>(dir == 0 ? in : out));
        h_coef[i] = reinterpret_cast<double2*>(const_cast<double*>(dir == 0 ? out : in));
        h_ws[i] = reinterpret_cast<double2*>(static_cast<char*>(s->arena_base) + b->plan.offset + b->plan.offs[i]);
    }
    DwtGroup g;
    g.B = B;
    g.N = 2 * B;
    g.T = k;
    g.cosb = t.cosb;
    g.w = t.w;
    g.normf = t.normf;
    g.pw_sin = t.pw_sin;
    g.pw_cos = t.pw_cos;
    g.rc_cf = t.rc_cf;
    g.rc_f1 = t.rc_f1;
    g.X = d_tab + 2 * cap;
    g.coeffs = d_tab + cap;
    std::memcpy(sl.h_stage, &g, sizeof(g));
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < k && e == cudaSuccess; ++i)
        if (io[i].ready) e = cudaStreamWaitEvent(sl.stream, io[i].ready, 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(sl.d_stage, sl.h_stage, kStageHeader + 3 * cap * sizeof(double2*),
                                    cudaMemcpyHostToDevice, sl.stream);
    if (e != cudaSuccess) return fail(PFSOFT_ECUDA, std::string("server upload: ") + cudaGetErrorString(e));
    rc = launch_group(dir, t, k, d_tab, d_tab + 2 * cap, reinterpret_cast<const DwtGroup*>(sl.d_stage), d_items,
                      n_items, sl.d_counter, tpc, h_coef, h_ws, sl.stream);
    if (rc) return rc;
    e = cudaLaunchHostFunc(sl.stream, on_batch_done, b);
    if (e != cudaSuccess) return fail(PFSOFT_ECUDA, std::string("server completion hook: ") + cudaGetErrorString(e));
    return PFSOFT_OK;
}

// Marks the requests of a reaped or failed batch finished (mutex held).
void finish_batch(pfsoft_server* s, Batch* b, double t_done, int status)
{
    s->arena.release(b->plan.offset);
    if (b->slot >= 0) s->slots[b->slot].batch = nullptr;
    for (long long id : b->plan.ids) {
        auto it = s->reqs.find(id);
        if (it == s->reqs.end()) continue;
        Request& r = it->second;
        r.state = kFinished;
        r.status = status;
        r.t_done = t_done;
        if (status == PFSOFT_OK) {
            ++s->completed;
            const double ms = (t_done - r.t_submit) * 1e3;
            if (s->lat_ms.size() < kLatencyWindow)
                s->lat_ms.push_back(ms);
            else
                s->lat_ms[s->lat_next] = ms;
            s->lat_next = (s->lat_next + 1) % kLatencyWindow;
            s->t_last = std::max(s->t_last, t_done);
        } else {
            ++s->failed;
        }
    }
}

void worker_main(pfsoft_server* s)
{
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        // reap batches the device has finished
        for (Batch* b : s->finished) {
            finish_batch(s, b, b->t_done, b->status);
            --s->running;
            delete b;
        }
        if (!s->finished.empty()) {
            s->finished.clear();
            s->cv.notify_all();
        }
        if (s->stop) {
            for (const auto& p : s->sched.take_all()) {
                auto it = s->reqs.find(p.id);
                if (it != s->reqs.end()) {
                    it->second.state = kFinished;
                    it->second.status = PFSOFT_ECANCELED;
                    if (it->second.ready) s->dead_events.push_back(it->second.ready);
                    it->second.ready = nullptr;
                    ++s->cancelled;
                }
            }
            if (s->running == 0) break;
        }
        // form as many batches as there are free streams and arena space
        std::vector<std::pair<Batch*, std::vector<Request> > > todo;
        if (!s->paused && !s->stop) {
            for (size_t si = 0; si < s->slots.size(); ++si) {
                if (s->slots[si].batch) continue;
                pfsoft_serving::BatchPlan plan;
                if (!s->sched.next(s->arena, now_s(), &plan)) break;
                Batch* b = new Batch();
                b->srv = s;
                b->slot = (int)si;
                b->plan = plan;
                std::vector<Request> io;
                for (long long id : plan.ids) {
                    Request& r = s->reqs[id];
                    r.state = kRunning;
                    io.push_back(r);
                    r.ready = nullptr;   // destroyed by the launch below
                }
                s->slots[si].batch = b;
                ++s->running;
                ++s->batches;
                s->batched += (long long)plan.ids.size();
                s->max_concurrent = std::max(s->max_concurrent, s->running);
                todo.push_back(std::make_pair(b, io));
            }
        }
        std::vector<cudaEvent_t> dead;
        dead.swap(s->dead_events);
        if (!todo.empty() || !dead.empty()) {
            lk.unlock();
            for (cudaEvent_t ev : dead)
                if (ev) cudaEventDestroy(ev);
            std::vector<std::pair<Batch*, int> > failed;
            for (auto& bt : todo) {
                const int rc = launch_batch(s, bt.first, bt.second);
                if (rc != PFSOFT_OK) failed.push_back(std::make_pair(bt.first, rc));
                for (const Request& r : bt.second)
                    if (r.ready) cudaEventDestroy(r.ready);   // released once the waits are done
            }
            if (!failed.empty()) {
                // a batch whose launch failed part-way may still have work queued on its stream
                for (auto& f : failed) cudaStreamSynchronize(s->slots[f.first->slot].stream);
            }
            lk.lock();
            for (auto& f : failed) {
                finish_batch(s, f.first, now_s(), PFSOFT_ECUDA);
                --s->running;
                delete f.first;
            }
            if (!failed.empty()) s->cv.notify_all();
            continue;
        }
        s->cv.wait(lk);
    }
}

}  // namespace

extern "C" {

int pfsoft_server_create(size_t budget_bytes, int max_batch, int streams, pfsoft_server** out)
{
    return pfsoft_server_create_ex(budget_bytes, max_batch, streams, 0, out);
}

int pfsoft_server_create_ex(size_t budget_bytes, int max_batch, int streams, int flags, pfsoft_server** out)
{
    set_last_error("");
    if (!out) return fail(PFSOFT_EINVAL, "null output handle");
    *out = nullptr;
    if (max_batch < 1 || max_batch > kMaxBatchLimit) return fail(PFSOFT_EINVAL, "max_batch must be in [1, 256]");
    if (streams < 1 || streams > kMaxStreams) return fail(PFSOFT_EINVAL, "streams must be in [1, 16]");
    if (flags & ~PFSOFT_SERVER_SPLIT) return fail(PFSOFT_EINVAL, "unknown server flag");
    if (budget_bytes < pfsoft_workspace_bytes(1)) return fail(PFSOFT_EINVAL, "budget below one transform");
    pfsoft_server* s = new pfsoft_server();
    s->max_batch = max_batch;
    s->split = (flags & PFSOFT_SERVER_SPLIT) != 0;
    s->sched.set_max_batch(max_batch);
    s->sched.set_mixed(s->split);
    cudaError_t e = cudaGetDevice(&s->device);
    if (e == cudaSuccess && s->split) e = dwt_split_prepare();
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->table_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&s->arena_base, budget_bytes);
    s->arena.reset(e == cudaSuccess ? budget_bytes : 0, 256);
    s->slots.resize(streams);
    const size_t tables = 3 * (size_t)max_batch * sizeof(double2*);
    const size_t stage = s->split ? (((size_t)max_batch * (sizeof(DwtGroup) + dwt_split_seg_bytes()) + 255) & ~size_t(255)) + tables
                                  : kStageHeader + tables;
    s->stage_bytes = stage;
    for (auto& sl : s->slots) {
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void**>(&sl.h_stage), stage, cudaHostAllocDefault);
        if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&sl.d_stage), stage);
        if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&sl.d_counter), sizeof(int));
        if (e == cudaSuccess && s->split) e = cudaHostAlloc(reinterpret_cast<void**>(&sl.h_status), sizeof(int), cudaHostAllocMapped);
        if (e == cudaSuccess && s->split) {
            *sl.h_status = 0;
            e = cudaHostGetDevicePointer(reinterpret_cast<void**>(&sl.d_status), sl.h_status, 0);
        }
        if (e == cudaSuccess) std::memset(sl.h_stage, 0, stage);
    }
    if (e != cudaSuccess) {
        const int status = e == cudaErrorMemoryAllocation ? PFSOFT_ENOMEM : PFSOFT_ECUDA;
        const std::string msg = std::string("server setup: ") + cudaGetErrorString(e);
        for (auto& sl : s->slots) {
            if (sl.stream) cudaStreamDestroy(sl.stream);
            cudaFreeHost(sl.h_stage);
            cudaFree(sl.d_stage);
            cudaFree(sl.d_counter);
            cudaFreeHost(sl.h_status);
        }
        if (s->table_stream) cudaStreamDestroy(s->table_stream);
        cudaFree(s->arena_base);
        delete s;
        cudaGetLastError();
        return fail(status, msg);
    }
    s->worker = std::thread(worker_main, s);
    *out = s;
    return PFSOFT_OK;
}

int pfsoft_server_destroy(pfsoft_server* s)
{
    if (!s) return PFSOFT_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->worker.joinable()) s->worker.join();
    for (auto& sl : s->slots) {
        cudaStreamSynchronize(sl.stream);
        cudaStreamDestroy(sl.stream);
        cudaFreeHost(sl.h_stage);
        cudaFree(sl.d_stage);
        cudaFree(sl.d_counter);
        cudaFreeHost(sl.h_status);
    }
    for (auto& kv : s->items) cudaFree(kv.second.first);
    if (s->table_stream) cudaStreamDestroy(s->table_stream);
    for (cudaEvent_t ev : s->dead_events)
        if (ev) cudaEventDestroy(ev);
    cudaFree(s->arena_base);
    delete s;
    return PFSOFT_OK;
}

int pfsoft_server_submit(pfsoft_server* s, int direction, int B, const double* d_in, double* d_out, void* stream,
                         long long* id)
{
    if (!s || !id) return fail(PFSOFT_EINVAL, "null server or id");
    *id = 0;
    if (direction != 0 && direction != 1) return fail(PFSOFT_EINVAL, "direction must be 0 (DSOFT) or 1 (iDSOFT)");
    if (B < 1 || B > 512) return fail(PFSOFT_EINVAL, "bandwidth must be in [1, 512]");
    if (s->split && !dwt_split_supported(B)) return fail(PFSOFT_EINVAL, "a split-mode server takes bandwidths up to 256");
    if (!d_in || !d_out) return fail(PFSOFT_EINVAL, "null buffer");
    if ((reinterpret_cast<uintptr_t>(d_in) & 15) || (reinterpret_cast<uintptr_t>(d_out) & 15))
        return fail(PFSOFT_EINVAL, "buffers must be 16-byte aligned");
    // pfsoft_workspace_bytes includes the FFT counters; in split mode they follow the scale table
    const size_t bytes = pfsoft_workspace_bytes(B) + (s->split ? dwt_split_aux_elems(B) * sizeof(double2) : 0);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) return fail(PFSOFT_EBUSY, "server is shutting down");
        if (s->arena.footprint(bytes) > s->arena.capacity()) {
            ++s->rejected;
            return fail(PFSOFT_ENOMEM, "one transform of this bandwidth exceeds the server's HBM budget");
        }
    }
    // the bandwidth's constant tables are built here, at admission (once per device and
    // bandwidth, on the server's own stream), so that no batch waits for them and the request's
    // latency, counted from the end of this call, does not include them
    {
        BandTables t;
        const int rc = tables_for(B, s->table_stream, &t);
        if (rc) return rc;
    }
    cudaEvent_t ready = nullptr;
    cudaError_t e = cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(ready, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        if (ready) cudaEventDestroy(ready);
        return fail(PFSOFT_ECUDA, std::string("submit: ") + cudaGetErrorString(e));
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) {
            s->dead_events.push_back(ready);
            return fail(PFSOFT_EBUSY, "server is shutting down");
        }
        const long long rid = s->next_id++;
        Request r;
        r.dir = direction;
        r.B = B;
        r.in = d_in;
        r.out = d_out;
        r.ready = ready;
        r.t_submit = now_s();
        s->reqs[rid] = r;
        s->sched.push(pfsoft_serving::Pending{rid, direction, B, bytes, r.t_submit});
        ++s->submitted;
        if (s->t_first < 0) s->t_first = r.t_submit;
        *id = rid;
    }
    s->cv.notify_all();
    return PFSOFT_OK;
}

static int take_result(pfsoft_server* s, long long id)   // mutex held
{
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return fail(PFSOFT_EINVAL, "unknown request id");
    if (it->second.state != kFinished) return PFSOFT_EBUSY;
    const int st = it->second.status;
    s->reqs.erase(it);
    return st;
}

int pfsoft_server_poll(pfsoft_server* s, long long id)
{
    if (!s) return fail(PFSOFT_EINVAL, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    return take_result(s, id);
}

int pfsoft_server_wait(pfsoft_server* s, long long id, double timeout_s)
{
    if (!s) return fail(PFSOFT_EINVAL, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double>(std::max(0.0, timeout_s));
    for (;;) {
        auto it = s->reqs.find(id);
        if (it == s->reqs.end()) return fail(PFSOFT_EINVAL, "unknown request id");
        if (it->second.state == kFinished) return take_result(s, id);
        if (s->cv.wait_until(lk, deadline) == std::cv_status::timeout) {
            auto jt = s->reqs.find(id);
            if (jt != s->reqs.end() && jt->second.state == kFinished) return take_result(s, id);
            return PFSOFT_ETIMEOUT;
        }
    }
}

int pfsoft_server_cancel(pfsoft_server* s, long long id)
{
    if (!s) return fail(PFSOFT_EINVAL, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return fail(PFSOFT_EINVAL, "unknown request id");
    if (it->second.state != kQueued || !s->sched.cancel(id)) return PFSOFT_EBUSY;
    if (it->second.ready) s->dead_events.push_back(it->second.ready);
    it->second.ready = nullptr;
    it->second.state = kFinished;
    it->second.status = PFSOFT_ECANCELED;
    ++s->cancelled;
    s->cv.notify_all();
    return PFSOFT_OK;
}

int pfsoft_server_pause(pfsoft_server* s, int paused)
{
    if (!s) return fail(PFSOFT_EINVAL, "null server");
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->paused = paused != 0;
    }
    s->cv.notify_all();
    return PFSOFT_OK;
}

int pfsoft_server_drain(pfsoft_server* s, double timeout_s)
{
    if (!s) return fail(PFSOFT_EINVAL, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double>(std::max(0.0, timeout_s));
    while (!(s->sched.empty() && s->running == 0 && s->finished.empty())) {
        if (s->cv.wait_until(lk, deadline) == std::cv_status::timeout) {
            if (s->sched.empty() && s->running == 0 && s->finished.empty()) break;
            return PFSOFT_ETIMEOUT;
        }
    }
    return PFSOFT_OK;
}

int pfsoft_server_get_stats(pfsoft_server* s, pfsoft_server_stats* o)
{
    if (!s || !o) return fail(PFSOFT_EINVAL, "null server or output");
    std::lock_guard<std::mutex> lk(s->mu);
    std::memset(o, 0, sizeof(*o));
    o->submitted = s->submitted;
    o->completed = s->completed;
    o->cancelled = s->cancelled;
    o->rejected = s->rejected;
    o->failed = s->failed;
    o->batches = s->batches;
    o->mean_batch = s->batches ? (double)s->batched / (double)s->batches : 0.0;
    o->p50_ms = pfsoft_serving::quantile(s->lat_ms, 0.50);
    o->p99_ms = pfsoft_serving::quantile(s->lat_ms, 0.99);
    double sum = 0, mx = 0;
    for (double v : s->lat_ms) {
        sum += v;
        mx = std::max(mx, v);
    }
    o->mean_ms = s->lat_ms.empty() ? 0.0 : sum / (double)s->lat_ms.size();
    o->max_ms = mx;
    o->wall_s = (s->t_first >= 0 && s->t_last > s->t_first) ? s->t_last - s->t_first : 0.0;
    o->transforms_per_s = o->wall_s > 0 ? (double)s->completed / o->wall_s : 0.0;
    o->budget_bytes = s->arena.capacity();
    o->peak_bytes = s->arena.peak();
    o->max_concurrent_batches = s->max_concurrent;
    o->queued = (int)s->sched.pending();
    o->running = s->running;
    return PFSOFT_OK;
}

int pfsoft_server_reset_stats(pfsoft_server* s)
{
    if (!s) return fail(PFSOFT_EINVAL, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    s->submitted = s->completed = s->cancelled = s->rejected = s->failed = s->batches = s->batched = 0;
    s->lat_ms.clear();
    s->lat_next = 0;
    s->t_first = -1;
    s->t_last = 0;
    s->max_concurrent = s->running;
    s->arena.reset_peak();
    return PFSOFT_OK;
}

}  // extern "C"
