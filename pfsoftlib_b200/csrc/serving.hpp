// Host-side policy of the transform server (pfsoft_server_*): the workspace arena that admission
// is counted against, and the batch former. Plain C++ with no CUDA, so that the policy can be
// compiled and tested on its own.
//
// A request needs, besides its caller-owned input and output, one beta-innermost spectrum of
// (2B)^3 complex doubles on the device while it runs. The server reserves one arena of the HBM
// budget at start-up; a batch of k requests takes one contiguous range of it (the sum of their
// workspaces) and gives it back when the batch finishes. A request is admitted to the GPU when its
// batch fits; until then it waits in the queue.
#pragma once

#include <algorithm>
#include <cstddef>
#include <cmath>
#include <cstdint>
#include <deque>
#include <iterator>
#include <map>
#include <vector>

namespace pfsoft_serving {

// First-fit range allocator over [0, capacity) with coalescing of freed neighbours.
class Arena {
  public:
    explicit Arena(size_t capacity = 0, size_t align = 256) { reset(capacity, align); }

    void reset(size_t capacity, size_t align = 256)
    {
        align_ = align ? align : 1;
        capacity_ = capacity / align_ * align_;
        free_.clear();
        live_.clear();
        used_ = peak_ = 0;
        if (capacity_) free_[0] = capacity_;
    }

    // Offset of a range of at least `bytes`, or -1 when no free range is large enough.
    long long alloc(size_t bytes)
    {
        if (bytes == 0) bytes = 1;
        const size_t need = (bytes + align_ - 1) / align_ * align_;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < need) continue;
            const size_t off = it->first, len = it->second;
            free_.erase(it);
            if (len > need) free_[off + need] = len - need;
            live_[off] = need;
            used_ += need;
            peak_ = std::max(peak_, used_);
            return (long long)off;
        }
        return -1;
    }

    // Returns false for an offset that is not live.
    bool release(long long offset)
    {
        auto it = live_.find((size_t)offset);
        if (offset < 0 || it == live_.end()) return false;
        size_t off = it->first, len = it->second;
        live_.erase(it);
        used_ -= len;
        auto next = free_.lower_bound(off);
        if (next != free_.end() && off + len == next->first) {
            len += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == off) {
                prev->second += len;
                return true;
            }
        }
        free_[off] = len;
        return true;
    }

    // Bytes a request of `bytes` occupies (rounded up to the alignment).
    size_t footprint(size_t bytes) const { return (std::max<size_t>(bytes, 1) + align_ - 1) / align_ * align_; }
    size_t capacity() const { return capacity_; }
    size_t used() const { return used_; }
    size_t peak() const { return peak_; }
    void reset_peak() { peak_ = used_; }
    size_t largest_free() const
    {
        size_t m = 0;
        for (const auto& kv : free_) m = std::max(m, kv.second);
        return m;
    }
    size_t live_ranges() const { return live_.size(); }

  private:
    size_t align_ = 256, capacity_ = 0, used_ = 0, peak_ = 0;
    std::map<size_t, size_t> free_;   // offset -> length
    std::map<size_t, size_t> live_;
};

struct Pending {
    long long id;
    int dir;          // 0 forward (DSOFT), 1 inverse (iDSOFT)
    int B;
    size_t bytes;     // device workspace one transform needs
    double t_submit;  // seconds, any monotonic clock
};

struct BatchPlan {
    int dir = 0, B = 0;           // B: the bandwidth of the first request (all of them unless mixed)
    std::vector<long long> ids;   // FIFO order
    std::vector<int> Bs;          // bandwidth of each request
    std::vector<size_t> offs;     // workspace of each request, relative to `offset`
    long long offset = -1;        // arena range of the batch
    size_t stride = 0;            // workspace bytes of one request when all bandwidths are equal
};

// FIFO queue with batch forming: the next batch takes the oldest waiting request and up to
// max_batch - 1 later requests of the same direction and bandwidth (with mixed bandwidths on: of
// the same direction, any bandwidth), as many as the arena can hold. When even one of them does
// not fit, younger groups may go ahead (backfill), unless the oldest request has waited longer
// than `aging` seconds, in which case nothing else starts until memory frees up for it.
class Scheduler {
  public:
    Scheduler(int max_batch = 16, double aging = 0.05) : max_batch_(std::max(1, max_batch)), aging_(aging) {}

    void set_max_batch(int m) { max_batch_ = std::max(1, m); }
    int max_batch() const { return max_batch_; }
    void set_aging(double s) { aging_ = s; }
    void set_mixed(bool on) { mixed_ = on; }
    bool mixed() const { return mixed_; }

    void push(const Pending& p) { q_.push_back(p); }
    size_t pending() const { return q_.size(); }
    bool empty() const { return q_.empty(); }

    bool cancel(long long id)
    {
        for (auto it = q_.begin(); it != q_.end(); ++it)
            if (it->id == id) {
                q_.erase(it);
                return true;
            }
        return false;
    }

    // Removes and returns every waiting request (server shutdown).
    std::vector<Pending> take_all()
    {
        std::vector<Pending> v(q_.begin(), q_.end());
        q_.clear();
        return v;
    }

    // Forms the next batch that fits in the arena and allocates its range; false when none can
    // start now.
    bool next(Arena& arena, double now, BatchPlan* out)
    {
        std::vector<std::pair<int, int> > tried;
        bool first = true;
        for (size_t i = 0; i < q_.size(); ++i) {
            const Pending& head = q_[i];
            const std::pair<int, int> key(head.dir, mixed_ ? 0 : head.B);
            if (std::find(tried.begin(), tried.end(), key) != tried.end()) continue;
            tried.push_back(key);
            std::vector<size_t> members;
            for (size_t j = i; j < q_.size() && (int)members.size() < max_batch_; ++j)
                if (q_[j].dir == head.dir && (mixed_ || q_[j].B == head.B)) members.push_back(j);
            // prefix sums of the members' footprints: the first k members take sum[k] bytes
            std::vector<size_t> sum(members.size() + 1, 0);
            for (size_t m = 0; m < members.size(); ++m) sum[m + 1] = sum[m] + arena.footprint(q_[members[m]].bytes);
            for (size_t k = members.size(); k >= 1; --k) {
                const long long off = arena.alloc(sum[k]);
                if (off < 0) continue;
                out->dir = head.dir;
                out->B = head.B;
                out->offset = off;
                out->stride = arena.footprint(head.bytes);
                out->ids.clear();
                out->Bs.clear();
                out->offs.clear();
                for (size_t m = 0; m < k; ++m) {
                    out->ids.push_back(q_[members[m]].id);
                    out->Bs.push_back(q_[members[m]].B);
                    out->offs.push_back(sum[m]);
                }
                for (size_t m = k; m-- > 0;) q_.erase(q_.begin() + (long)members[m]);
                return true;
            }
            if (first && now - head.t_submit >= aging_) return false;
            first = false;
        }
        return false;
    }

  private:
    int max_batch_;
    double aging_;
    bool mixed_ = false;
    std::deque<Pending> q_;
};

// q-quantile (0 <= q <= 1) of a sample by the nearest-rank method; 0 for an empty sample.
inline double quantile(std::vector<double> v, double q)
{
    if (v.empty()) return 0.0;
    q = std::min(1.0, std::max(0.0, q));
    size_t rank = (size_t)std::ceil(q * (double)v.size());
    if (rank < 1) rank = 1;
    std::nth_element(v.begin(), v.begin() + (long)(rank - 1), v.end());
    return v[rank - 1];
}

}  // namespace pfsoft_serving
