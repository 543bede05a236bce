// Checks of the transform server's host policy (pfsoftlib_b200/csrc/serving.hpp): the workspace
// arena, batch forming, admission by footprint, backfill and aging, cancellation, and a random
// simulation of a serving run. Prints "ok" and exits 0 when every check holds.
#include <cstdio>
#include <algorithm>
#include <cstdlib>
#include <map>
#include <random>
#include <set>
#include <vector>

#include "serving.hpp"

using namespace pfsoft_serving;

static int failures = 0;
#define CHECK(cond)                                                          \
    do {                                                                     \
        if (!(cond)) {                                                       \
            std::fprintf(stderr, "%s:%d: check failed: %s\n", __FILE__, __LINE__, #cond); \
            ++failures;                                                      \
        }                                                                    \
    } while (0)

static void arena_basics()
{
    Arena a(1000, 100);
    CHECK(a.capacity() == 1000);
    const long long x = a.alloc(250);   // rounds to 300
    const long long y = a.alloc(100);
    const long long z = a.alloc(500);
    CHECK(x == 0 && y == 300 && z == 400);
    CHECK(a.used() == 900 && a.alloc(200) == -1);
    CHECK(a.release(y));
    CHECK(!a.release(y));                // not live any more
    CHECK(a.alloc(200) == -1);           // 100 + 100 free, not adjacent
    CHECK(a.release(x));                 // coalesces with the freed 100 after it
    CHECK(a.largest_free() == 400);
    CHECK(a.alloc(400) == 0);
    CHECK(a.release(0) && a.release(z));
    CHECK(a.used() == 0 && a.largest_free() == 1000 && a.live_ranges() == 0);
    CHECK(a.peak() == 900);
}

static Pending req(long long id, int dir, int B, size_t bytes, double t) { return Pending{id, dir, B, bytes, t}; }

static void batching()
{
    Arena a(10000, 1);
    Scheduler s(3, 1.0);
    s.push(req(1, 0, 16, 1000, 0));
    s.push(req(2, 1, 16, 1000, 0));
    s.push(req(3, 0, 16, 1000, 0));
    s.push(req(4, 0, 32, 2000, 0));
    s.push(req(5, 0, 16, 1000, 0));
    s.push(req(6, 0, 16, 1000, 0));
    BatchPlan p;
    CHECK(s.next(a, 0, &p));   // oldest key (fwd, 16): ids 1, 3, 5 (max_batch 3)
    CHECK(p.dir == 0 && p.B == 16 && p.ids == std::vector<long long>({1, 3, 5}) && p.stride == 1000);
    CHECK(s.next(a, 0, &p));   // next oldest: (inv, 16)
    CHECK(p.dir == 1 && p.ids == std::vector<long long>({2}));
    CHECK(s.next(a, 0, &p));
    CHECK(p.B == 32 && p.ids == std::vector<long long>({4}));
    CHECK(s.next(a, 0, &p));
    CHECK(p.ids == std::vector<long long>({6}));
    CHECK(!s.next(a, 0, &p) && s.empty());
    CHECK(a.used() == 7000);
}

static void admission_and_backfill()
{
    // room for 2.5 transforms of 1000: a batch of 4 shrinks to 2
    Arena a(2500, 1);
    Scheduler s(4, 0.5);
    for (int i = 1; i <= 4; ++i) s.push(req(i, 0, 64, 1000, 0));
    BatchPlan p;
    CHECK(s.next(a, 0.0, &p) && p.ids.size() == 2);
    const long long off = p.offset;
    // the oldest (id 3, 1000) no longer fits, a small younger request backfills
    s.push(req(5, 0, 8, 400, 0.1));
    CHECK(s.next(a, 0.2, &p) && p.ids == std::vector<long long>({5}));
    s.push(req(6, 0, 8, 400, 0.3));
    // aging: the oldest has now waited 0.6 s >= 0.5 s, nothing else may start
    CHECK(!s.next(a, 0.6, &p));
    CHECK(a.release(off));
    CHECK(s.next(a, 0.7, &p) && p.ids == std::vector<long long>({3, 4}));
    CHECK(s.next(a, 0.7, &p) == false);   // 6 does not fit: 2000 + 400 live, 100 free
    CHECK(s.pending() == 1);
}

// Mixed bandwidths (split mode): a batch takes requests of one direction and any bandwidths, each
// with its own workspace size at its own offset inside the batch's range.
static void mixed_batches()
{
    Arena a(10000, 1);
    Scheduler s(3, 1.0);
    s.set_mixed(true);
    s.push(req(1, 0, 16, 1000, 0));
    s.push(req(2, 1, 20, 1500, 0));
    s.push(req(3, 0, 32, 2000, 0));
    s.push(req(4, 0, 17, 500, 0));
    s.push(req(5, 0, 16, 1000, 0));
    BatchPlan p;
    CHECK(s.next(a, 0, &p));   // direction 0, oldest three: 1, 3, 4
    CHECK(p.dir == 0 && p.ids == std::vector<long long>({1, 3, 4}));
    CHECK(p.Bs == std::vector<int>({16, 32, 17}));
    CHECK(p.offs == std::vector<size_t>({0, 1000, 3000}) && p.offset == 0 && a.used() == 3500);
    CHECK(s.next(a, 0, &p) && p.dir == 1 && p.ids == std::vector<long long>({2}) && p.offset == 3500);
    // room for 5000 more: request 5 alone
    CHECK(s.next(a, 0, &p) && p.ids == std::vector<long long>({5}) && p.offs == std::vector<size_t>({0}));
    CHECK(s.empty());
    // a batch that does not fit whole shrinks to the prefix that does
    Arena b(2550, 1);
    s.push(req(6, 0, 16, 1000, 0));
    s.push(req(7, 0, 64, 1500, 0));
    s.push(req(8, 0, 8, 100, 0));
    CHECK(s.next(b, 0, &p) && p.ids == std::vector<long long>({6, 7}) && b.used() == 2500);
}

static void cancel_and_shutdown()
{
    Scheduler s(8, 1.0);
    for (int i = 1; i <= 5; ++i) s.push(req(i, i & 1, 16, 10, 0));
    CHECK(s.cancel(3) && !s.cancel(3) && !s.cancel(99));
    Arena a(1000, 1);
    BatchPlan p;
    CHECK(s.next(a, 0, &p) && p.ids == std::vector<long long>({1, 5}));
    const auto rest = s.take_all();
    CHECK(rest.size() == 2 && s.empty());
}

static void quantiles()
{
    std::vector<double> v;
    for (int i = 1; i <= 100; ++i) v.push_back(101 - i);
    CHECK(quantile(v, 0.5) == 50 && quantile(v, 0.99) == 99 && quantile(v, 1.0) == 100 && quantile(v, 0.0) == 1);
    CHECK(quantile(std::vector<double>(), 0.5) == 0);
    CHECK(quantile(std::vector<double>{7}, 0.99) == 7);
}

// A serving run in simulated time: random arrivals of mixed bandwidths, a fixed number of
// streams, batch time proportional to its work. Every request runs exactly once, never with more
// than the budget in use, and batches hold one (direction, bandwidth).
static void simulation()
{
    std::mt19937_64 rng(7);
    const int bws[] = {8, 16, 32, 48, 64};
    const size_t budget = 40 * 64ull * 64 * 64;
    Arena a(budget, 256);
    Scheduler s(8, 0.02);
    struct Run {
        double end;
        BatchPlan p;
    };
    std::vector<Run> running;
    const int streams = 3, total = 2000;
    std::set<long long> seen;
    std::map<long long, std::pair<int, int> > key;
    int submitted = 0;
    double t = 0;
    size_t max_used = 0;
    while ((int)seen.size() < total) {
        // arrivals
        if (submitted < total && std::uniform_real_distribution<double>(0, 1)(rng) < 0.6) {
            const int B = bws[rng() % 5];
            const int dir = (int)(rng() & 1);
            s.push(req(++submitted, dir, B, (size_t)8 * B * B * B, t));
            key[submitted] = std::make_pair(dir, B);
        }
        // completions
        for (size_t i = 0; i < running.size();) {
            if (running[i].end <= t) {
                CHECK(a.release(running[i].p.offset));
                running.erase(running.begin() + (long)i);
            } else {
                ++i;
            }
        }
        // launches
        BatchPlan p;
        while ((int)running.size() < streams && s.next(a, t, &p)) {
            CHECK(!p.ids.empty() && (int)p.ids.size() <= 8);
            for (long long id : p.ids) {
                CHECK(seen.insert(id).second);
                CHECK(key[id] == std::make_pair(p.dir, p.B));
            }
            running.push_back(Run{t + 1e-3 * p.ids.size() * p.B / 8.0, p});
        }
        max_used = std::max(max_used, a.used());
        CHECK(a.used() <= budget);
        t += 1e-4;
        if (t > 1000) break;
    }
    CHECK((int)seen.size() == total);
    CHECK(max_used > budget / 4);   // the arena was really shared
}

int main()
{
    arena_basics();
    batching();
    mixed_batches();
    admission_and_backfill();
    cancel_and_shutdown();
    quantiles();
    simulation();
    if (failures) {
        std::fprintf(stderr, "%d check(s) failed\n", failures);
        return 1;
    }
    std::printf("ok\n");
    return 0;
}
