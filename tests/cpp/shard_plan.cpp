// Checks of the sharding plan (pfsoftlib_b200/csrc/shard.hpp): slabs tile the layers, every bin
// except the Nyquist row and column belongs to exactly one rank, classes are balanced, the plan is
// the same on every rank, and the exchange runs move every value to its place in both directions
// and both modes (direct scatter; pack, all-to-all, unpack), emulated here with P host buffers.
// Prints "ok" and exits 0 when every check holds.
#include <cstdio>
#include <set>
#include <vector>

#include "shard.hpp"

static int failures = 0;
#define CHECK(cond)                                                                      \
    do {                                                                                 \
        if (!(cond)) {                                                                   \
            std::fprintf(stderr, "%s:%d: check failed: %s\n", __FILE__, __LINE__, #cond); \
            ++failures;                                                                  \
        }                                                                                \
    } while (0)

using pfsoft_shard::Plan;
using pfsoft_shard::Run;

static void apply(const std::vector<Run>& runs, const std::vector<double>& src, std::vector<std::vector<double> >& dst)
{
    for (const Run& r : runs)
        for (int i = 0; i < r.len; ++i) dst[r.slot].at(r.dst_off + i) = src.at(r.src_off + i);
}

// The all-to-all: rank q's receive part from p is rank p's send part for q.
static std::vector<std::vector<double> > all_to_all(const std::vector<Plan>& plans, const std::vector<std::vector<double> >& send,
                                                    bool forward)
{
    const int P = (int)plans.size();
    std::vector<std::vector<double> > recv(P);
    for (int q = 0; q < P; ++q) {
        const std::vector<size_t> ro = pfsoft_shard::recv_offsets(plans[q], forward);
        recv[q].assign(ro[P], -1.0);
        for (int p = 0; p < P; ++p) {
            const std::vector<size_t> so = pfsoft_shard::send_offsets(plans[p], forward);
            CHECK(so[q + 1] - so[q] == ro[p + 1] - ro[p]);
            for (size_t i = 0; i < so[q + 1] - so[q]; ++i) recv[q][ro[p] + i] = send[p][so[q] + i];
        }
    }
    return recv;
}

static void check_exchange(int B, int P)
{
    std::vector<Plan> plans;
    for (int r = 0; r < P; ++r) plans.push_back(pfsoft_shard::make_plan(B, P, r));
    const int N = 2 * B;
    const Plan& p0 = plans[0];
    auto id = [&](int b, int k) { return (double)((long long)b * N + k); };

    // forward: slab spectra hold id(bin, global layer); owners must end with full columns
    std::vector<std::vector<double> > slab(P);
    for (int r = 0; r < P; ++r) {
        slab[r].assign(p0.slab_elems(r), 0.0);
        for (int b = 0; b < N * N; ++b)
            for (int kk = 0; kk < p0.nk[r]; ++kk) slab[r][(size_t)b * p0.nk[r] + kk] = id(b, p0.k0[r] + kk);
    }
    for (int mode = 0; mode < 2; ++mode) {
        std::vector<std::vector<double> > spec(P, std::vector<double>(p0.spectrum_elems(), -1.0));
        if (mode == 0) {
            for (int r = 0; r < P; ++r) apply(pfsoft_shard::make_runs(plans[r], pfsoft_shard::FWD_SCATTER), slab[r], spec);
        } else {
            std::vector<std::vector<double> > send(P);
            for (int r = 0; r < P; ++r) {
                send[r].assign(pfsoft_shard::send_offsets(plans[r], true)[P], -2.0);
                std::vector<std::vector<double> > one(1);
                one[0].swap(send[r]);
                apply(pfsoft_shard::make_runs(plans[r], pfsoft_shard::FWD_PACK), slab[r], one);
                one[0].swap(send[r]);
                for (double v : send[r]) CHECK(v >= 0);   // every send value written
            }
            std::vector<std::vector<double> > recv = all_to_all(plans, send, true);
            for (int q = 0; q < P; ++q) {
                std::vector<std::vector<double> > one(1);
                one[0].swap(spec[q]);
                apply(pfsoft_shard::make_runs(plans[q], pfsoft_shard::FWD_UNPACK), recv[q], one);
                one[0].swap(spec[q]);
            }
        }
        for (int b = 0; b < N * N; ++b) {
            const int q = p0.owner[b];
            for (int r = 0; r < P; ++r)
                for (int k = 0; k < N; ++k) {
                    const double v = spec[r][(size_t)b * N + k];
                    CHECK(r == q ? v == id(b, k) : v == -1.0);
                }
        }
    }

    // inverse: owners' spectra hold id(bin, layer) at their bins; slabs must end with their layers
    std::vector<std::vector<double> > spec(P, std::vector<double>(p0.spectrum_elems(), -3.0));
    for (int b = 0; b < N * N; ++b)
        if (p0.owner[b] >= 0)
            for (int k = 0; k < N; ++k) spec[p0.owner[b]][(size_t)b * N + k] = id(b, k);
    for (int mode = 0; mode < 2; ++mode) {
        std::vector<std::vector<double> > out(P);
        for (int r = 0; r < P; ++r) out[r].assign(p0.slab_elems(r), -1.0);
        if (mode == 0) {
            for (int q = 0; q < P; ++q) apply(pfsoft_shard::make_runs(plans[q], pfsoft_shard::INV_SCATTER), spec[q], out);
        } else {
            std::vector<std::vector<double> > send(P);
            for (int q = 0; q < P; ++q) {
                std::vector<std::vector<double> > one(1, std::vector<double>(pfsoft_shard::send_offsets(plans[q], false)[P], -2.0));
                apply(pfsoft_shard::make_runs(plans[q], pfsoft_shard::INV_PACK), spec[q], one);
                for (double v : one[0]) CHECK(v >= 0);
                send[q].swap(one[0]);
            }
            std::vector<std::vector<double> > recv = all_to_all(plans, send, false);
            for (int r = 0; r < P; ++r) {
                std::vector<std::vector<double> > one(1);
                one[0].swap(out[r]);
                apply(pfsoft_shard::make_runs(plans[r], pfsoft_shard::INV_UNPACK), recv[r], one);
                one[0].swap(out[r]);
            }
        }
        for (int r = 0; r < P; ++r)
            for (int b = 0; b < N * N; ++b)
                for (int kk = 0; kk < p0.nk[r]; ++kk) {
                    const double v = out[r][(size_t)b * p0.nk[r] + kk];
                    CHECK(p0.owner[b] >= 0 ? v == id(b, p0.k0[r] + kk) : v == -1.0);
                }
    }
}

int main()
{
    const int Bs[] = {1, 2, 3, 8, 16, 33, 64};
    const int Ps[] = {1, 2, 3, 4, 8};
    for (int B : Bs)
        for (int P : Ps) {
            const Plan p = pfsoft_shard::make_plan(B, P, 0);
            const int N = 2 * B;
            int covered = 0;
            for (int r = 0; r < P; ++r) {
                CHECK(p.k0[r] == covered);
                covered += p.nk[r];
            }
            CHECK(covered == N);
            std::set<int> seen;
            size_t nb = 0;
            int ncls = 0;
            double lo = 1e300, hi = 0;
            for (int r = 0; r < P; ++r) {
                for (size_t j = 0; j < p.bins[r].size(); ++j) {
                    const int b = p.bins[r][j];
                    CHECK(seen.insert(b).second);   // each bin once
                    CHECK(b / N != B && b % N != B);
                    CHECK(p.owner[b] == r && p.slot_of_bin[b] == (int)j);
                }
                nb += p.bins[r].size();
                ncls += (int)p.classes[r].size();
                for (size_t i = 1; i < p.classes[r].size(); ++i) CHECK(p.classes[r][i - 1] < p.classes[r][i]);
                lo = std::min(lo, p.load[r]);
                hi = std::max(hi, p.load[r]);
            }
            CHECK(nb == (size_t)(N - 1) * (N - 1));   // all but the Nyquist row and column
            CHECK(ncls == B * (B + 1) / 2);
            if (B >= 16) CHECK(hi <= 1.05 * lo + B + 1);   // balanced to within one class
            for (int rank = 1; rank < P; ++rank) {        // rank-independent
                const Plan q = pfsoft_shard::make_plan(B, P, rank);
                CHECK(q.bins == p.bins && q.k0 == p.k0 && q.classes == p.classes);
            }
            size_t sent = 0;
            for (int a = 0; a < P; ++a)
                for (int b = 0; b < P; ++b) sent += p.piece(a, b);
            CHECK(sent == (size_t)(N - 1) * (N - 1) * N);   // every bin column crosses once
            if (B <= 33) check_exchange(B, P);
        }
    if (failures) {
        std::fprintf(stderr, "%d check(s) failed\n", failures);
        return 1;
    }
    std::printf("ok\n");
    return 0;
}
