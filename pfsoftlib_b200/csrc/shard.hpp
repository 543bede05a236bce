// Plan of one SO(3) transform sharded over P ranks (host code; compiles without nvcc).
//
// The layer-wise FFT is independent per beta layer and the DWT per order class
// (src/fn_dsoft.cpp:214 splits the DWT over the classes too), so
//   * rank p owns the beta layers k0[p] .. k0[p] + nk[p] - 1 of the grid (and runs the FFT
//     passes on that slab), and
//   * rank q owns a set of order classes, balanced by their work (B - M degrees each, longest
//     first to the least loaded rank), and runs their DWT.
// Between the two, one exchange moves every FFT bin column: in the forward direction rank p
// sends, for each bin of rank q's classes, the nk[p] values of its slab; rank q assembles full
// beta columns. The inverse moves the same pieces the other way. The Nyquist bins (row or
// column B) belong to no class; the inverse zeroes them on every slab.
//
// Layouts (complex values):
//   slab grid       [nk][N][N]   layers k0 .. k0+nk-1 of the (2B)^3 grid, as in the grid
//   slab spectrum   [N][N][nk]   bin (row, col) = (gamma frequency, alpha frequency), beta inner
//   spectrum        [N][N][N]    the full beta-innermost spectrum; a rank fills only its bins
//   send / receive  by peer rank in rank order; within peer q, bins in q's (resp. this rank's)
//                   bin order, each with the layers of the slab that owns them
// Every data movement of the exchange is a list of contiguous runs (Run), built here once.
#pragma once

#include <math.h>   // fma for the device helpers when compiled by a plain host compiler

#include <algorithm>
#include <cstddef>
#include <vector>

#include "common.cuh"

namespace pfsoft_shard {

constexpr int kMaxRanks = 64;

// Run kinds: forward / inverse x (direct stores into each peer's buffer | pack into this rank's
// send buffer | unpack this rank's receive buffer).
enum RunKind { FWD_SCATTER, FWD_PACK, FWD_UNPACK, INV_SCATTER, INV_PACK, INV_UNPACK, RUN_KINDS };

// Copy len values from src + src_off to (destination slot) + dst_off.
struct Run {
    long long src_off, dst_off;
    int slot, len;
};

struct Plan {
    int B = 0, N = 0, P = 1, rank = 0;
    std::vector<int> k0, nk;                    // layer slab of each rank
    std::vector<std::vector<int> > classes;     // order classes of each rank, ascending (longest first)
    std::vector<std::vector<int> > bins;        // bins (row * N + col) of those classes' cases
    std::vector<double> load;                   // work of each rank's classes
    std::vector<int> owner;                     // rank owning each bin, -1 for the Nyquist bins
    std::vector<int> slot_of_bin;               // index of each bin in its owner's bin list

    // complex values that the slab of rank `layers_of` holds of the bins of rank `bins_of`: what
    // moves from layers_of to bins_of in the forward exchange and back in the inverse
    size_t piece(int layers_of, int bins_of) const { return bins[bins_of].size() * (size_t)nk[layers_of]; }
    size_t slab_elems(int r) const { return (size_t)nk[r] * N * N; }
    size_t spectrum_elems() const { return (size_t)N * N * N; }
};

inline Plan make_plan(int B, int P, int rank)
{
    Plan p;
    p.B = B;
    p.N = 2 * B;
    p.P = P;
    p.rank = rank;
    p.k0.resize(P);
    p.nk.resize(P);
    for (int r = 0; r < P; ++r) {   // contiguous slabs, the first N % P ranks one layer more
        const int base = p.N / P, extra = p.N % P;
        p.nk[r] = base + (r < extra ? 1 : 0);
        p.k0[r] = r * base + std::min(r, extra);
    }
    p.classes.assign(P, std::vector<int>());
    p.bins.assign(P, std::vector<int>());
    p.load.assign(P, 0.0);
    p.owner.assign((size_t)p.N * p.N, -1);
    p.slot_of_bin.assign((size_t)p.N * p.N, -1);
    const int ncls = pfsoft_dev::num_classes(B);
    for (int c = 0; c < ncls; ++c) {   // ascending class index = descending work
        int M, Mp;
        pfsoft_dev::class_orders(c, M, Mp);
        const double w = (double)(B - M) + 1.0;
        int best = 0;
        for (int r = 1; r < P; ++r)
            if (p.load[r] < p.load[best]) best = r;
        p.load[best] += w;
        p.classes[best].push_back(c);
        const int nc = pfsoft_dev::class_case_count(M, Mp);
        for (int q = 0; q < nc; ++q) {
            const pfsoft_dev::PairCase pc = pfsoft_dev::class_case(M, Mp, q, p.N);
            const int b = pc.row * p.N + pc.col;
            p.owner[b] = best;
            p.slot_of_bin[b] = (int)p.bins[best].size();
            p.bins[best].push_back(b);
        }
    }
    return p;
}

// Offsets of each peer's part in this rank's send (resp. receive) buffer for a direction.
inline std::vector<size_t> send_offsets(const Plan& p, bool forward)
{
    std::vector<size_t> off(p.P + 1, 0);
    for (int r = 0; r < p.P; ++r) off[r + 1] = off[r] + (forward ? p.piece(p.rank, r) : p.piece(r, p.rank));
    return off;
}

inline std::vector<size_t> recv_offsets(const Plan& p, bool forward)
{
    std::vector<size_t> off(p.P + 1, 0);
    for (int r = 0; r < p.P; ++r) off[r + 1] = off[r] + (forward ? p.piece(r, p.rank) : p.piece(p.rank, r));
    return off;
}

// The runs of one kind for this rank (Plan::rank). Scatter runs address each peer's buffer
// (slot = peer); pack and unpack runs address a single buffer (slot 0).
inline std::vector<Run> make_runs(const Plan& p, RunKind kind)
{
    std::vector<Run> runs;
    const int me = p.rank, N = p.N;
    const long long nkm = p.nk[me];
    switch (kind) {
        case FWD_SCATTER:
        case FWD_PACK: {   // my slab spectrum -> each owner's spectrum (or my send buffer)
            if (nkm == 0) break;
            const std::vector<size_t> so = send_offsets(p, true);
            for (int b = 0; b < N * N; ++b) {
                const int q = p.owner[b];
                if (q < 0) continue;
                Run r;
                r.src_off = (long long)b * nkm;
                r.len = (int)nkm;
                if (kind == FWD_SCATTER) {
                    r.slot = q;
                    r.dst_off = (long long)b * N + p.k0[me];
                } else {
                    r.slot = 0;
                    r.dst_off = (long long)so[q] + (long long)p.slot_of_bin[b] * nkm;
                }
                runs.push_back(r);
            }
            break;
        }
        case FWD_UNPACK: {   // receive buffer (by source slab) -> my spectrum
            const std::vector<size_t> ro = recv_offsets(p, true);
            for (int src = 0; src < p.P; ++src) {
                if (p.nk[src] == 0) continue;
                for (size_t j = 0; j < p.bins[me].size(); ++j) {
                    Run r;
                    r.src_off = (long long)ro[src] + (long long)j * p.nk[src];
                    r.dst_off = (long long)p.bins[me][j] * N + p.k0[src];
                    r.slot = 0;
                    r.len = p.nk[src];
                    runs.push_back(r);
                }
            }
            break;
        }
        case INV_SCATTER:
        case INV_PACK: {   // my spectrum -> each slab owner's slab spectrum (or my send buffer)
            const std::vector<size_t> so = send_offsets(p, false);
            for (size_t j = 0; j < p.bins[me].size(); ++j) {
                const int b = p.bins[me][j];
                for (int dst = 0; dst < p.P; ++dst) {
                    if (p.nk[dst] == 0) continue;
                    Run r;
                    r.src_off = (long long)b * N + p.k0[dst];
                    r.len = p.nk[dst];
                    if (kind == INV_SCATTER) {
                        r.slot = dst;
                        r.dst_off = (long long)b * p.nk[dst];
                    } else {
                        r.slot = 0;
                        r.dst_off = (long long)so[dst] + (long long)j * p.nk[dst];
                    }
                    runs.push_back(r);
                }
            }
            break;
        }
        case INV_UNPACK: {   // receive buffer (by source class owner) -> my slab spectrum
            if (nkm == 0) break;
            const std::vector<size_t> ro = recv_offsets(p, false);
            for (int src = 0; src < p.P; ++src)
                for (size_t j = 0; j < p.bins[src].size(); ++j) {
                    Run r;
                    r.src_off = (long long)ro[src] + (long long)j * nkm;
                    r.dst_off = (long long)p.bins[src][j] * nkm;
                    r.slot = 0;
                    r.len = (int)nkm;
                    runs.push_back(r);
                }
            break;
        }
        default:
            break;
    }
    return runs;
}

}  // namespace pfsoft_shard
