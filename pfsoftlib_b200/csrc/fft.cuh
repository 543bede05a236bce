// Batched layer-wise 2D DFT passes (the reference's uzl_fftw_layer_wise_{DFT2,IDFT2}_grid3D,
// src/fftw_wrapper.cpp:47-173, re-designed for HBM): each pass is one 1D DFT direction over
// every beta layer, tiled so that one CTA transforms KB vectors, with the transpose to or from
// the beta-innermost spectrum layout fused into the load or store.
#pragma once

#include <cuda_runtime.h>

namespace pfsoft_dev {

constexpr int kFftMaxStages = 12;

// Element e of vector v in tile b lives at  base + v*sv + b*sb + e*se  (units of double2).
struct FftStrides {
    long long sv, sb, se;
};

struct FftPassArgs {
    int n;                       // transform length
    int nvec;                    // total vectors along the tiled index (k)
    int kb;                      // vectors per CTA
    int nstages;
    int radix[kFftMaxStages];
    int ns[kFftMaxStages];       // product of the radices of the earlier stages
    FftStrides src, dst;
    double scale;                // applied to the stored values (1 = none)
    const double2* twiddle;      // twiddle[t] = exp(-2*pi*i*t/n), t < n
    // batched passes: when set, transform z = blockIdx.z reads srcs[z] and writes dsts[z]
    const double2* const* srcs;
    double2* const* dsts;
    int coherent;                // first-stage loads through the coherent path (0: read-only path)
    // last-stage stores marked evict-first (st.global.cs): set by fft_pass_launch, whose output is
    // not read again before it has left L2; left 0 where another pass reads it through L2
    int stream_out;
    // lengths with a prime factor above 16 (fft_needs_bluestein): Bluestein's chirp tables
    // (fft_bluestein_fill); null keeps the direct O(R^2) stages for that factor
    const double2* bluestein;
};

// Bluestein's algorithm for a length n <= 512 whose largest prime factor exceeds 16: the DFT as a
// cyclic convolution of length M (the power of two >= 2n - 1) done with two radix-2 transforms in
// shared memory (X_k = w_k sum_e x_e w_e conj(w_(k-e)), w_e = exp(sign pi i e^2 / n)).
bool fft_needs_bluestein(int n);
int fft_bluestein_m(int n);
size_t fft_bluestein_elems(int n);   // double2 entries of the table
// The table, computed on the host in long double: w_e (e < n, sign -1), the bit-reversed length-M
// transforms of the chirp kernel for sign -1 and +1 (1/M included), exp(-2 pi i t / M) (t < M/2).
void fft_bluestein_fill(int n, double2* out);

// Radix plan for length n; returns the number of stages (0 if n cannot be planned).
int fft_plan_radices(int n, int* radix, int* ns);

// Launch one pass over a grid of (ceil(nvec/kb), ntiles, nz) CTAs. sign = -1 forward, +1 inverse.
// nz > 1 requires a.srcs / a.dsts (one base pointer per transform).
cudaError_t fft_pass_launch(const double2* src, double2* dst, const FftPassArgs& a, int ntiles, int sign,
                            cudaStream_t stream, int nz = 1);

size_t fft_pass_smem_bytes(const FftPassArgs& a);

// Both passes of one direction in one persistent launch, chunk by chunk over the layers, so that
// the second pass reads the first pass's output of a chunk from L2 (see fft.cu). p0 / p1: the
// passes as fft_pass_launch takes them (same length, plan and tile vectors; ntiles0 / ntiles1
// their tile counts), nz transforms (nz > 1: the pointer tables of both passes; nz == 1: the
// pointers src0..dst1). Each transform's workspace -- the second pass's source, `ws` when nz == 1 --
// holds kFftSyncBytes bytes of counters at double2 offset sync_off. Returns cudaErrorInvalidValue
// when the passes cannot be fused (fft_fused_chunk == 0).
constexpr int kFftSyncBytes = 4096;
int fft_fused_chunk(const FftPassArgs& p0, const FftPassArgs& p1);
// Whether transforms of length n use the fused launch (default off; pfsoft_tune_fft_fused sets it
// per length, or for every length with n <= 0).
bool fft_fused_enabled(int n);
void fft_set_fused(int n, int on);
cudaError_t fft_fused_launch(int sign, const FftPassArgs& p0, const FftPassArgs& p1, int ntiles0, int ntiles1, int nz,
                             const double2* src0, double2* dst0, const double2* src1, double2* dst1, double2* ws,
                             long long sync_off, cudaStream_t stream);

// Vectors per tile for length n: 8 (128 contiguous bytes on the transposed side) unless the
// ping-pong buffers of 8 vectors would leave a single CTA per SM, then 4; plans of three or more
// radix-8 stages (n = 512) run the in-place kernel with as many vectors as keep one butterfly
// per thread (4).
int fft_tile_vectors(int n);

}  // namespace pfsoft_dev
