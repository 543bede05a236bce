// Discrete Wigner transform over beta (the DWT stage of DSOFT / iDSOFT), FP64 on CUDA cores.
#pragma once

#include <cuda_runtime.h>

#include <vector>

namespace pfsoft_dev {

// Per-bandwidth constant tables, built once on the device (tables_build) and cached.
// All doubles; N = 2B, beta_k = pi(2k+1)/(4B) (include/PFSOFTlib_headers/fn_dwt.hpp:155-159).
struct BandTables {
    int B = 0, N = 0;
    double* cosb = nullptr;     // cos(beta_k)                    [N]
    double* sinh = nullptr;     // sin(beta_k / 2)                [N]
    double* cosh = nullptr;     // cos(beta_k / 2)                [N]
    double* w = nullptr;        // quadrature weights w_B(k)      [N]   (fn_dwt.hpp:62-83)
    double* normf = nullptr;    // seed norm per order class      [B(B+1)/2] (fn_dwt.hpp:117-121)
    double2* twiddle = nullptr; // exp(-2 pi i t / N)             [N]
    double2* pw_sin = nullptr;  // sin(beta_k/2)^p as {mantissa, exponent}  [2B][N], p < 2B
    double2* pw_cos = nullptr;  // cos(beta_k/2)^p as {mantissa, exponent}  [2B][N]
    // recurrence coefficients of the step l -> l+1 for every order class and degree M <= l < B,
    // class (M, M') from rc_offset(B, M, M'): {c1, f1 f2} and f1      [rc_entries(B)]
    double2* rc_cf = nullptr;
    double* rc_f1 = nullptr;
    void* block = nullptr;      // single allocation holding all of the above
    double2* bluestein = nullptr;   // N with a prime factor above 16: the FFT's Bluestein table (own allocation)
};

// Entries of the recurrence-coefficient table before class (M, M'): classes run M = 0, 1, ...
// and M' = 0..M within M, each with B - M degrees.
__host__ __device__ __forceinline__ long long rc_offset(int B, int M, int Mp)
{
    const long long m = M;
    return (long long)(B + 1) * m * (m + 1) / 2 - m * (m + 1) * (2 * m + 1) / 6 + (long long)Mp * (B - M);
}
__host__ __device__ __forceinline__ long long rc_entries(int B) { return rc_offset(B, B, 0); }

size_t tables_bytes(int B);
// Carve the tables out of `mem` (tables_bytes(B) bytes, 256-byte aligned) and fill them.
cudaError_t tables_build(int B, void* mem, BandTables* t, cudaStream_t stream);

struct DwtArgs {
    int B, N;
    const double* cosb;
    const double* sinh;
    const double* cosh;
    const double* w;
    const double* normf;
    const double2* pw_sin;
    const double2* pw_cos;
    int team_warps;   // warps cooperating on one order class (1..4)
    const double2* rc_cf;   // recurrence coefficients (BandTables::rc_cf / rc_f1)
    const double* rc_f1;
    // Optional subset of order classes (ascending, so longest first): when set, the kernels run
    // classes[0 .. n_classes-1] only and leave every other class's outputs untouched.
    const int* classes;
    int n_classes;
    // Inverse only: also zero the Nyquist bins (row B or column B of X, which no order class
    // writes) in the kernel's tail, instead of a separate launch.
    int zero_nyquist;
};

// Arguments of the DWT launches over every order class of a bandwidth's tables.
DwtArgs dwt_args_for(const BandTables& t);

// nblocks <= 0 launches the persistent grid (all resident CTAs).
// Forward: X (beta-innermost spectrum, N^3) -> packed coefficients, scale pi/(2B^2).
cudaError_t dwt_forward_launch(const double2* X, double2* coeffs, const DwtArgs& a, int nblocks,
                               cudaStream_t stream);
// Inverse: packed coefficients -> X (all non-Nyquist beta columns), scale 2B^2/pi.
cudaError_t dwt_inverse_launch(const double2* coeffs, double2* X, const DwtArgs& a, int nblocks,
                               cudaStream_t stream);
// Zero the beta columns of the Nyquist bins (row == B or col == B) of X.
cudaError_t zero_nyquist_launch(double2* X, int B, cudaStream_t stream);

// Tuning: dir 0 = forward, 1 = inverse; cs 1 = all eight cases per warp, 2 = four cases per
// warp (warp pairs share the recurrence), 0 = default.
void dwt_set_case_split(int dir, int cs);

// ---- batched DWT over many transforms and bandwidths (dwt_batch.cu) -------------------------
// A group holds T transforms of one bandwidth; X[t] is transform t's beta-innermost spectrum
// (N^3) and coeffs[t] its packed coefficients. Forward reads X and writes coeffs, inverse the
// other way. A work item is one order class of a group for transforms t0 .. t0+nt-1.
struct DwtGroup {
    int B, N, T;
    const double* cosb;
    const double* w;
    const double* normf;
    const double2* pw_sin;
    const double2* pw_cos;
    const double2* rc_cf;   // recurrence coefficients (BandTables::rc_cf / rc_f1)
    const double* rc_f1;
    double2* const* X;
    double2* const* coeffs;
};

struct DwtItem {
    int group, cls, t0, nt;
};

// Transforms per CTA (1, 2 or 4) and the largest beta-column count the launch supports.
int dwt_batch_transforms_per_cta(int nmax);
size_t dwt_batch_smem_bytes(int direction, int tpc, int nmax);
// One persistent launch over all items; *d_counter must be 0 (the kernel hands out items from
// it). direction 0 = forward, 1 = inverse. nmax >= every group's N, nmax <= 256.
cudaError_t dwt_batch_launch(int direction, const DwtGroup* d_groups, const DwtItem* d_items, int n_items,
                             int* d_counter, int tpc, int nmax, cudaStream_t stream);

// Split-precision DWT on the tensor cores (dwt_split.cu) for groups whose bandwidth passes
// dwt_split_supported. A launch covers several groups of d_groups, described by segments
// (dwt_split_segments: group index, bandwidth and transform count of each); one persistent
// launch per direction; a bounded wait that ran out sets *d_status to 1.
bool dwt_split_supported(int B);
int dwt_split_segments(int direction, const std::vector<int>& group, const std::vector<int>& B,
                       const std::vector<int>& T, std::vector<unsigned char>& out);   // returns the item count
size_t dwt_split_seg_bytes();
cudaError_t dwt_split_prepare();   // kernel attributes; call once per device before any capture
// The split kernels read operand scales from a table of dwt_split_aux_elems(B) double2 that
// follows each transform's spectrum (N^3 double2) in its workspace; dwt_split_scales fills it
// (forward: from the spectra, after the FFT passes; inverse: from the coefficients), and the
// row scales of the generated operand. w: the group's quadrature weights.
size_t dwt_split_aux_elems(int B);
cudaError_t dwt_split_scales(int direction, int B, int T, double2* const* d_ws, const double2* const* d_coeffs,
                             const double* w, cudaStream_t stream);
cudaError_t dwt_split_launch(int direction, const DwtGroup* d_groups, const void* d_segs, int nseg, int n_items,
                             int* d_status, cudaStream_t stream);
// Test knob: when nonzero, every later split launch first waits up to `ns` nanoseconds on a
// barrier that nothing signals, before any MMA is issued, so that its bounded-wait exit runs.
void dwt_split_set_fail_ns(unsigned long long ns);

// Sets the detail string returned by pfsoft_last_error() on the calling thread.
void set_last_error(const char* msg);

// Team shape for a bandwidth: warps per class so that each lane owns at most 4 beta columns.
int dwt_team_warps(int N);

}  // namespace pfsoft_dev
