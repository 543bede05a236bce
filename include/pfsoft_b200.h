/*
 * pfsoft_b200 -- C ABI of the B200 SO(3) Fourier transform engine (DSOFT / iDSOFT).
 *
 * Drop-in boundary for PFSOFTlib's hot path. Every entry point takes plain pointers and
 * sizes; `stream` is a cudaStream_t passed as void* (NULL = the legacy default stream).
 * All functions return a pfsoft_status; pfsoft_last_error() gives the detail of the last
 * failure on the calling thread. Nothing here exits the process: where the reference prints a
 * warning and returns (src/fn_dsoft.cpp:82-94, src/fn_idsoft.cpp:78-90 via
 * cmake_aux/compiler_config.hpp.in:112-120) these functions return PFSOFT_EINVAL.
 *
 * Layouts (N = 2B, complex values as interleaved {re, im} doubles):
 *   grid    N*N*N complex; element (row, col, lay) at (lay*N + col)*N + row, the layout of the
 *           reference's grid3D<complex<double>> (include/PFSOFTlib_headers/grid3D_cx.hpp:293-303).
 *   coeffs  B(4B^2-1)/3 complex; degree l starts at l(4l^2-1)/3 and holds a column-major
 *           (2l+1)x(2l+1) block, row index M, column index M', a negative order M stored at
 *           2l+1+M -- the storage of DSOFTFourierCoefficients
 *           (src/dsoft_fourier_coefficients.cpp:48-57, :80-89), packed contiguously.
 *
 * First use of a bandwidth on a device builds its constant tables (one cudaMalloc and a few
 * small kernels, then a stream synchronisation); make that first call before any stream
 * capture. Later calls for the same bandwidth allocate nothing. The tables stay until exit:
 * about 11 MB at B = 128, 77 MB at B = 256, 575 MB at B = 512 per bandwidth and device.
 */
#ifndef PFSOFT_B200_H
#define PFSOFT_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum pfsoft_status {
    PFSOFT_OK = 0,
    PFSOFT_EINVAL = 1,   /* bad argument (size, pointer, bandwidth mismatch) */
    PFSOFT_ENOMEM = 2,   /* device or pinned allocation failed / budget exceeded */
    PFSOFT_ETIMEOUT = 3, /* a bounded wait ran out */
    PFSOFT_ECUDA = 4,    /* a CUDA runtime call failed */
    PFSOFT_EBUSY = 5,    /* a resource is in use (serving: request still queued or running) */
    PFSOFT_ECANCELED = 6 /* serving: the request was cancelled before it reached the GPU */
} pfsoft_status;

const char* pfsoft_status_string(int status);
/* Detail of the most recent failure on this thread ("" if none). */
const char* pfsoft_last_error(void);
/* Library version as MAJOR*10000 + MINOR*100 + PATCH. */
int pfsoft_version(void);

/* Sizes. */
size_t pfsoft_coef_count(int B);            /* B(4B^2-1)/3 complex values */
size_t pfsoft_grid_bytes(int B);            /* (2B)^3 * 16 */
size_t pfsoft_workspace_bytes(int B);       /* device scratch for one transform: (2B)^3 * 16 + 4096 */

/* ---- Forward / inverse transforms on device-resident data (stream ordered) -------------
 * pfsoft_cuda_dsoft replaces pfsoft::FourierTransforms::DSOFT
 *   (include/PFSOFTlib_headers/fn_fourier_transforms.hpp:75, src/fn_dsoft.cpp:76).
 *   d_grid is not modified (the reference takes the grid by value). d_coeffs receives all
 *   B(4B^2-1)/3 coefficients. d_workspace: pfsoft_workspace_bytes(B) bytes of device memory,
 *   or NULL to use a library-owned buffer (allocated on first use, then reused; calls that
 *   share it are serialised on `stream` order only, so do not pass NULL from two streams).
 * pfsoft_cuda_idsoft replaces pfsoft::FourierTransforms::IDSOFT
 *   (fn_fourier_transforms.hpp:78, src/fn_idsoft.cpp:72). Every grid value is written; the
 *   Nyquist bins (row or col order == B), which the reference leaves as it found them, are
 *   synthesised from zero, i.e. the result the reference gives on a fresh grid.
 */
int pfsoft_cuda_dsoft(const double* d_grid, int B, double* d_coeffs, void* d_workspace,
                      size_t workspace_bytes, void* stream);
int pfsoft_cuda_idsoft(const double* d_coeffs, int B, double* d_grid, void* d_workspace,
                       size_t workspace_bytes, void* stream);

/* pfsoft_cuda_dsoft_noalloc has no counterpart in the reference. It is pfsoft_cuda_dsoft for
 * callers that cannot allocate device memory (a framework-owned, capped memory pool; a hard
 * per-process memory limit; a loop that must not take cudaMalloc's locks or cudaFree's device
 * synchronisation): it makes no allocation at all and uses a scratch array that the library
 * holds in device memory from load to exit (4.31 MiB per GPU). Limit: bandwidth B <= 32; a
 * larger B returns PFSOFT_EINVAL. The first call on a device looks up that array's device
 * address and builds the tables for B in it; make that first call before any stream capture.
 * All calls on a device share the array, so calls that overlap on the GPU race; nothing in it
 * has to start at zero. Same layouts and results as pfsoft_cuda_dsoft. */
int pfsoft_cuda_dsoft_noalloc(const double* d_grid, int B, double* d_coeffs, void* stream);

/* ---- Batches of transforms, uneven bandwidths ------------------------------------------------
 * No counterpart in the reference (which transforms one grid per call). A plan groups `count`
 * transforms by bandwidth; each execution runs batched FFT passes per bandwidth and ONE
 * persistent DWT launch over every (bandwidth, order class, transform block) item, longest
 * first, in which one on-chip Wigner recurrence serves up to `transforms_per_cta` transforms
 * (0 = default: 4 for B <= 64, 2 above). Bandwidths up to 128 share the fused FP64 launch;
 * larger ones use the per-transform FP64 DWT (or the split launch, below). The sequence is captured once into a CUDA graph and replayed
 * (PFSOFT_BATCH_NO_GRAPH disables the graph). The plan owns one spectrum workspace per
 * transform (pfsoft_batch_workspace_bytes). Pointer tables are host arrays of `count` device
 * pointers in the caller's order; every buffer has the single-transform layouts above. Stream
 * ordered. Calls on one plan are serialised by the plan.
 * PFSOFT_BATCH_SPLIT runs the DWT of the bandwidths that pfsoft_split_supported() accepts
 * (1 <= B <= 256) on the tensor cores instead, all of them in one launch per direction: the FP64
 * Wigner rows and FP64 data are cut into six signed 8-bit digit planes, multiplied exactly
 * (8-bit x 8-bit products summed in 32-bit integers) and combined in FP64; relative L2 error
 * about 1e-13 against the FP64 path. Two transforms of one bandwidth share each generated Wigner
 * tile. pfsoft_batch_status reports PFSOFT_ETIMEOUT if a bounded wait inside that kernel ever ran
 * out (it synchronises the device). */
#define PFSOFT_BATCH_NO_GRAPH 1
#define PFSOFT_BATCH_SPLIT 2
typedef struct pfsoft_batch pfsoft_batch;
int pfsoft_split_supported(int B);
int pfsoft_batch_status(pfsoft_batch* batch);
int pfsoft_batch_create(const int* bandwidths, int count, int transforms_per_cta, int flags, pfsoft_batch** out);
int pfsoft_batch_destroy(pfsoft_batch* batch);
size_t pfsoft_batch_workspace_bytes(const pfsoft_batch* batch);
int pfsoft_batch_transforms_per_cta(const pfsoft_batch* batch);
int pfsoft_batch_dsoft(pfsoft_batch* batch, const double* const* d_grids, double* const* d_coeffs, void* stream);
int pfsoft_batch_idsoft(pfsoft_batch* batch, const double* const* d_coeffs, double* const* d_grids, void* stream);

/* ---- Host-resident drop-in (synchronous) ---------------------------------------------------
 * The same transforms on host buffers: copy in, transform, copy out, wait. Pinned host
 * buffers (cudaHostAlloc) make the copies asynchronous DMA; pageable ones work too.
 * Calls from different host threads run concurrently, each with its own device staging buffers
 * and stream (a per-device pool, grown on demand and kept until exit), so one call's
 * device-to-host copy can overlap another's host-to-device copy. */
int pfsoft_dsoft_host(const double* h_grid, int B, double* h_coeffs);
int pfsoft_idsoft_host(const double* h_coeffs, int B, double* h_grid);

/* ---- FFT boundary ------------------------------------------------------------------------
 * Replace the reference's internal C ABI uzl_fftw_layer_wise_DFT2_grid3D /
 * uzl_fftw_layer_wise_IDFT2_grid3D (include/PFSOFTlib_headers/fftw_wrapper.hpp:31-32,
 * src/fftw_wrapper.cpp:47-173): an in-place 2D DFT of each of `lays` layers of cols x rows
 * complex values (rows contiguous), exp(-i..) for DFT2 and exp(+i..) for IDFT2, every value
 * multiplied by `scale` (1.0 = unnormalised, as FFTW). `threads` of the reference has no
 * counterpart. */
int pfsoft_cuda_layer_wise_dft2(int cols, int rows, int lays, double* d_arr, double scale, void* stream);
int pfsoft_cuda_layer_wise_idft2(int cols, int rows, int lays, double* d_arr, double scale, void* stream);
/* The same on a host array (grid3D::layer_wise_DFT2/IDFT2, grid3D_cx.hpp:309-427): copy in,
 * transform, copy out, wait. */
int pfsoft_layer_wise_dft2_host(int cols, int rows, int lays, double* h_arr, double scale);
int pfsoft_layer_wise_idft2_host(int cols, int rows, int lays, double* h_arr, double scale);

/* ---- Discrete Wigner transform helpers ---------------------------------------------------
 * pfsoft_cuda_quadrature_weights replaces DWT::quadrature_weights
 *   (include/PFSOFTlib_headers/fn_dwt.hpp:64): d_w receives w_B(j), j < 2B.
 * pfsoft_cuda_wigner_d_matrix replaces DWT::wigner_d_matrix / weighted_wigner_d_matrix
 *   (fn_dwt.hpp:239, :107): rows l = J..B-1 (J = max(|M|,|M'|)) by 2B columns, written
 *   row-major d_out[(l-J)*2B + k] (the reference's matrix is column-major; transpose on the
 *   caller side if needed). weighted != 0 multiplies column k by w_B(k). */
int pfsoft_cuda_quadrature_weights(int B, double* d_w, void* stream);
int pfsoft_cuda_wigner_d_matrix(int B, int M, int Mp, int weighted, double* d_out, void* stream);

/* ---- Seeded coefficients on the device -------------------------------------------------------
 * Counterpart of rand(DSOFTFourierCoefficients&, ...) (include/PFSOFTlib_headers/random.hpp:80),
 * which seeds from the clock; this one is reproducible: value i is a function of (seed, i).
 * kind 0: re, im uniform in [-1, 1); kind 1: |f| = (1+l)^-power |N(0,1)|, uniform phase;
 * kind 2: |f| = (1+l)^-power, uniform phase. Fills all B(4B^2-1)/3 packed values. */
int pfsoft_cuda_random_coeffs(double* d_coeffs, int B, unsigned long long seed, int kind, double power, void* stream);


/* ---- Transform server (continuous batching) -----------------------------------------------
 * No counterpart in the reference, which transforms one grid per call (src/fn_dsoft.cpp:76,
 * src/fn_idsoft.cpp:72); each request here is one such call, queued.
 * A server owns, on the device that is current at creation, one workspace arena of
 * `budget_bytes` (admission is counted against it: a request runs when the spectrum it needs,
 * pfsoft_workspace_bytes(B), fits), `streams` CUDA streams, and a scheduler thread. Requests
 * name caller-owned device buffers that stay on the device; the caller keeps them alive and
 * unchanged until the request finishes. The scheduler puts waiting requests of one direction
 * and bandwidth into one batch (up to `max_batch`), launches it on a free stream as soon as a
 * stream and arena space are free, and keeps doing so while earlier batches run, so work of
 * requests that arrive later overlaps on the device with work already there.
 *   direction 0: DSOFT, d_in = grid (2B)^3, d_out = coefficients.
 *   direction 1: iDSOFT, d_in = coefficients, d_out = grid.
 * submit: `stream` is where the caller produced d_in (NULL: the legacy default stream): the
 *   request's batch waits for the work queued there before the call. The result is complete on
 *   the device once poll / wait report PFSOFT_OK. The first submission of a bandwidth on a device
 *   builds its constant tables inside this call (on the server's own stream; the request's
 *   latency counts from the end of the call).
 *   PFSOFT_ENOMEM if one transform of that bandwidth alone exceeds the budget (it is
 *   rejected, not queued); PFSOFT_EBUSY after the server began shutting down.
 * poll: PFSOFT_EBUSY while queued or running; otherwise the request's final status (PFSOFT_OK,
 *   PFSOFT_ECANCELED, PFSOFT_ECUDA), returned once: the id is forgotten after that.
 * wait: as poll, after waiting up to timeout_s seconds (PFSOFT_ETIMEOUT if still busy).
 * cancel: PFSOFT_OK if the request was still queued (it then finishes as PFSOFT_ECANCELED),
 *   PFSOFT_EBUSY if it is already on the GPU.
 * pause(1) stops new launches (queued requests keep accumulating); pause(0) resumes.
 * drain: waits until nothing is queued or running (PFSOFT_ETIMEOUT after timeout_s).
 * destroy: cancels what is queued, waits for what runs, frees everything; no other call on the
 *   same server may run concurrently with it or follow it. Other calls are thread-safe.
 * Latency statistics cover the most recent 2^20 completed requests since the last reset. */
typedef struct pfsoft_server pfsoft_server;
typedef struct pfsoft_server_stats {
    long long submitted, completed, cancelled, rejected, failed;
    long long batches;              /* batches launched */
    double mean_batch;              /* transforms per batch */
    double p50_ms, p99_ms, mean_ms, max_ms;   /* submit -> result on the device, per request */
    double wall_s;                  /* first submit -> last completion since the last reset */
    double transforms_per_s;        /* completed / wall_s */
    size_t budget_bytes, peak_bytes;           /* arena capacity and high-water mark */
    int max_concurrent_batches;     /* most batches on the device at one time */
    int queued, running;            /* right now */
} pfsoft_server_stats;
int pfsoft_server_create(size_t budget_bytes, int max_batch, int streams, pfsoft_server** out);
/* As pfsoft_server_create, with flags. PFSOFT_SERVER_SPLIT: a batch takes waiting requests of one
 * direction and ANY bandwidths (1 <= B <= 256; larger ones are rejected with PFSOFT_EINVAL) and runs
 * their discrete Wigner transforms in one split-precision launch (the arithmetic of
 * PFSOFT_BATCH_SPLIT; FFT passes per bandwidth). A request's workspace then also holds the split
 * kernel's operand area: pfsoft_workspace_bytes(B) plus (8B(B+1) + B) * 16 + 6144 ceil(D(B)/2)
 * bytes, D(B) = B(B+1)/2 ceil(B/16) (the data operand's digit blocks, one per class and 32-sample
 * chunk; about three quarters of the grid bytes at B = 128 and 256). A bounded wait that ran out
 * finishes that batch's requests with PFSOFT_ETIMEOUT. */
#define PFSOFT_SERVER_SPLIT 1
int pfsoft_server_create_ex(size_t budget_bytes, int max_batch, int streams, int flags, pfsoft_server** out);
int pfsoft_server_destroy(pfsoft_server* srv);
int pfsoft_server_submit(pfsoft_server* srv, int direction, int B, const double* d_in, double* d_out, void* stream,
                         long long* id);
int pfsoft_server_poll(pfsoft_server* srv, long long id);
int pfsoft_server_wait(pfsoft_server* srv, long long id, double timeout_s);
int pfsoft_server_cancel(pfsoft_server* srv, long long id);
int pfsoft_server_pause(pfsoft_server* srv, int paused);
int pfsoft_server_drain(pfsoft_server* srv, double timeout_s);
int pfsoft_server_get_stats(pfsoft_server* srv, pfsoft_server_stats* out);
int pfsoft_server_reset_stats(pfsoft_server* srv);

/* ---- One transform sharded over several GPUs (no counterpart in the reference) -------------
 * The reference parallelises one transform over the order classes with OpenMP
 * (src/fn_dsoft.cpp:134-214, src/fn_idsoft.cpp:124-211) and runs the layer-wise FFT over every beta
 * layer (src/fftw_wrapper.cpp:47-173). A shard plan splits both over nranks GPUs: rank r owns
 * the beta layers [first, first + count) of the (2B)^3 grid (pfsoft_shard_layers; grid index
 * beta outermost, so a slab is one contiguous block of count (2B)^2 values) and a set of order
 * classes balanced by their work. One exchange moves the FFT bins between the two stages.
 *
 * Buffers (complex128, as pairs of doubles; N = 2B; nk = this rank's layer count):
 *   slab grid        nk * N * N      this rank's layers of the grid
 *   slab spectrum    nk * N * N      workspace of the FFT passes (bin-major, beta innermost)
 *   spectrum         N * N * N       workspace of the DWT (only this rank's bins are used)
 *   coefficients     pfsoft_coef_count(B)
 *   send / receive   sums of pfsoft_shard_counts (parts by peer rank, in rank order)
 * DSOFT:  fft_forward(slab grid -> slab spectrum)
 *         exchange FORWARD (slab spectrum -> every rank's spectrum)
 *         dwt_forward(spectrum -> coefficients): this rank's classes, zero elsewhere, so the
 *         element-wise sum over ranks (an all-reduce) is the DSOFT of the whole grid.
 * iDSOFT: dwt_inverse(coefficients -> spectrum): every rank holds the whole coefficient vector
 *         and computes its classes' bins
 *         exchange INVERSE (spectrum -> every rank's slab spectrum)
 *         fft_inverse(slab spectrum -> slab grid); the slab spectrum is overwritten.
 * The exchange is either
 *   scatter: direct stores into each rank's destination buffer; d_dst holds nranks device
 *            pointers (peer mappings for other GPUs, e.g. symmetric memory or CUDA IPC; a rank
 *            that receives nothing may be NULL). All ranks' scatters must be complete before
 *            any rank's next step: the caller synchronises the ranks in between.
 *   pack, all-to-all, unpack: pack into this rank's send buffer, move it with the caller's
 *            all-to-all (NCCL), unpack from the receive buffer.
 * Device tables are made on the first call of each step that takes a stream (allocations and
 * synchronous copies: make those first calls before any stream capture), on the current
 * device; a plan serves one device. pfsoft_shard_classes / _bins / _counts / _runs are host-only queries (the
 * classes and bins of a rank, the values sent to and received from each peer, and the copy runs
 * of an exchange step: step 0 scatter, 1 pack, 2 unpack; a run copies len values from
 * src + src_off to buffer `slot` + dst_off). */
#define PFSOFT_SHARD_FORWARD 0
#define PFSOFT_SHARD_INVERSE 1
typedef struct pfsoft_shard_plan pfsoft_shard_plan;
int pfsoft_shard_create(int B, int nranks, int rank, pfsoft_shard_plan** out);
void pfsoft_shard_destroy(pfsoft_shard_plan* plan);
int pfsoft_shard_layers(const pfsoft_shard_plan* plan, int rank, int* first, int* count);
int pfsoft_shard_classes(const pfsoft_shard_plan* plan, int rank, int* out, int capacity);
long long pfsoft_shard_bins(const pfsoft_shard_plan* plan, int rank, int* out, long long capacity);
int pfsoft_shard_counts(const pfsoft_shard_plan* plan, int direction, long long* send, long long* recv);
long long pfsoft_shard_runs(pfsoft_shard_plan* plan, int direction, int step, long long* src_off, long long* dst_off,
                            int* slot, int* len, long long capacity);
int pfsoft_shard_fft_forward(pfsoft_shard_plan* plan, const double* d_slab_grid, double* d_slab_spectrum, void* stream);
int pfsoft_shard_dwt_forward(pfsoft_shard_plan* plan, const double* d_spectrum, double* d_coeffs, void* stream);
int pfsoft_shard_dwt_inverse(pfsoft_shard_plan* plan, const double* d_coeffs, double* d_spectrum, void* stream);
int pfsoft_shard_fft_inverse(pfsoft_shard_plan* plan, double* d_slab_spectrum, double* d_slab_grid, void* stream);
int pfsoft_shard_scatter(pfsoft_shard_plan* plan, int direction, const double* d_src, double* const* d_dst, void* stream);
int pfsoft_shard_pack(pfsoft_shard_plan* plan, int direction, const double* d_src, double* d_send, void* stream);
int pfsoft_shard_unpack(pfsoft_shard_plan* plan, int direction, const double* d_recv, double* d_dst, void* stream);

/* ---- Diagnostics (no counterpart in the reference) -----------------------------------------
 * pfsoft_launch_count: number of CUDA kernels this library has launched in the process.
 * pfsoft_profile_enable(1) brackets every stage the library launches with CUDA events on the
 * stage's stream; pfsoft_profile_read() waits for them and returns, per stage, the summed
 * device milliseconds and launch count (and resets them). Returns the number of stages;
 * pfsoft_profile_stage_name(i) names stage i. */
long long pfsoft_launch_count(void);
/* Tuning knob used by the autotuner: direction 0 = DSOFT, 1 = IDSOFT; case_split 1 = each warp
 * applies all eight symmetry cases, 2 = warp pairs split them, 0 = library default. */
int pfsoft_tune_dwt_case_split(int direction, int case_split);
/* Tuning knob: on != 0 runs the two FFT passes of a direction in one persistent launch, layer
 * chunk by layer chunk, so that the second pass reads the first pass's output from L2; 0 (the
 * default) runs them as two launches. For bandwidth B (B <= 0: every bandwidth, clearing the
 * per-bandwidth choices). Process-wide; for measurements and the autotuner. */
int pfsoft_tune_fft_fused(int B, int on);
/* Tuning knob: whether a plan created with PFSOFT_BATCH_SPLIT runs bandwidth B's DWT on the split
 * kernel (use_split != 0, the default) or on the FP64 kernels (0). B <= 0: every bandwidth,
 * clearing the per-bandwidth choices. Set by the autotuner; read when a plan is created. */
int pfsoft_tune_split_bandwidth(int B, int use_split);
/* Test knob for the split-precision DWT's failure path (no counterpart in the reference): when
 * wait_ns > 0, every later split launch first waits up to wait_ns nanoseconds on a barrier that
 * nothing signals, before it issues any MMA; the wait runs out, every warp of the kernel leaves,
 * the tensor memory is freed and pfsoft_batch_status then reports PFSOFT_ETIMEOUT. 0 restores
 * normal operation. */
int pfsoft_test_split_wait_ns(unsigned long long wait_ns);
int pfsoft_profile_enable(int on);
int pfsoft_profile_read(double* ms, long long* launches, int max_stages);
const char* pfsoft_profile_stage_name(int stage);

#ifdef __cplusplus
}
#endif

#endif /* PFSOFT_B200_H */
