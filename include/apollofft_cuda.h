/* apollofft_cuda.h -- C ABI of apollofft_b200, the B200 (sm_100a) backend for
 * apollo-fft's dense FFT plan execution.
 *
 * Plain C types only: pointers, sizes, enums.  A Rust crate binds these with an
 * `extern "C"` block; Python binds them with ctypes (apollofft_b200/_lib.py).
 *
 * Conventions (crates/apollo-fft/src/domain/metadata/precision.rs:15-19,
 * Normalization::FftwCompatible): forward is unnormalized, inverse is scaled by
 * 1/N (N = product of the transform dims).  Data are C-order, interleaved
 * (re, im), with `batch` transforms back to back.  Every call returns an
 * afc_status; nothing aborts.  Kernels run asynchronously on the caller's
 * stream; only the *_host variants and plan creation synchronize.
 */
#ifndef APOLLOFFT_CUDA_H
#define APOLLOFFT_CUDA_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define AFC_API __attribute__((visibility("default")))
#else
#define AFC_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces ApolloError (crates/apollo-fft/src/domain/contracts/error.rs:10-47):
 * Validation, ShapeMismatch, NonContiguous, BackendUnavailable, plus device,
 * memory and timeout conditions the CPU backend does not have. */
typedef enum {
  AFC_OK = 0,
  AFC_ERR_VALIDATION = 1,
  AFC_ERR_SHAPE_MISMATCH = 2,
  AFC_ERR_NON_CONTIGUOUS = 3,
  AFC_ERR_BACKEND_UNAVAILABLE = 4,
  AFC_ERR_DEVICE = 5,
  AFC_ERR_OUT_OF_MEMORY = 6,
  AFC_ERR_TIMEOUT = 7,
  AFC_ERR_UNSUPPORTED = 8
} afc_status;

/* Precision profiles (precision.rs:55-85): F64 = HIGH_ACCURACY_F64 (the
 * `high_accuracy` plan), F32 = LOW_PRECISION_F32 (`low_precision`).  The two
 * tensor-core forms compute radix-16 stages as split-precision DFT-matrix
 * products with FP32 accumulation on complex64 data; they plan rank-1 C2C
 * lengths n = 2^k, 16 <= n <= 4096 (the one radix-2/4/8 stage of lengths that
 * are not 16^s runs in FP32 on the CUDA cores) and return AFC_ERR_UNSUPPORTED
 * for anything else. */
typedef enum {
  AFC_PREC_F32 = 0,
  AFC_PREC_F64 = 1,
  AFC_PREC_TC_BF16_SPLIT = 2,
  AFC_PREC_TC_FP16_SPLIT = 3
} afc_precision;

/* C2C: complex -> complex.
 * R2C_FULL: the reference's "R2C": real input widened to complex, full C2C,
 *   output of the same shape (plan/fft/real_storage.rs:186-303); its inverse is
 *   a full C2C inverse followed by taking the real part ("C2R").  Rank >= 2
 *   forward: the columns past n/2 of the last axis are stored as the exact
 *   conjugates of their partners X[(-k) mod n0][n1 - c].
 * R2C_HALF: Hermitian half spectrum, last dim n -> n/2 + 1 (new explicit API;
 *   the reference models HalfSpectrum3D in domain/metadata/shape.rs:79-95 but
 *   never wires it). */
typedef enum { AFC_KIND_C2C = 0, AFC_KIND_R2C_FULL = 1, AFC_KIND_R2C_HALF = 2 } afc_kind;

typedef enum { AFC_FORWARD = 0, AFC_INVERSE = 1 } afc_direction;

typedef struct afc_plan_s* afc_plan;

/* Mirrors BackendCapabilities (domain/contracts/backend.rs:9-29). */
typedef struct {
  int kind; /* 2 = CUDA (the reference has Cpu = 0, Wgpu = 1) */
  int normalization; /* 0 = FftwCompatible */
  int supports_1d, supports_2d, supports_3d;
  int supports_real_to_complex;
  int supports_mixed_precision;
  int default_precision; /* afc_precision */
  int device_count;
  int sm_count;
  int cc_major, cc_minor;
  size_t max_smem_per_block;
} afc_capabilities_t;

/* Reference dispatch decision for one length (mixed_radix/dispatch.rs:26-132),
 * reported bit-exactly from this library's own integer layer. */
typedef struct {
  int strategy;          /* 0 noop, 1 stockham, 2 four_step, 3 winograd, 4 pfa_static,
                            5 composite, 6 pfa_generic, 7 rader_full, 8 rader_half,
                            9 untransformed (prime power the reference leaves as is) */
  int n_radices;         /* lowered prime23 radices (radix_shape.rs:60-234), -1 if None */
  uint64_t radices[64];
  uint64_t coprime_n1, coprime_n2; /* radix_shape.rs:192-219, 0 if None */
  uint64_t four_step_n1, four_step_n2; /* four_step/mod.rs:66-70, 0 unless pow2 */
  uint64_t primitive_root, primitive_root_inv; /* rader/generator.rs:18-120, 0 unless prime */
  int is_prime;
  int is_short_winograd;
  int has_static_coprime_codelet;
  /* GPU execution chosen by this library for the length */
  int gpu_algo;          /* 0 smem Stockham, 1 four-step, 2 Rader, 3 Bluestein, 4 noop */
  int gpu_n_radices;
  int gpu_radices[24];
  uint64_t gpu_conv_len; /* convolution length for Rader/Bluestein */
  uint64_t gpu_split_n1, gpu_split_n2;
} afc_length_info_t;

/* ── plans (FftPlan1D/2D/3D::new, plan/fft/dimension_{1,2,3}d.rs) ──────────── */

/* Replaces FftPlan1D/2D/3D::new (dimension_1d.rs:24-41, dimension_2d.rs:77-100,
 * dimension_3d.rs:92-123) and Shape{1,2,3}D::new validation (shape.rs:14-56):
 * rank 1..3, dims[0..rank) > 0, batch >= 1.  Twiddle, Rader and Bluestein
 * tables are generated on `device` and stay resident with the plan. */
AFC_API afc_status afc_plan_create(afc_plan* out, int rank, const int64_t* dims, afc_precision precision,
                           afc_kind kind, int64_t batch, int device);

/* Replaces PlanCacheProvider::get_{1,2,3}d_plan (orchestration/cache/plans.rs:15-231):
 * a process-wide, mutex-guarded, reference-counted cache keyed by
 * (rank, dims, precision, kind, batch, device).  Release with afc_plan_destroy. */
AFC_API afc_status afc_plan_get_cached(afc_plan* out, int rank, const int64_t* dims, afc_precision precision,
                               afc_kind kind, int64_t batch, int device);

/* Drops one reference; frees device tables when the last one goes. */
AFC_API afc_status afc_plan_destroy(afc_plan plan);

/* Replaces forward_complex_inplace / inverse_complex_inplace and their slice
 * forms (dimension_1d.rs:55-82, dimension_2d.rs:102-122, dimension_3d.rs:148-169).
 * Device pointers; in == out runs in place (C2C only).  Input element counts:
 * C2C batch*N complex; R2C_FULL forward batch*N real -> batch*N complex,
 * inverse batch*N complex -> batch*N real; R2C_HALF forward batch*N real ->
 * batch*N/n_last*(n_last/2+1) complex, inverse the reverse. */
AFC_API afc_status afc_execute(afc_plan plan, const void* in, void* out, afc_direction direction, void* stream);

/* Same with an explicit overall scale in place of the convention (1 forward,
 * 1/N inverse). */
AFC_API afc_status afc_execute_scaled(afc_plan plan, const void* in, void* out, afc_direction direction,
                              double scale, void* stream);

/* Adjoint (conjugate transpose, real inner product for real spaces) of the
 * linear map afc_execute(plan, ., ., direction): the backward pass of an
 * autograd function.  C2C forward -> unnormalized inverse; C2C inverse -> forward
 * times 1/N; R2C_FULL forward -> real part of the unnormalized inverse;
 * R2C_HALF adds the Hermitian weights (1/2 on bins 1..ceil(n/2)-1 going back,
 * 2 going forward).  No reference counterpart (the reference has no autograd). */
AFC_API afc_status afc_execute_adjoint(afc_plan plan, const void* in, void* out, afc_direction direction,
                               void* stream);

/* Host-pointer convenience form (mirrors the slice API callers such as
 * apollo-nufft/stft/czt use): copies host -> device, executes, copies back,
 * synchronizes.  Safe from many host threads on one shared (cached) plan, as
 * the reference's Send + Sync plans are: each call in flight takes its own
 * staging set (device stream, input and output buffers, workspace); up to 4
 * calls of one plan run at once and further callers wait for a free set. */
AFC_API afc_status afc_execute_host(afc_plan plan, const void* host_in, void* host_out, afc_direction direction);

/* Workspace the plan needs for one execution on one stream, in bytes (0 if
 * none).  afc_execute keeps plan-owned workspaces, one per stream that uses the
 * plan (up to 4; further streams take turns on the least recently used one):
 * each is ordered after its last use by an event the next user's stream waits
 * on, so calls on one shared plan from several streams and threads are safe
 * without host synchronization.  Calls captured into a CUDA graph skip that
 * ordering: replay such a graph ordered with other calls on the plan.
 * afc_execute_ws takes a caller-owned workspace and does no ordering at all. */
AFC_API afc_status afc_workspace_size(afc_plan plan, size_t* bytes);
AFC_API afc_status afc_execute_ws(afc_plan plan, const void* in, void* out, afc_direction direction, double scale,
                          int use_scale, void* workspace, size_t workspace_bytes, void* stream);

/* Element counts of one execution's input and output (complex or real elements). */
AFC_API afc_status afc_plan_io_elems(afc_plan plan, afc_direction direction, int64_t* in_elems, int64_t* out_elems);

/* ── uneven batches (new: many lengths in one persistent launch) ─────────── */

typedef struct afc_batch_plan_s* afc_batch_plan;

/* Lanes of lengths[i] packed back to back (offset = prefix sum).  Precision
 * F32 or F64.  Each length gets an autotuned configuration from the plan cache. */
AFC_API afc_status afc_batch_plan_create(afc_batch_plan* out, const int64_t* lengths, int64_t count,
                                 afc_precision precision, int device);
AFC_API afc_status afc_batch_plan_destroy(afc_batch_plan plan);
/* mode 0: one persistent launch per phase; the first call per buffer pair and
 * direction runs the phases directly and captures them into a CUDA graph that
 * later calls replay (a capture the driver refuses only means the next call
 * runs directly again; inside a caller's own capture the phases are recorded
 * into it), mode 1: one plain launch per distinct length, mode 2: the
 * persistent phases without the graph.  Calls on
 * one batch plan from several streams are ordered on the GPU (its workspace is
 * shared), so they are safe but do not overlap. */
AFC_API afc_status afc_batch_execute(afc_batch_plan plan, const void* in, void* out, afc_direction direction,
                             int mode, void* stream);
AFC_API afc_status afc_batch_total_elems(afc_batch_plan plan, int64_t* elems);

/* ── introspection / integer layer ───────────────────────────────────────── */

AFC_API afc_status afc_capabilities(afc_capabilities_t* caps);
AFC_API afc_status afc_length_info(uint64_t n, afc_length_info_t* info);
/* Rader maps (rader/mod.rs:215-246): gather[q] = g^q mod p, scatter[q] = g^{-q} mod p. */
AFC_API afc_status afc_rader_maps(uint64_t p, uint64_t* gather, uint64_t* scatter);
/* Good-Thomas CRT permutations (mixed_radix/caches/misc.rs:233-256). */
AFC_API afc_status afc_pfa_perm(uint64_t n1, uint64_t n2, uint64_t* in_perm, uint64_t* out_perm);
AFC_API afc_status afc_plan_describe(afc_plan plan, int axis, afc_length_info_t* info);
/* Thread-local message of the last failing call on this thread. */
AFC_API const char* afc_last_error_message(void);
/* Number of kernels this library launched in this process (all devices). */
AFC_API uint64_t afc_kernel_launch_count(void);

/* ── fused caller operations ──────────────────────────────────────────────── */

/* STFT analysis on the device, frames gathered and windowed inside the FFT's
 * load: replaces the frame loop of apollo-stft StftPlan::forward_with_window /
 * forward_f64_slice_into (apollo-stft/.../plan/stft/dimension_1d.rs:132-239),
 * which copies each frame into a host slice and calls
 * FftPlan1D::forward_complex_slice_inplace on it.  `plan` is a rank-1 C2C F32 or
 * F64 plan of length frame_len whose length fits one CTA; `signal` (signal_len
 * reals) and `window` (frame_len reals) are device arrays of the plan's real
 * type; frame m covers signal[m hop - frame_len/2 + i] * window[i] (zero
 * outside the signal), frames = 1 + ceil(signal_len / hop)
 * (dimension_1d.rs:102-108); `out` receives frames x frame_len complex values,
 * `out_elems` must equal that count.  Errors as the reference's StftError:
 * hop 0 or hop > frame_len, signal shorter than a frame -> AFC_ERR_VALIDATION. */
AFC_API afc_status afc_stft_frame_count(int64_t frame_len, int64_t hop, int64_t signal_len, int64_t* frames);
AFC_API afc_status afc_stft_forward(afc_plan plan, const void* signal, int64_t signal_len, const void* window,
                                    int64_t hop, void* out, int64_t out_elems, void* stream);
/* Inverse STFT by weighted overlap-add, apollo-stft StftPlan::inverse_into
 * (stft/dimension_1d.rs:250-345): every frame's normalized inverse FFT, real
 * part, times the window, overlap-added at m hop - frame_len/2 and divided by
 * the summed squared window (zero where no frame covers a sample).
 * `spectrum_elems` = frames x frame_len with frames from signal_len as in the
 * forward; `out` receives signal_len reals.  `workspace` holds the transformed
 * frames: at least afc_stft_inverse_workspace() bytes (frames x frame_len reals),
 * caller-owned device memory. */
AFC_API afc_status afc_stft_inverse_workspace(afc_plan plan, int64_t hop, int64_t signal_len, size_t* bytes);
AFC_API afc_status afc_stft_inverse(afc_plan plan, const void* spectrum, int64_t spectrum_elems, const void* window,
                                    int64_t hop, void* out, int64_t signal_len, void* workspace, size_t workspace_bytes,
                                    void* stream);

/* Chirp z-transform on the device: X_k = sum_j x_j A^-j W^(j k), j < n, k < m,
 * by Bluestein's identity in one launch (chirp premultiply fused into the
 * convolution's load, FFT, product with the kernel spectrum, inverse FFT and
 * chirp postmultiply fused into its store).  Replaces apollo-czt CztPlan::new /
 * forward_into (apollo-czt/.../plan/czt/dimension_1d.rs:60-120 and
 * kernel/bluestein.rs:83-130), which run the premultiply, the two
 * FftPlan1D slice transforms and the postmultiply on host buffers; same chirp
 * tables (num-complex powf, polar form) and the same convolution length
 * L = next_pow2(n + m - 1).  When L does not fit one CTA the same steps run
 * around the library's multi-pass plan of length L (five launches, workspace
 * stream-ordered on `stream`).  n, m > 0 and finite non-zero A, W
 * (CztError::EmptyLength / InvalidParameters -> AFC_ERR_VALIDATION).  Execute:
 * `batch` contiguous lanes of n complex inputs -> `batch` lanes of m complex
 * outputs (F32: complex64, F64: complex128), device pointers, on `stream`.
 *
 * afc_czt_inverse replaces CztPlan::inverse (plan/czt/dimension_1d.rs:250-293,
 * czt_bjork_pereyra_inverse_into in kernel/bluestein.rs:167-223): the exact
 * inverse of a square plan by the Björck-Pereyra solve of the Vandermonde
 * system on z_k = W^k, then x_k = y_k A^k, in FP64 (complex64 plans convert
 * on load and store), one CTA per lane.  Errors as the reference's
 * CztError::NotInvertible (AFC_ERR_VALIDATION): m != n, or two nodes closer
 * than 1024 eps (W a root of unity of order <= n); n beyond one CTA's shared
 * memory (n > 7040) is AFC_ERR_UNSUPPORTED.  `batch` lanes of n in, n out. */
typedef struct afc_czt_plan_s* afc_czt_plan;
AFC_API afc_status afc_czt_plan_create(afc_czt_plan* out, int64_t n, int64_t m, double a_re, double a_im,
                                       double w_re, double w_im, afc_precision precision, int device);
AFC_API afc_status afc_czt_execute(afc_czt_plan plan, const void* in, void* out, int64_t batch, void* stream);
AFC_API afc_status afc_czt_inverse(afc_czt_plan plan, const void* spectrum, void* out, int64_t batch, void* stream);
AFC_API afc_status afc_czt_conv_len(afc_czt_plan plan, int64_t* conv_len);
AFC_API afc_status afc_czt_plan_destroy(afc_czt_plan plan);

/* Analytic signal on the device, apollo-hilbert HilbertPlan::analytic_signal_into
 * (apollo-hilbert/.../plan/hilbert.rs:52-75 over infrastructure/kernel/direct.rs:
 * 85-143): forward FFT of each real lane, the analytic mask (1 at DC and, for
 * even n, at n/2; 2 on bins 1..(n+1)/2-1; 0 above), normalized inverse FFT,
 * as one fused launch (one shared-memory tile per lane).  `signal` is
 * batch x n real (float64 for F64, float32 for F32), `out` batch x n complex,
 * device pointers.  The quadrature H{x} is the imaginary part; the real part
 * is the inverse FFT's value (the reference then overwrites it with x; here it
 * equals x to rounding).  n must be smooth (2, 3, 5, 7, 11, 13 factors) and fit
 * one CTA, else AFC_ERR_UNSUPPORTED; n = 1 gives x + 0i. */
typedef struct afc_hilbert_plan_s* afc_hilbert_plan;
AFC_API afc_status afc_hilbert_plan_create(afc_hilbert_plan* out, int64_t n, afc_precision precision, int device);
AFC_API afc_status afc_hilbert_analytic(afc_hilbert_plan plan, const void* signal, void* out, int64_t batch,
                                        void* stream);
AFC_API afc_status afc_hilbert_plan_destroy(afc_hilbert_plan plan);

/* 1D non-uniform FFT on the device, apollo-nufft NufftPlan1D
 * (apollo-nufft/.../transform/dimension_1d.rs:101-272): n uniform bins on the
 * periodic domain [0, n dx), oversampled grid m = sigma n, Kaiser-Bessel kernel
 * of half width kernel_width (reference defaults: sigma 2, width 6).  Type 1:
 * out[k] ~ sum_j values_j exp(-2 pi i k_signed x_j / (n dx)), k < n; type 2:
 * out[j] ~ sum_k coeffs_k exp(+2 pi i k_signed x_j / (n dx)).  Positions are
 * float64, values / coeffs / outputs complex128, all device pointers.  The
 * spreading, the FFT of this library and the deconvolution follow the
 * reference step by step (type 1 spreads with atomic adds instead of the
 * reference's bucket sort, so sums differ in rounding only).  Calls on one plan
 * share its grid: calls on the same stream are ordered, overlapping calls on
 * different streams race.  Invalid n, dx, sigma < 2 or width outside 2..32 ->
 * AFC_ERR_VALIDATION. */
typedef struct afc_nufft_plan_s* afc_nufft_plan;
AFC_API afc_status afc_nufft1d_plan_create(afc_nufft_plan* out, int64_t n, double dx, int64_t sigma,
                                           int64_t kernel_width, int device);
AFC_API afc_status afc_nufft1d_type1(afc_nufft_plan plan, const double* positions, const void* values, int64_t npts,
                                     void* out, void* stream);
AFC_API afc_status afc_nufft1d_type2(afc_nufft_plan plan, const void* coeffs, const double* positions, int64_t npts,
                                     void* out, void* stream);
AFC_API afc_status afc_nufft_plan_destroy(afc_nufft_plan plan);

/* 3D non-uniform FFT on the device, apollo-nufft NufftPlan3D
 * (apollo-nufft/.../transform/dimension_3d.rs:193-620): nx x ny x nz modes on
 * the periodic box [0, nx dx) x [0, ny dy) x [0, nz dz); per axis the
 * oversampled length is next_pow2(max(sigma n, 2 kernel_width + 1))
 * (dimension_3d.rs:48-54); separable Kaiser-Bessel weights over
 * (2 kernel_width + 1)^3 cells.  Positions are npts x 3 float64 (x, y, z per
 * point), values / modes / outputs complex128, modes and type-1 outputs C order
 * [kx][ky][kz]; all device pointers.  Type 1: out[kx,ky,kz] ~ sum_j values_j
 * exp(-2 pi i (kx_s x_j / Lx + ky_s y_j / Ly + kz_s z_j / Lz)).  Type 2 follows
 * the reference's normalized inverse axis passes (dimension_3d.rs:548-551):
 * out[j] ~ sum_k modes_k exp(+2 pi i (...)) / (mx my mz).  Spreading uses
 * atomic adds instead of the reference's bucket sort (rounding differs only).
 * One grid per plan: overlapping calls on different streams race.
 * afc_nufft3d_grid_dims writes (mx, my, mz). */
typedef struct afc_nufft3d_plan_s* afc_nufft3d_plan;
AFC_API afc_status afc_nufft3d_plan_create(afc_nufft3d_plan* out, int64_t nx, int64_t ny, int64_t nz, double dx,
                                           double dy, double dz, int64_t sigma, int64_t kernel_width, int device);
AFC_API afc_status afc_nufft3d_grid_dims(afc_nufft3d_plan plan, int64_t* m);
AFC_API afc_status afc_nufft3d_type1(afc_nufft3d_plan plan, const double* positions, const void* values, int64_t npts,
                                     void* out, void* stream);
AFC_API afc_status afc_nufft3d_type2(afc_nufft3d_plan plan, const void* modes, const double* positions, int64_t npts,
                                     void* out, void* stream);
AFC_API afc_status afc_nufft3d_plan_destroy(afc_nufft3d_plan plan);

/* Allocation-free execution of a rank-1 C2C plan whose length runs on the
 * two-pass (four-step) kernels: the intermediate between the passes lives in a
 * 16 MiB static device array instead of a cudaMalloc'd workspace, so the call
 * allocates and frees nothing (cudaMalloc/cudaFree can synchronize the device
 * and are not allowed inside CUDA stream capture; callers such as streaming
 * STFT frame loops, allocator-owned memory pools or capture regions cannot
 * afford them).  No counterpart in the reference.  Create the plan beforehand.
 * batch * n * sizeof(complex) must not exceed 16 MiB (AFC_ERR_VALIDATION
 * otherwise).  The first call on a device looks up the array's address and
 * should come before any stream capture.  All calls share the one array:
 * calls that overlap on the GPU (different streams, no ordering) race. */
AFC_API afc_status afc_execute_1d_no_alloc(afc_plan plan, const void* in, void* out, afc_direction direction,
                                           void* stream);

/* ── exact direct non-uniform DFTs ─────────────────────────────────────────── */

/* Replace apollo-nufft's exact direct sums behind apollo-python's
 * nufft_type1_1d / nufft_type2_1d / nufft_type1_3d
 * (crates/apollo-nufft/src/application/execution/transform/dimension_1d.rs:428-472,
 * dimension_3d.rs:677-712; bindings crates/apollo-python/src/lib.rs:753-850):
 * every output is the full O(inputs) sum, phase (2 pi / L) k x with k the
 * FFT-signed index (k <= n/2 stays, else k - n) and L = n dx per axis, in
 * FP64.  Device pointers: positions float64 (3D: npts x 3, row major), values,
 * coefficients and outputs complex128.  Domain checks as UniformDomain1D::new /
 * UniformGrid3D::new (n > 0, spacing finite and > 0).  Runs on `device`, on
 * the caller's stream.
 * type1: out[k] = sum_j v_j exp(-i 2 pi k x_j / L), k < n.
 * type2: out[j] = sum_k c_k exp(+i 2 pi k x_j / L), j < npts.
 * 3D type1: out[kx, ky, kz] (C order) = sum_j v_j exp(-i 2 pi (kx x_j / Lx + ky y_j / Ly + kz z_j / Lz)). */
AFC_API afc_status afc_nudft1d_type1(const double* positions, const void* values, int64_t npts, int64_t n, double dx,
                                     void* out, int device, void* stream);
AFC_API afc_status afc_nudft1d_type2(const void* coeffs, int64_t n, const double* positions, int64_t npts, double dx,
                                     void* out, int device, void* stream);
AFC_API afc_status afc_nudft3d_type1(const double* positions, const void* values, int64_t npts, int64_t nx,
                                     int64_t ny, int64_t nz, double dx, double dy, double dz, void* out, int device,
                                     void* stream);

#ifdef __cplusplus
}
#endif

#endif /* APOLLOFFT_CUDA_H */
