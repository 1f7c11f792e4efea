/*
 * echidna_b200 — C ABI of the B200-native batched BytecodeTape engine.
 *
 * Every entry point replaces one method of echidna's CUDA backend; the comment on
 * each names the reference interface (path:line inside the echidna crate).  All
 * host buffers are caller-owned, borrowed for the duration of the call, and
 * every length is passed explicitly and checked.  Calls on a context are
 * synchronous (they return after the device work and copies have finished),
 * like the reference's `&self` methods that end in `stream.synchronize()`.
 *
 * Errors are returned as `ech_status`; `ech_last_error()` gives the message of
 * the last failing call on the calling thread.  Messages for the cases the
 * reference reports as `GpuError::Other` use the reference's text (for example
 * "batch_size must be non-zero").  Length mismatches, which the Rust API treats
 * as `assert_eq!` panics, return ECH_ERR_INVALID_ARG.
 *
 * Layouts: inputs are row-major [batch][num_inputs]; outputs are row-major
 * [batch][num_outputs]; Taylor coefficients are coefficient-major
 * [order][batch * num_outputs] (the reference's `TaylorKthBatchResult`).
 */
#ifndef ECHIDNA_B200_H
#define ECHIDNA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define ECH_API __attribute__((visibility("default")))
#else
#define ECH_API
#endif

typedef struct ech_ctx ech_ctx;
typedef struct ech_tape ech_tape;

/* Mirrors GpuError (src/gpu/mod.rs:276-287) plus two codes of this ABI. */
typedef enum ech_status {
  ECH_OK = 0,
  ECH_ERR_NO_DEVICE = 1,                /* GpuError::NoDevice */
  ECH_ERR_SHADER_COMPILATION = 2,       /* GpuError::ShaderCompilation (kernels are built offline) */
  ECH_ERR_OUT_OF_MEMORY = 3,            /* GpuError::OutOfMemory */
  ECH_ERR_CUSTOM_OPS_NOT_SUPPORTED = 4, /* GpuError::CustomOpsNotSupported */
  ECH_ERR_OTHER = 5,                    /* GpuError::Other(msg) */
  ECH_ERR_TIMEOUT = 6,                  /* a bounded device-side wait gave up */
  ECH_ERR_INVALID_ARG = 7               /* length mismatch / null pointer (Rust: assert panic) */
} ech_status;

/* EstimatorResult<F> (src/stde/types.rs:9-22), widened to double. */
typedef struct ech_estimator_result {
  double value;
  double estimate;
  double sample_variance;
  double standard_error;
  uint64_t num_samples;
} ech_estimator_result;

/* Message of the last failing call on this thread ("" if none). */
ECH_API const char* ech_last_error(void);
ECH_API const char* ech_version(void);

/* ── context ─────────────────────────────────────────────────────────────── */
/* CudaContext::new (src/gpu/cuda_backend.rs:503-552).  NO_DEVICE when the
 * device is absent; kernels are compiled offline, so nothing is JIT-compiled. */
ECH_API ech_status ech_ctx_create(int device, ech_ctx** out);
ECH_API void ech_ctx_destroy(ech_ctx* ctx);

/* ── validation (host only, no device needed) ──────────────────────────────── */
/* BytecodeTape::validate (src/bytecode_tape/mod.rs:575-705). */
ECH_API ech_status ech_validate_bytecode_tape(const uint32_t* opcodes, const uint32_t* arg0, const uint32_t* arg1,
                                              uint32_t num_variables, uint32_t num_inputs, uint32_t output_index,
                                              const uint32_t* output_indices, uint32_t n_output_indices,
                                              int has_custom_ops);
/* GpuTapeData::validate (src/gpu/mod.rs:397-564). */
ECH_API ech_status ech_validate_gpu_tape_data(const uint32_t* opcodes, uint32_t n_opcodes, const uint32_t* arg0,
                                              uint32_t n_arg0, const uint32_t* arg1, uint32_t n_arg1,
                                              uint32_t n_constants, uint32_t num_ops, uint32_t num_inputs,
                                              uint32_t num_variables, uint32_t output_index,
                                              const uint32_t* output_indices, uint32_t n_output_indices);

/* ── tape upload ───────────────────────────────────────────────────────────── */
/* GpuBackend::upload_tape (src/gpu/cuda_backend.rs:628-659): GpuTapeData fields
 * (src/gpu/mod.rs:313-334) with f32 constants.  Invalid data -> ECH_ERR_OTHER
 * with "refusing to upload invalid GpuTapeData: ..." (the Rust method panics). */
ECH_API ech_status ech_upload_tape_f32(ech_ctx* ctx, const uint32_t* opcodes, uint32_t n_opcodes,
                                       const uint32_t* arg0, uint32_t n_arg0, const uint32_t* arg1, uint32_t n_arg1,
                                       const float* constants, uint32_t n_constants, uint32_t num_ops,
                                       uint32_t num_inputs, uint32_t num_variables, uint32_t output_index,
                                       const uint32_t* output_indices, uint32_t n_output_indices, ech_tape** out);
/* CudaContext::upload_tape_f64 (src/gpu/cuda_backend.rs:566-611): BytecodeTape<f64>
 * fields.  Custom ops -> CUSTOM_OPS_NOT_SUPPORTED; invalid tape -> OTHER. */
ECH_API ech_status ech_upload_tape_f64(ech_ctx* ctx, const uint32_t* opcodes, const uint32_t* arg0,
                                       const uint32_t* arg1, const double* values, uint32_t num_variables,
                                       uint32_t num_inputs, uint32_t output_index, const uint32_t* output_indices,
                                       uint32_t n_output_indices, int has_custom_ops, ech_tape** out);
ECH_API void ech_tape_destroy(ech_tape* tape);
/* GpuBackend::num_outputs (src/gpu/mod.rs:113). */
ECH_API uint32_t ech_tape_num_outputs(const ech_tape* tape);
ECH_API uint32_t ech_tape_num_inputs(const ech_tape* tape);
ECH_API uint32_t ech_tape_num_variables(const ech_tape* tape);

/* ── batched sweeps (host buffers) ─────────────────────────────────────────── */
/* forward_batch / forward_batch_f64 (src/gpu/cuda_backend.rs:661-676, 878-893). */
ECH_API ech_status ech_forward_batch_f32(ech_ctx* ctx, const ech_tape* tape, const float* inputs, size_t n_inputs,
                                         uint32_t batch_size, float* outputs, size_t n_outputs);
ECH_API ech_status ech_forward_batch_f64(ech_ctx* ctx, const ech_tape* tape, const double* inputs, size_t n_inputs,
                                         uint32_t batch_size, double* outputs, size_t n_outputs);
/* gradient_batch / gradient_batch_f64 (src/gpu/cuda_backend.rs:678-694, 896-912). */
ECH_API ech_status ech_gradient_batch_f32(ech_ctx* ctx, const ech_tape* tape, const float* inputs, size_t n_inputs,
                                          uint32_t batch_size, float* outputs, size_t n_outputs, float* grads,
                                          size_t n_grads);
ECH_API ech_status ech_gradient_batch_f64(ech_ctx* ctx, const ech_tape* tape, const double* inputs,
                                          size_t n_inputs, uint32_t batch_size, double* outputs, size_t n_outputs,
                                          double* grads, size_t n_grads);
/* hvp_batch / hvp_batch_f64 (src/gpu/cuda_backend.rs:705-722, 935-952): one x,
 * batch_size directions. */
ECH_API ech_status ech_hvp_batch_f32(ech_ctx* ctx, const ech_tape* tape, const float* x, size_t n_x,
                                     const float* tangent_dirs, size_t n_dirs, uint32_t batch_size, float* grads,
                                     size_t n_grads, float* hvps, size_t n_hvps);
ECH_API ech_status ech_hvp_batch_f64(ech_ctx* ctx, const ech_tape* tape, const double* x, size_t n_x,
                                     const double* tangent_dirs, size_t n_dirs, uint32_t batch_size, double* grads,
                                     size_t n_grads, double* hvps, size_t n_hvps);
/* Extension (no reference counterpart): per-point HVP, x row-major [batch][n]. */
ECH_API ech_status ech_hvp_batch_points_f32(ech_ctx* ctx, const ech_tape* tape, const float* xs, size_t n_xs,
                                            const float* tangent_dirs, size_t n_dirs, uint32_t batch_size,
                                            float* grads, size_t n_grads, float* hvps, size_t n_hvps);
ECH_API ech_status ech_hvp_batch_points_f64(ech_ctx* ctx, const ech_tape* tape, const double* xs, size_t n_xs,
                                            const double* tangent_dirs, size_t n_dirs, uint32_t batch_size,
                                            double* grads, size_t n_grads, double* hvps, size_t n_hvps);
/* The tangent_forward kernel of the reference (src/gpu/kernels/tape_eval.cu:357-510)
 * that sparse_jacobian dispatches (src/gpu/cuda_backend.rs:306-358): JVP per row. */
ECH_API ech_status ech_tangent_forward_batch_f32(ech_ctx* ctx, const ech_tape* tape, const float* primals,
                                                 size_t n_primals, const float* seeds, size_t n_seeds,
                                                 uint32_t batch_size, float* values, float* tangents,
                                                 size_t n_outputs);
ECH_API ech_status ech_tangent_forward_batch_f64(ech_ctx* ctx, const ech_tape* tape, const double* primals,
                                                 size_t n_primals, const double* seeds, size_t n_seeds,
                                                 uint32_t batch_size, double* values, double* tangents,
                                                 size_t n_outputs);
/* taylor_forward_kth_batch{,_f64} (src/gpu/cuda_backend.rs:829-873): order 1..=5,
 * otherwise ECH_ERR_OTHER "unsupported Taylor order {k}, must be 1..=5".
 * coefficients: [order][batch_size * num_outputs]. */
ECH_API ech_status ech_taylor_forward_kth_batch_f32(ech_ctx* ctx, const ech_tape* tape, const float* primals,
                                                    size_t n_primals, const float* seeds, size_t n_seeds,
                                                    uint32_t batch_size, uint32_t order, float* coefficients,
                                                    size_t n_coefficients);
ECH_API ech_status ech_taylor_forward_kth_batch_f64(ech_ctx* ctx, const ech_tape* tape, const double* primals,
                                                    size_t n_primals, const double* seeds, size_t n_seeds,
                                                    uint32_t batch_size, uint32_t order, double* coefficients,
                                                    size_t n_coefficients);

/* ── STDE (src/gpu/stde_gpu.rs) ───────────────────────────────────────────── */
/* laplacian_gpu (src/gpu/stde_gpu.rs:51-97): directions row-major [S][n]. */
ECH_API ech_status ech_laplacian_gpu_f32(ech_ctx* ctx, const ech_tape* tape, const float* x, size_t n,
                                         const float* directions, uint32_t num_directions,
                                         ech_estimator_result* out);
/* hessian_diagonal_gpu (src/gpu/stde_gpu.rs:103-129). */
ECH_API ech_status ech_hessian_diagonal_gpu_f32(ech_ctx* ctx, const ech_tape* tape, const float* x, size_t n,
                                                float* value, float* diag);
/* laplacian_with_control_gpu (src/gpu/stde_gpu.rs:135-200). */
ECH_API ech_status ech_laplacian_with_control_gpu_f32(ech_ctx* ctx, const ech_tape* tape, const float* x, size_t n,
                                                      const float* directions, uint32_t num_directions,
                                                      const float* control_diagonal, ech_estimator_result* out);
/* Extension (no reference counterpart): many points x S directions in one launch
 * with the per-point reduction on the device.  dir_mode 0: directions
 * [batch][S][n]; 1: directions [S][n] shared by all points; 2: Rademacher
 * directions from a counter-based device RNG (Philox-4x32-10) keyed by `seed`.
 * results: [batch] EstimatorResult of the samples 2*c2 (Welford order = S). */
ECH_API ech_status ech_laplacian_batch_f32(ech_ctx* ctx, const ech_tape* tape, const float* xs, size_t n_xs,
                                           uint32_t batch_size, const float* directions, size_t n_directions,
                                           uint32_t num_directions, int dir_mode, uint64_t seed,
                                           ech_estimator_result* results);
ECH_API ech_status ech_laplacian_batch_f64(ech_ctx* ctx, const ech_tape* tape, const double* xs, size_t n_xs,
                                           uint32_t batch_size, const double* directions, size_t n_directions,
                                           uint32_t num_directions, int dir_mode, uint64_t seed,
                                           ech_estimator_result* results);

/* ── device-pointer variants (inputs already resident in HBM) ─────────────── */
/* Same semantics as the host-buffer calls; pointers are device pointers, the
 * work is enqueued on `stream` (a cudaStream_t, NULL = the context's stream)
 * and the call returns without synchronising.  Scratch is owned by the
 * context, so calls on one context must not overlap on different streams. */
ECH_API ech_status ech_forward_batch_device(ech_ctx* ctx, const ech_tape* tape, int f64, const void* inputs,
                                            uint32_t batch_size, void* outputs, void* stream);
ECH_API ech_status ech_gradient_batch_device(ech_ctx* ctx, const ech_tape* tape, int f64, const void* inputs,
                                             uint32_t batch_size, void* outputs, void* grads, void* stream);
ECH_API ech_status ech_hvp_batch_device(ech_ctx* ctx, const ech_tape* tape, int f64, const void* xs, int x_per_point,
                                        const void* dirs, uint32_t batch_size, void* grads, void* hvps, void* stream);
ECH_API ech_status ech_taylor_batch_device(ech_ctx* ctx, const ech_tape* tape, int f64, const void* primals,
                                           const void* seeds, uint32_t batch_size, uint32_t order,
                                           void* coefficients, void* stream);
/* Device-pointer form of ech_laplacian_batch_*: xs [B][n], dirs as dir_mode says,
 * results[B] (device memory). */
ECH_API ech_status ech_laplacian_batch_device(ech_ctx* ctx, const ech_tape* tape, int f64, const void* xs,
                                              uint32_t batch_size, const void* dirs, uint32_t num_directions,
                                              int dir_mode, uint64_t seed, ech_estimator_result* results,
                                              void* stream);
/* Waits for the context's stream and reports any device-side error word. */
ECH_API ech_status ech_ctx_synchronize(ech_ctx* ctx);

/* ── gradient without device allocation ─────────────────────────────────────
 * No counterpart in the reference.  Same arguments, results and checks as
 * ech_gradient_batch_device, but the call allocates no device memory: the
 * programs and the per-CTA slot scratch live in one fixed region of
 * ech_noalloc_region_bytes() bytes (64 MiB) compiled into the library, one per
 * device.  For callers that must not allocate: a host runtime that owns a
 * fixed device-memory budget or its own pool, or a latency-critical loop that
 * cannot take the device-wide synchronisation cudaMalloc/cudaFree may imply.
 * The first call on a device looks the region up (cudaGetSymbolAddress);
 * make it before any stream capture.  The address is kept for the life of the
 * process, so the call must not be used on a device after cudaDeviceReset.
 * A call copies the tape's programs into the region (from pageable host
 * memory, stream-ordered) only when the region holds a different program;
 * repeated calls on one tape skip the copy.  Large batches run with a smaller grid;
 * a tape whose program plus one CTA's scratch exceeds the region fails with
 * ECH_ERR_OUT_OF_MEMORY.  Nothing in the region needs to start at zero.
 * Calls share the one region per device, so calls whose work overlaps in
 * time (different streams, or different contexts on one device) race on it:
 * order them on one stream.  Device-side errors are reported by
 * ech_ctx_synchronize, as for the other *_device calls. */
ECH_API size_t ech_noalloc_region_bytes(void);
ECH_API ech_status ech_gradient_batch_device_noalloc(ech_ctx* ctx, const ech_tape* tape, int f64, const void* inputs,
                                                     uint32_t batch_size, void* outputs, void* grads, void* stream);

/* Extension: stde::diagonal_kth_order_stochastic (src/stde/higher_order.rs:173-227)
 * on the GPU: one jet of order k+1 along e_j per sampled index j, samples k!*c_k,
 * Welford in the sample type, estimate / variance / SE rescaled by n, n^2, n.
 * k in 2..=8 (jets up to order 9).  Errors use the reference's texts
 * ("sampled_indices must not be empty", "k must be >= 2 (use gradient for k=1)",
 * "k must be <= 18 ...", "k must be <= 12 for f32 ...", "sampled index {j} out of
 * bounds (n={n})"), then "unsupported Taylor order {k+1}, must be 1..=9" for
 * 9 <= k <= 18; scalar-output tapes only. */
ECH_API ech_status ech_diagonal_kth_order_stochastic_f32(ech_ctx* ctx, const ech_tape* tape, const float* x, size_t n,
                                                         uint32_t k, const uint32_t* sampled_indices,
                                                         size_t n_indices, ech_estimator_result* out);
ECH_API ech_status ech_diagonal_kth_order_stochastic_f64(ech_ctx* ctx, const ech_tape* tape, const double* x,
                                                         size_t n, uint32_t k, const uint32_t* sampled_indices,
                                                         size_t n_indices, ech_estimator_result* out);

/* stde::diagonal_kth_order (src/stde/higher_order.rs:40-95) on the GPU: diag[n]
 * = [d^k f / dx_j^k] as k! * c_k of an order-(k+1) jet along every e_j (one
 * launch), value = f(x).  k range and error texts as for the stochastic form;
 * a zero-input tape returns its recorded output value and writes no diagonal;
 * scalar-output tapes only. */
ECH_API ech_status ech_diagonal_kth_order_f32(ech_ctx* ctx, const ech_tape* tape, const float* x, size_t n,
                                              uint32_t k, float* value, float* diag);
ECH_API ech_status ech_diagonal_kth_order_f64(ech_ctx* ctx, const ech_tape* tape, const double* x, size_t n,
                                              uint32_t k, double* value, double* diag);

/* stde::stde_sparse (src/stde/sparse.rs:37-78) over a SparseSamplingDistribution
 * (src/diffop.rs:896-1045), for `batch` points xs [batch][n] with their own
 * sampled entry indices sampled_indices [batch][n_samples]; batch = 1 is the
 * reference call.  The distribution is passed flattened: entry e seeds inputs
 * vars[q] at coefficient slots[q] with input_coeffs[q] (1/slot!) for q in
 * [entry_offsets[e], entry_offsets[e+1]); output_coeff_index[e],
 * extraction_prefactor[e] and sign[e] extract its sample sign * Z * prefactor *
 * c_k with Z = normalization.  Jets run on the GPU up to order 9 (output
 * coefficient index <= 8); Welford in the sample type, value = c0.  Errors:
 * "sampled_indices must not be empty", out-of-range indices, scalar-output
 * tapes only. */
ECH_API ech_status ech_stde_sparse_batch_f32(ech_ctx* ctx, const ech_tape* tape, const float* xs, size_t n_xs,
                                             uint32_t batch, uint32_t n_entries, const uint32_t* entry_offsets,
                                             const uint32_t* vars, const uint32_t* slots, const float* input_coeffs,
                                             const uint32_t* output_coeff_index, const float* extraction_prefactor,
                                             const float* sign, float normalization, const uint64_t* sampled_indices,
                                             uint32_t n_samples, ech_estimator_result* results);
ECH_API ech_status ech_stde_sparse_batch_f64(ech_ctx* ctx, const ech_tape* tape, const double* xs, size_t n_xs,
                                             uint32_t batch, uint32_t n_entries, const uint32_t* entry_offsets,
                                             const uint32_t* vars, const uint32_t* slots, const double* input_coeffs,
                                             const uint32_t* output_coeff_index, const double* extraction_prefactor,
                                             const double* sign, double normalization,
                                             const uint64_t* sampled_indices, uint32_t n_samples,
                                             ech_estimator_result* results);

/* ── many tapes in one launch (extension, no reference counterpart) ─────────
 * Gradient + per-point HVP for a batch of different tapes with uneven input
 * sizes and point counts, as one persistent launch.  Every pointer in an item is
 * a device pointer: xs and dirs [n_points][num_inputs], grads and hvps
 * [n_points][num_inputs].  All tapes belong to `ctx` and share the precision
 * `f64`.  ech_multi_create lowers every tape for one launch shape (with
 * autotune != 0 it times the candidate shapes on the items' own buffers and
 * waits for them), orders the work by cost and sizes the scratch; the buffers
 * are bound to the handle.  ech_multi_launch enqueues a counter reset and one
 * kernel on `stream` (NULL = the context's) and returns without synchronising;
 * device-side errors surface at ech_ctx_synchronize.  Results equal
 * ech_hvp_batch_device with x_per_point = 1 on each item.  Destroy the handle
 * before its context. */
typedef struct ech_multi ech_multi;
typedef struct ech_multi_item {
  const ech_tape* tape;
  const void* xs;
  const void* dirs;
  uint32_t n_points;
  uint32_t pad;
  void* grads;
  void* hvps;
} ech_multi_item;
ECH_API ech_status ech_multi_create(ech_ctx* ctx, int f64, const ech_multi_item* items, uint32_t n_items,
                                    int autotune, ech_multi** out);
ECH_API ech_status ech_multi_launch(ech_multi* multi, void* stream);
/* info[9]: threads, points per thread, CTAs per SM, shared-register cap, grid,
 * tiles, jobs, scratch bytes per CTA, and a word: bit 0 tuned, bit 1 the kernel
 * build with the dense-group executor (as in ech_tape_launch_shape). */
ECH_API ech_status ech_multi_info(const ech_multi* multi, uint64_t* info);
ECH_API void ech_multi_destroy(ech_multi* multi);

/* Extension: exact Hessian diagonals of many points (device arrays): xs [B][n]
 * -> diag [B][n] = 2 * c2 of order-3 jets along every e_j (the batched form of
 * hessian_diagonal_gpu, src/gpu/stde_gpu.rs:103-129, with the values on the GPU). */
ECH_API ech_status ech_hessian_diagonal_batch_device(ech_ctx* ctx, const ech_tape* tape, int f64, const void* xs,
                                                     uint32_t batch_size, void* diag, void* stream);
/* Extension: sparse STDE trace estimate sum_j H_jj for many points (device
 * arrays).  Per point, S coordinates are drawn from the fp32 probability row
 * probs[b][*] (NULL: uniform, as stde::diagonal_kth_order_stochastic with k = 2)
 * with a device Philox stream keyed by `seed`; each sample is 2*c2 / p_j of an
 * order-3 jet along e_j; results[B] are FP64 Welford statistics of the samples
 * (estimate = their mean, unbiased for the trace). */
ECH_API ech_status ech_sparse_trace_batch_device(ech_ctx* ctx, const ech_tape* tape, int f64, const void* xs,
                                                 uint32_t batch_size, const float* probs, uint32_t num_samples,
                                                 uint64_t seed, ech_estimator_result* results, void* stream);

/* ── operator estimators on jets (host buffers; the jets run on the GPU) ──────
 * laplacian_hutchpp (src/stde/laplacian.rs:252-344): sketch [k][n] HVPs, modified
 * Gram-Schmidt (columns with norm < sqrt(eps) dropped), exact trace on the span,
 * Hutchinson on the projected stochastic directions [m][n]. */
ECH_API ech_status ech_laplacian_hutchpp_f32(ech_ctx* ctx, const ech_tape* tape, const float* x, size_t n,
                                             const float* sketch, uint32_t k, const float* stochastic, uint32_t m,
                                             ech_estimator_result* out);
ECH_API ech_status ech_laplacian_hutchpp_f64(ech_ctx* ctx, const ech_tape* tape, const double* x, size_t n,
                                             const double* sketch, uint32_t k, const double* stochastic, uint32_t m,
                                             ech_estimator_result* out);
/* parabolic_diffusion (src/stde/pde.rs:128-162): value and 1/2 sum_i (sigma e_i)^T H (sigma e_i)
 * over the columns sigma [d][n]. */
ECH_API ech_status ech_parabolic_diffusion_f32(ech_ctx* ctx, const ech_tape* tape, const float* x, size_t n,
                                               const float* sigma_columns, uint32_t d, float* value, float* estimate);
ECH_API ech_status ech_parabolic_diffusion_f64(ech_ctx* ctx, const ech_tape* tape, const double* x, size_t n,
                                               const double* sigma_columns, uint32_t d, double* value, double* estimate);
/* parabolic_diffusion_stochastic (src/stde/pde.rs:164-240): sampled columns, estimate d/2 * mean. */
ECH_API ech_status ech_parabolic_diffusion_stochastic_f32(ech_ctx* ctx, const ech_tape* tape, const float* x,
                                                          size_t n, const float* sigma_columns, uint32_t d,
                                                          const uint32_t* sampled_indices, uint32_t m,
                                                          ech_estimator_result* out);
ECH_API ech_status ech_parabolic_diffusion_stochastic_f64(ech_ctx* ctx, const ech_tape* tape, const double* x,
                                                          size_t n, const double* sigma_columns, uint32_t d,
                                                          const uint32_t* sampled_indices, uint32_t m,
                                                          ech_estimator_result* out);
/* stde::estimate and stde::estimate_weighted (src/stde/pipeline.rs:20-142) with
 * estimator 0 = Laplacian (samples 2 c2) or 1 = GradientSquaredNorm (c1^2),
 * src/stde/estimator.rs: order-3 jets along dirs [S][n] at x on the GPU, then
 * Welford (weights NULL) or West's weighted statistics (weights [S], >= 0) in
 * the sample type.  Errors: "directions must not be empty", "estimate_weighted:
 * weights must be non-negative and non-NaN"; scalar-output tapes only. */
ECH_API ech_status ech_estimate_f32(ech_ctx* ctx, const ech_tape* tape, const float* x, size_t n, int estimator,
                                    const float* dirs, uint32_t S, const float* weights, ech_estimator_result* out);
ECH_API ech_status ech_estimate_f64(ech_ctx* ctx, const ech_tape* tape, const double* x, size_t n, int estimator,
                                    const double* dirs, uint32_t S, const double* weights, ech_estimator_result* out);
/* dense_stde_2nd (src/stde/pde.rs:242-296): samples 2 c2 along L z (L row-major n x n,
 * lower triangle used), z_vectors [m][n]. */
ECH_API ech_status ech_dense_stde_2nd_f32(ech_ctx* ctx, const ech_tape* tape, const float* x, size_t n,
                                          const float* cholesky, const float* z_vectors, uint32_t m,
                                          ech_estimator_result* out);
ECH_API ech_status ech_dense_stde_2nd_f64(ech_ctx* ctx, const ech_tape* tape, const double* x, size_t n,
                                          const double* cholesky, const double* z_vectors, uint32_t m,
                                          ech_estimator_result* out);
/* divergence (src/stde/pde.rs:52-106): v^T J v over directions [m][n] of a tape with
 * num_outputs == num_inputs; values[n] receives the outputs (may be NULL). */
ECH_API ech_status ech_divergence_f32(ech_ctx* ctx, const ech_tape* tape, const float* x, size_t n,
                                      const float* directions, uint32_t m, float* values, ech_estimator_result* out);
ECH_API ech_status ech_divergence_f64(ech_ctx* ctx, const ech_tape* tape, const double* x, size_t n,
                                      const double* directions, uint32_t m, double* values, ech_estimator_result* out);

/* grad_checkpointed (src/checkpoint.rs:67-126) for a batch of starting points:
 * x_{t+1} = step(x_t) (a tape with num_outputs == num_inputs = n), objective
 * loss(x_T) (n inputs, one output); grads [B][n] = d loss / d x_0.  Only the
 * states at min(max(num_checkpoints, 1), num_steps) evenly spread positions are
 * kept; each reverse segment recomputes its states from its checkpoint and pulls
 * the adjoint back one step at a time (vector-Jacobian products as gradients of
 * sum_j w_j step(x)_j).  Device arrays; synchronous.  num_steps = 0 gives the
 * gradient of loss(x_0). */
ECH_API ech_status ech_grad_checkpointed_device(ech_ctx* ctx, const ech_tape* step, const ech_tape* loss, int f64,
                                                const void* x0, uint32_t batch_size, uint32_t num_steps,
                                                uint32_t num_checkpoints, void* grads);

/* ── learned sampling proposal for sparse STDE (extension, no reference counterpart) ──
 * A softmax MLP n_in -> hidden -> hidden -> n_out (ReLU), trained on the GPU with
 * BF16 tensor-core GEMMs (tcgen05, FP32 accumulation) and Adam on FP32 master
 * weights.  Sizes are multiples of 64; weights are row-major [out][in]. */
typedef struct ech_mlp ech_mlp;
ECH_API ech_status ech_mlp_create(ech_ctx* ctx, int n_in, int hidden, int n_out, const float* w1, const float* b1,
                                  const float* w2, const float* b2, const float* w3, const float* b3,
                                  ech_mlp** out);
/* x [B][n_in], q [B][n_out] (rows of target probabilities) in device memory;
 * B a positive multiple of 64; synchronous; *loss_out = mean cross-entropy. */
ECH_API ech_status ech_mlp_train_step(ech_mlp* mlp, const float* x, const float* q, int batch, float lr,
                                      float* loss_out);
/* The parameter gradients (and loss) one ech_mlp_train_step would apply, without
 * applying them: same forward / backward kernels, then fp32 copies into host
 * arrays of the create-time sizes (NULL skips one).  For checking the backward
 * pass against a host computation; synchronous. */
ECH_API ech_status ech_mlp_gradients(ech_mlp* mlp, const float* x, const float* q, int batch, float* g_w1,
                                     float* g_b1, float* g_w2, float* g_b2, float* g_w3, float* g_b3,
                                     float* loss_out);
/* probs [B][n_out] = softmax(MLP(x)), device arrays, enqueued on `stream`. */
ECH_API ech_status ech_mlp_forward(ech_mlp* mlp, const float* x, int batch, float* probs, void* stream);
ECH_API ech_status ech_mlp_get_weights(ech_mlp* mlp, float* w1, float* b1, float* w2, float* b2, float* w3,
                                       float* b3);
ECH_API void ech_mlp_destroy(ech_mlp* mlp);
/* The GEMM the MLP uses: C[M][N] (fp32) = A[M][K] * B[N][K]^T (+ bias[N]), A and B
 * bf16 row-major device arrays, K a multiple of 64, lda/ldb multiples of 8. */
ECH_API ech_status ech_gemm_bf16(ech_ctx* ctx, const void* A, const void* B, float* C, const float* bias, int M,
                                 int N, int K, int lda, int ldb, int ldc, void* stream);

/* ── structural sparsity and coloring (host only, no device needed) ──────────
 * Used by the sparse Jacobian / Hessian drop-ins (src/gpu/cuda_backend.rs:306-441),
 * which seed the tangent / HVP sweeps with one row per color.  Two-call
 * pattern: with rows == cols == NULL and cap == 0 only *nnz is set.
 * BytecodeTape::detect_sparsity (src/bytecode_tape/sparse.rs:463-593): the
 * lower triangle (row >= col) of the Hessian pattern, sorted by (row, col). */
ECH_API ech_status ech_detect_hessian_sparsity(const uint32_t* opcodes, const uint32_t* arg0, const uint32_t* arg1,
                                               uint32_t num_variables, uint32_t num_inputs, uint32_t* rows,
                                               uint32_t* cols, size_t cap, size_t* nnz);
/* BytecodeTape::detect_jacobian_sparsity (src/bytecode_tape/sparse.rs:716-776):
 * (output row, input col) in output order, columns ascending. */
ECH_API ech_status ech_detect_jacobian_sparsity(const uint32_t* opcodes, const uint32_t* arg0, const uint32_t* arg1,
                                                uint32_t num_variables, uint32_t num_inputs,
                                                const uint32_t* output_indices, uint32_t n_outputs, uint32_t* rows,
                                                uint32_t* cols, size_t cap, size_t* nnz);
/* sparse::greedy_coloring (src/sparse.rs:57-98): distance-2 coloring of the
 * Hessian pattern; colors[dim]. */
ECH_API ech_status ech_greedy_coloring(uint32_t dim, const uint32_t* rows, const uint32_t* cols, size_t nnz,
                                       uint32_t* colors, uint32_t* num_colors);
/* sparse::column_coloring / row_coloring (src/sparse.rs:292-316): colors[num_inputs]
 * / colors[num_outputs] of the Jacobian pattern's intersection graph. */
ECH_API ech_status ech_column_coloring(uint32_t num_outputs, uint32_t num_inputs, const uint32_t* rows,
                                       const uint32_t* cols, size_t nnz, uint32_t* colors, uint32_t* num_colors);
ECH_API ech_status ech_row_coloring(uint32_t num_outputs, uint32_t num_inputs, const uint32_t* rows,
                                    const uint32_t* cols, size_t nnz, uint32_t* colors, uint32_t* num_colors);

/* ── FP32 precision options of the batch STDE calls (extension) ─────────────
 * Flags for ech_ctx_set_fp32_mode, applied to the FP32 calls of
 * ech_laplacian_batch_f32 / ech_laplacian_batch_device (the drop-in
 * laplacian_gpu family keeps the reference's rounding and f32 Welford):
 *   ECH_FP32_COMPENSATED_JETS   the jet sweep sums linear combinations with
 *                               Neumaier-compensated additions per coefficient
 *   ECH_FP32_COMPENSATED_MEANS  per-point mean and variance in FP32 from
 *                               compensated sums (corrected two-pass variance)
 *   ECH_FP32_PLAIN_MEANS        per-point FP32 Welford, uncompensated
 * 0 (the default): reference rounding in the sweep, FP64 Welford per point.
 * The two MEANS flags exclude each other. */
#define ECH_FP32_COMPENSATED_JETS 1u
#define ECH_FP32_COMPENSATED_MEANS 2u
#define ECH_FP32_PLAIN_MEANS 4u
ECH_API ech_status ech_ctx_set_fp32_mode(ech_ctx* ctx, uint32_t flags);

/* ── introspection ────────────────────────────────────────────────────────── */
/* kind: 0 forward, 1 gradient, 2 hvp, 3 tangent, 4 taylor(order), 5 taylor with
 * linear combinations of inputs read at their source (the program that
 * point-direction jet launches with shared, Rademacher or basis directions run).  Fills
 * stats[12]: fwd_ops, rev_ops, max_live_fwd, max_live_rev, traj_values,
 * flops_fwd, flops_rev, specials_fwd, specials_rev, smem_regs, far_slots,
 * n_instructions. */
ECH_API ech_status ech_tape_plan_stats(ech_ctx* ctx, const ech_tape* tape, int kind, uint32_t order, int f64,
                                       uint64_t* stats);
/* Host-only lowering dump (no device needed): the forward / reverse programs
 * (32-byte records) and constant pool for `kind` with `smem_reg_cap` shared
 * registers, plus the fused-chain terms (48-byte records), the reverse
 * gather records (32-byte) and the outputs of dense groups (32-byte records;
 * groups of up to `dense_max` chains, 1 = none).  counts[9]: n_fwd, n_rev,
 * n_pool, smem_regs, far_slots, traj_slots, n_terms, n_gather_records,
 * n_dense_outputs.  Used to check the lowering on machines without a GPU. */
ECH_API ech_status ech_plan_dump(const uint32_t* opcodes, const uint32_t* arg0, const uint32_t* arg1,
                                 const double* values, uint32_t num_variables, uint32_t num_inputs,
                                 uint32_t output_index, const uint32_t* output_indices, uint32_t n_output_indices,
                                 int kind, uint32_t smem_reg_cap, void* fwd, size_t fwd_cap, void* rev,
                                 size_t rev_cap, double* pool, size_t pool_cap, void* terms, size_t terms_cap,
                                 void* gathers, size_t gathers_cap, void* dense, size_t dense_cap,
                                 uint32_t dense_max, uint64_t* counts);
/* Launch configuration override for tuning (0 = automatic): threads per CTA,
 * points per thread and the shared-register cap. */
ECH_API ech_status ech_ctx_set_launch(ech_ctx* ctx, uint32_t threads, uint32_t points_per_thread,
                                      uint32_t smem_reg_cap);
/* always != 0: every sweep runs the kernel build with the dense-group
 * executor, on the fixed launch shape (an override, like ech_ctx_set_launch).
 * The engine has two builds of each sweep kernel: one carries the dense-group
 * executor, which programs with dense groups need, and one leaves it out, which
 * needs fewer registers; both compute the same results.  By default the
 * autotuner picks per shape. */
ECH_API ech_status ech_ctx_set_dense_kernel(ech_ctx* ctx, int always);
/* Launch-shape autotuning (default on).  Without overrides, the first sweep of
 * a (tape, kind, order, batch-size octave) with at least 512 units times a
 * fixed set of shapes (threads per CTA, points per thread, CTAs per SM) on the
 * call's own inputs and keeps the fastest; every shape computes bit-identical
 * results.  That first call waits for its timing runs; calls made while the
 * stream is being captured use the fixed shape. */
ECH_API ech_status ech_ctx_set_autotune(ech_ctx* ctx, int enable);
/* The shape a sweep of `n_units` units uses.  shape[8]: threads, points per
 * thread, CTAs per SM (0 = fixed shape), shared-register cap, shared registers
 * used, global slots, trajectory slots, and a word whose bit 0 says the shape is
 * tuned and bit 1 that the tuner chose the kernel build with the dense-group
 * executor for a program without dense groups (both builds compute the same
 * results). */
ECH_API ech_status ech_tape_launch_shape(ech_ctx* ctx, const ech_tape* tape, int kind, uint32_t order,
                                        uint64_t n_units, uint64_t* shape);
/* The device program a sweep of `n_units` units runs with that shape (kind 0..4
 * as above, 5 = input-direct jets; built and uploaded if needed).  stats[5]:
 * forward records, reverse records, dense groups, reverse gather tiles, and 1
 * when the sweep runs the kernel build with the dense-group executor. */
ECH_API ech_status ech_tape_program_stats(ech_ctx* ctx, const ech_tape* tape, int kind, uint32_t order,
                                         uint64_t n_units, uint64_t* stats);

#ifdef __cplusplus
}
#endif
#endif /* ECHIDNA_B200_H */
