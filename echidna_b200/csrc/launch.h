// Kernel registry: maps a value kind / precision / points-per-thread to the
// template instantiation of the sweep kernel and launches it.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include "ech_types.h"

namespace ech {
struct KParams;
struct MultiParams;

enum class VKind { Plain, Dual, Jet };

struct LaunchReq {
  VKind vk = VKind::Plain;
  bool f64 = true;
  int K = 0;      // jet order (Jet kind)
  int P = 1;      // points per thread
  bool rev = false;
  bool dense = false;  // the program holds dense groups: the kernel with the dense-group executor
  bool warp_point = false;  // order-3 jets, one unit per thread: each warp's units share a point
};

size_t value_bytes(const LaunchReq& r);
// Each returns cudaErrorInvalidValue for an unsupported combination.  DN: the
// kernel with the dense-group executor (r.dense).
template <bool DN>
cudaError_t launch_plain(const LaunchReq& r, const KParams& kp, int grid, int block, size_t smem, cudaStream_t st,
                         int* blocks_per_sm);
template <bool DN>
cudaError_t launch_dual(const LaunchReq& r, const KParams& kp, int grid, int block, size_t smem, cudaStream_t st,
                        int* blocks_per_sm);
cudaError_t launch_jet(const LaunchReq& r, const KParams& kp, int grid, int block, size_t smem, cudaStream_t st,
                       int* blocks_per_sm);
// Order-3 jets with dense groups, one unit per thread, every warp's units
// directions of one point (r.warp_point): coefficient 0 of a dense group's
// outputs is accumulated one output per lane and broadcast.
cudaError_t launch_jet3_warp_point(const LaunchReq& r, const KParams& kp, int grid, int block, size_t smem,
                                   cudaStream_t st, int* blocks_per_sm);

// Launch (grid > 0) or query occupancy (grid == 0, result in *blocks_per_sm).
cudaError_t launch_sweep(const LaunchReq& r, const KParams& kp, int grid, int block, size_t smem, cudaStream_t st,
                         int* blocks_per_sm);

// Many-tape persistent gradient + per-point HVP launch (grid == 0: occupancy
// query); dense: some job's program holds dense groups.
template <bool DN>
cudaError_t launch_multi_hvp_dn(bool f64, int P, const MultiParams& mp, int grid, int block, size_t smem,
                                cudaStream_t st, int* blocks_per_sm);
cudaError_t launch_multi_hvp(bool dense, bool f64, int P, const MultiParams& mp, int grid, int block, size_t smem,
                             cudaStream_t st, int* blocks_per_sm);

// STDE per-point reduction of scale*c_k samples (Welford in direction order);
// acc64 selects a double accumulator for f32 samples.
cudaError_t launch_stde_reduce_t(bool f64, bool acc64, const void* c0, const void* ck, double scale, uint64_t npoints,
                                 uint32_t S, const void* cv, double trace, int control, const void* wmul,
                                 void* results, cudaStream_t st);
// The same per-point reduction of FP32 samples in FP32 with compensated sums
// (mean, then the corrected two-pass variance); no control term.
cudaError_t launch_stde_reduce_comp(const void* c0, const void* ck, double scale, uint64_t npoints, uint32_t S,
                                    const void* wmul, void* results, cudaStream_t st);
// S coordinates per point from probability rows (or uniform when probs is null),
// with their importance weights; y *= a.
cudaError_t launch_sample_coords(bool f64, const float* probs, uint32_t n, uint64_t npoints, uint32_t S,
                                 uint64_t seed, uint32_t* idx, void* wmul, cudaStream_t st);
cudaError_t launch_scale(bool f64, void* y, double a, size_t n, cudaStream_t st);
// Sparse STDE over a differential operator: per point, samples sign_e * Z *
// prefactor_e * c_{kout[e]} of the sampled entries (Welford in the sample type).
cudaError_t launch_stde_sparse_reduce(bool f64, const void* coeffs, uint64_t units, const uint32_t* ent,
                                      const uint32_t* kout, const void* pref, const void* sign, double z,
                                      uint64_t npoints, uint32_t S, void* results, cudaStream_t st);
cudaError_t launch_control_term(bool f64, const void* dirs, const void* diag, uint32_t S, uint32_t n, void* cv,
                                cudaStream_t st);

}  // namespace ech
