// Shared launcher body for the sweep-kernel instantiation units.
//
// Each unit is compiled twice, with ECH_DN=0 and ECH_DN=1: the kernels without
// and with the dense-group executor (DN), in separate objects so that the two
// builds of a unit compile in parallel.  A unit compiled without ECH_DN
// instantiates both.
#pragma once
#include <atomic>

#include "interp.cuh"
#include "launch.h"

// ECH_INSTANTIATE_DN(launch_x, parameter types) instantiates launch_x<DN>.
#if !defined(ECH_DN)
#define ECH_INSTANTIATE_DN(NAME, ...)              \
  template cudaError_t NAME<false>(__VA_ARGS__); \
  template cudaError_t NAME<true>(__VA_ARGS__);
#elif ECH_DN
#define ECH_INSTANTIATE_DN(NAME, ...) template cudaError_t NAME<true>(__VA_ARGS__);
#else
#define ECH_INSTANTIATE_DN(NAME, ...) template cudaError_t NAME<false>(__VA_ARGS__);
#endif

namespace ech {

// The kernel's dynamic shared-memory limit is raised once per device to the
// largest size asked so far; launches that need no more skip the attribute call
// (a host round trip that would otherwise precede every launch).
template <class V, int P, bool REV, bool DN, bool WS = false>
cudaError_t launch_one(const KParams& kp, int grid, int block, size_t smem, cudaStream_t st, int* blocks_per_sm) {
  constexpr int kDevices = 64;
  static std::atomic<int> smem_set[kDevices];  // static storage: zero-initialised
  auto fn = sweep_kernel<V, P, REV, DN, WS>;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const bool known = dev >= 0 && dev < kDevices;
  if (!known || (int)smem > smem_set[dev].load(std::memory_order_acquire)) {
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (known) {
      int cur = smem_set[dev].load(std::memory_order_relaxed);
      while ((int)smem > cur && !smem_set[dev].compare_exchange_weak(cur, (int)smem)) {
      }
    }
  }
  if (grid == 0) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, fn, block, smem);
  }
  fn<<<grid, block, smem, st>>>(kp);
  return cudaGetLastError();
}

template <class V, bool DN>
cudaError_t launch_by_p(const LaunchReq& r, const KParams& kp, int grid, int block, size_t smem, cudaStream_t st,
                        int* bps) {
  if (r.rev) {
    switch (r.P) {
      case 1: return launch_one<V, 1, true, DN>(kp, grid, block, smem, st, bps);
      case 2: return launch_one<V, 2, true, DN>(kp, grid, block, smem, st, bps);
      case 4: return launch_one<V, 4, true, DN>(kp, grid, block, smem, st, bps);
      default: return cudaErrorInvalidValue;
    }
  }
  switch (r.P) {
    case 1: return launch_one<V, 1, false, DN>(kp, grid, block, smem, st, bps);
    case 2: return launch_one<V, 2, false, DN>(kp, grid, block, smem, st, bps);
    case 4: return launch_one<V, 4, false, DN>(kp, grid, block, smem, st, bps);
    default: return cudaErrorInvalidValue;
  }
}

// Forward-only kinds (jets): no reverse instantiations.
template <class V, bool DN>
cudaError_t launch_by_p_fwd(const LaunchReq& r, const KParams& kp, int grid, int block, size_t smem, cudaStream_t st,
                            int* bps) {
  if (r.rev) return cudaErrorInvalidValue;
  switch (r.P) {
    case 1: return launch_one<V, 1, false, DN>(kp, grid, block, smem, st, bps);
    case 2: return launch_one<V, 2, false, DN>(kp, grid, block, smem, st, bps);
    case 4: return launch_one<V, 4, false, DN>(kp, grid, block, smem, st, bps);
    default: return cudaErrorInvalidValue;
  }
}

// One point per thread only (wide jets used by the sparse STDE path).
template <class V, bool DN>
cudaError_t launch_p1(const LaunchReq& r, const KParams& kp, int grid, int block, size_t smem, cudaStream_t st,
                      int* bps) {
  if (r.rev || r.P != 1) return cudaErrorInvalidValue;
  return launch_one<V, 1, false, DN>(kp, grid, block, smem, st, bps);
}

}  // namespace ech
