// Sweep kernels on Taylor jets, orders 1..5 (forward only).
#include "k_common.cuh"

namespace ech {
template <class T>
static cudaError_t jet_by_k(const LaunchReq& r, const KParams& kp, int grid, int block, size_t smem, cudaStream_t st,
                            int* bps) {
  if (r.rev) return cudaErrorInvalidValue;
  switch (r.K) {
    case 1: return launch_by_p<dm::Jet<T, 1>>(r, kp, grid, block, smem, st, bps);
    case 2: return launch_by_p<dm::Jet<T, 2>>(r, kp, grid, block, smem, st, bps);
    case 3: return launch_by_p<dm::Jet<T, 3>>(r, kp, grid, block, smem, st, bps);
    case 4: return launch_by_p<dm::Jet<T, 4>>(r, kp, grid, block, smem, st, bps);
    case 5: return launch_by_p<dm::Jet<T, 5>>(r, kp, grid, block, smem, st, bps);
    default: return cudaErrorInvalidValue;
  }
}
cudaError_t launch_jet(const LaunchReq& r, const KParams& kp, int grid, int block, size_t smem, cudaStream_t st,
                       int* bps) {
  return r.f64 ? jet_by_k<double>(r, kp, grid, block, smem, st, bps) : jet_by_k<float>(r, kp, grid, block, smem, st, bps);
}
}  // namespace ech
