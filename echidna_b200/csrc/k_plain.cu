// Sweep kernels on plain values: forward evaluation and gradient.
#include "k_common.cuh"

namespace ech {
cudaError_t launch_plain(const LaunchReq& r, const KParams& kp, int grid, int block, size_t smem, cudaStream_t st,
                         int* bps) {
  return r.f64 ? launch_by_p<double>(r, kp, grid, block, smem, st, bps)
               : launch_by_p<float>(r, kp, grid, block, smem, st, bps);
}
}  // namespace ech
