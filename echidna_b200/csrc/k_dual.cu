// Sweep kernels on dual values: tangent forward (JVP) and forward-over-reverse HVP.
#include "k_common.cuh"

namespace ech {
cudaError_t launch_dual(const LaunchReq& r, const KParams& kp, int grid, int block, size_t smem, cudaStream_t st,
                        int* bps) {
  return r.f64 ? launch_by_p<dm::Dual<double>>(r, kp, grid, block, smem, st, bps)
               : launch_by_p<dm::Dual<float>>(r, kp, grid, block, smem, st, bps);
}
}  // namespace ech
