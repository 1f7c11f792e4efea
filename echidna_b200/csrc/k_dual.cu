// Sweep kernels on dual values: tangent forward (JVP) and forward-over-reverse HVP.
#include "k_common.cuh"

namespace ech {
template <bool DN>
cudaError_t launch_dual(const LaunchReq& r, const KParams& kp, int grid, int block, size_t smem, cudaStream_t st,
                        int* bps) {
  return r.f64 ? launch_by_p<dm::Dual<double>, DN>(r, kp, grid, block, smem, st, bps)
               : launch_by_p<dm::Dual<float>, DN>(r, kp, grid, block, smem, st, bps);
}
ECH_INSTANTIATE_DN(launch_dual, const LaunchReq&, const KParams&, int, int, size_t, cudaStream_t, int*)
}  // namespace ech
