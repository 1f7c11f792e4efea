// Sweep kernels on Taylor jets of order 4 (forward only).
#include "k_common.cuh"

namespace ech {
template <bool DN>
cudaError_t launch_jet4(const LaunchReq& r, const KParams& kp, int grid, int block, size_t smem, cudaStream_t st,
                        int* bps) {
  if (r.rev) return cudaErrorInvalidValue;
  return r.f64 ? launch_by_p_fwd<dm::Jet<double, 4>, DN>(r, kp, grid, block, smem, st, bps)
               : launch_by_p_fwd<dm::Jet<float, 4>, DN>(r, kp, grid, block, smem, st, bps);
}
ECH_INSTANTIATE_DN(launch_jet4, const LaunchReq&, const KParams&, int, int, size_t, cudaStream_t, int*)
}  // namespace ech
