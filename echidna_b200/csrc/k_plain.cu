// Sweep kernels on plain values: forward evaluation and gradient.
#include "k_common.cuh"

namespace ech {
template <bool DN>
cudaError_t launch_plain(const LaunchReq& r, const KParams& kp, int grid, int block, size_t smem, cudaStream_t st,
                         int* bps) {
  return r.f64 ? launch_by_p<double, DN>(r, kp, grid, block, smem, st, bps)
               : launch_by_p<float, DN>(r, kp, grid, block, smem, st, bps);
}
ECH_INSTANTIATE_DN(launch_plain, const LaunchReq&, const KParams&, int, int, size_t, cudaStream_t, int*)
}  // namespace ech
