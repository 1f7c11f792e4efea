// Sweep kernels on Taylor jets of order 9 (forward only, one point per thread):
// the wide jets of sparse STDE over differential operators.
#include "k_common.cuh"

namespace ech {
template <bool DN>
cudaError_t launch_jet9(const LaunchReq& r, const KParams& kp, int grid, int block, size_t smem, cudaStream_t st,
                        int* bps) {
  return r.f64 ? launch_p1<dm::Jet<double, 9>, DN>(r, kp, grid, block, smem, st, bps)
               : launch_p1<dm::Jet<float, 9>, DN>(r, kp, grid, block, smem, st, bps);
}
ECH_INSTANTIATE_DN(launch_jet9, const LaunchReq&, const KParams&, int, int, size_t, cudaStream_t, int*)
}  // namespace ech
