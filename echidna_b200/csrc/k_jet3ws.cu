// Order-3 jet sweeps with the dense-group executor whose warps each hold 32
// directions of one point (point-direction launches, one unit per thread, S a
// multiple of 32): a dense group's coefficient 0 is accumulated one output per
// lane and broadcast with shuffles.  Compiled once (always the dense build).
#include "k_common.cuh"

namespace ech {
cudaError_t launch_jet3_warp_point(const LaunchReq& r, const KParams& kp, int grid, int block, size_t smem,
                                   cudaStream_t st, int* bps) {
  if (r.rev || r.P != 1) return cudaErrorInvalidValue;
  return r.f64 ? launch_one<dm::Jet<double, 3>, 1, false, true, true>(kp, grid, block, smem, st, bps)
               : launch_one<dm::Jet<float, 3>, 1, false, true, true>(kp, grid, block, smem, st, bps);
}
}  // namespace ech
