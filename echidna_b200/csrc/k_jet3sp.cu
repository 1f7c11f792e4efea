// Order-3 jet sweeps whose P units per thread are directions of one point
// (point-direction STDE launches with S % P == 0), with the dense-group
// executor: coefficient 0 of a dense group is accumulated once for the P
// units.  Compiled once (always the dense build).
#include "k_common.cuh"

namespace ech {
cudaError_t launch_jet3_shared_point(const LaunchReq& r, const KParams& kp, int grid, int block, size_t smem,
                                     cudaStream_t st, int* bps) {
  if (r.rev) return cudaErrorInvalidValue;
  // two units per thread (four spill registers)
  if (r.P != 2) return cudaErrorInvalidValue;
  return r.f64 ? launch_one<dm::Jet<double, 3>, 2, false, true, true>(kp, grid, block, smem, st, bps)
               : launch_one<dm::Jet<float, 3>, 2, false, true, true>(kp, grid, block, smem, st, bps);
}
}  // namespace ech
