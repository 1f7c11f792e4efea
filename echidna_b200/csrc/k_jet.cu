// Dispatch over the per-order Taylor-jet kernel units (k_jet1.cu .. k_jet5.cu).
#include "launch.h"

namespace ech {
cudaError_t launch_jet1(const LaunchReq&, const KParams&, int, int, size_t, cudaStream_t, int*);
cudaError_t launch_jet2(const LaunchReq&, const KParams&, int, int, size_t, cudaStream_t, int*);
cudaError_t launch_jet3(const LaunchReq&, const KParams&, int, int, size_t, cudaStream_t, int*);
cudaError_t launch_jet4(const LaunchReq&, const KParams&, int, int, size_t, cudaStream_t, int*);
cudaError_t launch_jet5(const LaunchReq&, const KParams&, int, int, size_t, cudaStream_t, int*);

cudaError_t launch_jet(const LaunchReq& r, const KParams& kp, int grid, int block, size_t smem, cudaStream_t st,
                       int* bps) {
  switch (r.K) {
    case 1: return launch_jet1(r, kp, grid, block, smem, st, bps);
    case 2: return launch_jet2(r, kp, grid, block, smem, st, bps);
    case 3: return launch_jet3(r, kp, grid, block, smem, st, bps);
    case 4: return launch_jet4(r, kp, grid, block, smem, st, bps);
    case 5: return launch_jet5(r, kp, grid, block, smem, st, bps);
    default: return cudaErrorInvalidValue;
  }
}
}  // namespace ech
