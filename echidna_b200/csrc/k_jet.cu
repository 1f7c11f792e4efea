// Dispatch over the per-order Taylor-jet kernel units (k_jet1.cu .. k_jet9.cu;
// orders 6..9 exist for sparse STDE and run one point per thread).
#include "launch.h"

namespace ech {
cudaError_t launch_jet1(const LaunchReq&, const KParams&, int, int, size_t, cudaStream_t, int*);
cudaError_t launch_jet2(const LaunchReq&, const KParams&, int, int, size_t, cudaStream_t, int*);
cudaError_t launch_jet3(const LaunchReq&, const KParams&, int, int, size_t, cudaStream_t, int*);
cudaError_t launch_jet4(const LaunchReq&, const KParams&, int, int, size_t, cudaStream_t, int*);
cudaError_t launch_jet5(const LaunchReq&, const KParams&, int, int, size_t, cudaStream_t, int*);
cudaError_t launch_jet6(const LaunchReq&, const KParams&, int, int, size_t, cudaStream_t, int*);
cudaError_t launch_jet7(const LaunchReq&, const KParams&, int, int, size_t, cudaStream_t, int*);
cudaError_t launch_jet8(const LaunchReq&, const KParams&, int, int, size_t, cudaStream_t, int*);
cudaError_t launch_jet9(const LaunchReq&, const KParams&, int, int, size_t, cudaStream_t, int*);

cudaError_t launch_jet(const LaunchReq& r, const KParams& kp, int grid, int block, size_t smem, cudaStream_t st,
                       int* bps) {
  switch (r.K) {
    case 1: return launch_jet1(r, kp, grid, block, smem, st, bps);
    case 2: return launch_jet2(r, kp, grid, block, smem, st, bps);
    case 3: return launch_jet3(r, kp, grid, block, smem, st, bps);
    case 4: return launch_jet4(r, kp, grid, block, smem, st, bps);
    case 5: return launch_jet5(r, kp, grid, block, smem, st, bps);
    case 6: return launch_jet6(r, kp, grid, block, smem, st, bps);
    case 7: return launch_jet7(r, kp, grid, block, smem, st, bps);
    case 8: return launch_jet8(r, kp, grid, block, smem, st, bps);
    case 9: return launch_jet9(r, kp, grid, block, smem, st, bps);
    default: return cudaErrorInvalidValue;
  }
}
}  // namespace ech
