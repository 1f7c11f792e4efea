// Dispatch over the sweep-kernel units: value kind, the dense-group executor
// (LaunchReq::dense), and for jets the per-order units k_jet1.cu .. k_jet9.cu
// (orders 6..9 exist for sparse STDE and run one point per thread).  This unit
// holds no kernel templates, so it instantiates none: every kernel lives in the
// unit (and ECH_DN build) that defines its launcher.
#include "launch.h"

namespace ech {
template <bool DN> cudaError_t launch_jet1(const LaunchReq&, const KParams&, int, int, size_t, cudaStream_t, int*);
template <bool DN> cudaError_t launch_jet2(const LaunchReq&, const KParams&, int, int, size_t, cudaStream_t, int*);
template <bool DN> cudaError_t launch_jet3(const LaunchReq&, const KParams&, int, int, size_t, cudaStream_t, int*);
template <bool DN> cudaError_t launch_jet4(const LaunchReq&, const KParams&, int, int, size_t, cudaStream_t, int*);
template <bool DN> cudaError_t launch_jet5(const LaunchReq&, const KParams&, int, int, size_t, cudaStream_t, int*);
template <bool DN> cudaError_t launch_jet6(const LaunchReq&, const KParams&, int, int, size_t, cudaStream_t, int*);
template <bool DN> cudaError_t launch_jet7(const LaunchReq&, const KParams&, int, int, size_t, cudaStream_t, int*);
template <bool DN> cudaError_t launch_jet8(const LaunchReq&, const KParams&, int, int, size_t, cudaStream_t, int*);
template <bool DN> cudaError_t launch_jet9(const LaunchReq&, const KParams&, int, int, size_t, cudaStream_t, int*);

template <bool DN>
static cudaError_t launch_jet_dn(const LaunchReq& r, const KParams& kp, int grid, int block, size_t smem,
                                 cudaStream_t st, int* bps) {
  switch (r.K) {
    case 1: return launch_jet1<DN>(r, kp, grid, block, smem, st, bps);
    case 2: return launch_jet2<DN>(r, kp, grid, block, smem, st, bps);
    case 3: return launch_jet3<DN>(r, kp, grid, block, smem, st, bps);
    case 4: return launch_jet4<DN>(r, kp, grid, block, smem, st, bps);
    case 5: return launch_jet5<DN>(r, kp, grid, block, smem, st, bps);
    case 6: return launch_jet6<DN>(r, kp, grid, block, smem, st, bps);
    case 7: return launch_jet7<DN>(r, kp, grid, block, smem, st, bps);
    case 8: return launch_jet8<DN>(r, kp, grid, block, smem, st, bps);
    case 9: return launch_jet9<DN>(r, kp, grid, block, smem, st, bps);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_jet(const LaunchReq& r, const KParams& kp, int grid, int block, size_t smem, cudaStream_t st,
                       int* bps) {
  if (r.warp_point && r.dense && r.K == 3 && !r.rev && r.P == 1)
    return launch_jet3_warp_point(r, kp, grid, block, smem, st, bps);
  return r.dense ? launch_jet_dn<true>(r, kp, grid, block, smem, st, bps)
                 : launch_jet_dn<false>(r, kp, grid, block, smem, st, bps);
}

cudaError_t launch_sweep(const LaunchReq& r, const KParams& kp, int grid, int block, size_t smem, cudaStream_t st,
                         int* blocks_per_sm) {
  switch (r.vk) {
    case VKind::Plain:
      return r.dense ? launch_plain<true>(r, kp, grid, block, smem, st, blocks_per_sm)
                     : launch_plain<false>(r, kp, grid, block, smem, st, blocks_per_sm);
    case VKind::Dual:
      return r.dense ? launch_dual<true>(r, kp, grid, block, smem, st, blocks_per_sm)
                     : launch_dual<false>(r, kp, grid, block, smem, st, blocks_per_sm);
    case VKind::Jet: return launch_jet(r, kp, grid, block, smem, st, blocks_per_sm);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_multi_hvp(bool dense, bool f64, int P, const MultiParams& mp, int grid, int block, size_t smem,
                             cudaStream_t st, int* blocks_per_sm) {
  return dense ? launch_multi_hvp_dn<true>(f64, P, mp, grid, block, smem, st, blocks_per_sm)
               : launch_multi_hvp_dn<false>(f64, P, mp, grid, block, smem, st, blocks_per_sm);
}
}  // namespace ech
