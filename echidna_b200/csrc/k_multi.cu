// Many-tape persistent HVP sweep (gradient + per-point HVP over Dual values).
#include "k_common.cuh"

namespace ech {

template <class V, int P, bool DN>
static cudaError_t launch_multi_one(const MultiParams& mp, int grid, int block, size_t smem, cudaStream_t st,
                                    int* bps) {
  auto fn = multi_sweep_kernel<V, P, DN>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  if (grid == 0) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, fn, block, smem);
  fn<<<grid, block, smem, st>>>(mp);
  return cudaGetLastError();
}

template <class V, bool DN>
static cudaError_t launch_multi_v(int P, const MultiParams& mp, int grid, int block, size_t smem, cudaStream_t st,
                                  int* bps) {
  switch (P) {
    case 1: return launch_multi_one<V, 1, DN>(mp, grid, block, smem, st, bps);
    case 2: return launch_multi_one<V, 2, DN>(mp, grid, block, smem, st, bps);
    case 4: return launch_multi_one<V, 4, DN>(mp, grid, block, smem, st, bps);
    default: return cudaErrorInvalidValue;
  }
}

template <bool DN>
cudaError_t launch_multi_hvp_dn(bool f64, int P, const MultiParams& mp, int grid, int block, size_t smem,
                                cudaStream_t st, int* blocks_per_sm) {
  return f64 ? launch_multi_v<dm::Dual<double>, DN>(P, mp, grid, block, smem, st, blocks_per_sm)
             : launch_multi_v<dm::Dual<float>, DN>(P, mp, grid, block, smem, st, blocks_per_sm);
}
ECH_INSTANTIATE_DN(launch_multi_hvp_dn, bool, int, const MultiParams&, int, int, size_t, cudaStream_t, int*)

}  // namespace ech
