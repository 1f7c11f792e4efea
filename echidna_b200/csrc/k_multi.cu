// Many-tape persistent HVP sweep (gradient + per-point HVP over Dual values).
#include "interp.cuh"
#include "launch.h"

namespace ech {

template <class V, int P>
static cudaError_t launch_multi_one(const MultiParams& mp, int grid, int block, size_t smem, cudaStream_t st,
                                    int* bps) {
  auto fn = multi_sweep_kernel<V, P>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  if (grid == 0) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, fn, block, smem);
  fn<<<grid, block, smem, st>>>(mp);
  return cudaGetLastError();
}

template <class V>
static cudaError_t launch_multi_v(int P, const MultiParams& mp, int grid, int block, size_t smem, cudaStream_t st,
                                  int* bps) {
  switch (P) {
    case 1: return launch_multi_one<V, 1>(mp, grid, block, smem, st, bps);
    case 2: return launch_multi_one<V, 2>(mp, grid, block, smem, st, bps);
    case 4: return launch_multi_one<V, 4>(mp, grid, block, smem, st, bps);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_multi_hvp(bool f64, int P, const MultiParams& mp, int grid, int block, size_t smem,
                             cudaStream_t st, int* blocks_per_sm) {
  return f64 ? launch_multi_v<dm::Dual<double>>(P, mp, grid, block, smem, st, blocks_per_sm)
             : launch_multi_v<dm::Dual<float>>(P, mp, grid, block, smem, st, blocks_per_sm);
}

}  // namespace ech
