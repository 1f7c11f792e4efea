// BF16 GEMM on the sm_100a tensor cores (tcgen05.mma, accumulator in TMEM).
//
//   C[M x N] (fp32) = A[M x K] (bf16, row-major) * B[N x K]^T (bf16, row-major)  (+ bias[N])
//
// One CTA of 128 threads computes a 128 x 128 tile of C.  K advances in blocks
// of 64: every thread copies its share of the A and B blocks into shared memory
// in the canonical K-major, no-swizzle layout (8-row x 16-byte core matrices;
// K-adjacent core matrices 128 B apart, 8-row groups 1024 B apart), thread 0
// issues four tcgen05.mma (K = 16 each) and commits them to an mbarrier; the
// next block is copied into the other buffer meanwhile.  The epilogue reads the
// accumulator back with tcgen05.ld (warp w owns TMEM lanes / rows 32w..32w+31).
//
// Every wait is bounded (%globaltimer, 2 s): on a timeout the CTA records
// KERR_TIMEOUT, waits (bounded) for its own outstanding MMAs, releases its TMEM
// columns and returns.  No load uses cluster multicast.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

#include "ech_types.h"

namespace ech {
namespace umma {

constexpr int kBM = 128, kBN = 128, kBK = 64;
constexpr int kThreads = 128;
constexpr uint32_t kTileBytes = kBM * kBK * 2;           // 16 KiB per operand block
constexpr uint32_t kSmemBytes = 4 * kTileBytes + 1024;   // A, B double-buffered + alignment slack
constexpr uint32_t kTmemCols = 128;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: K-major, no swizzle, version 1 (sm_100).
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version
  return d;               // base offset 0, relative LBO, layout SWIZZLE_NONE
}

// Instruction descriptor, kind::f16: D fp32, A and B bf16, both K-major.
__host__ __device__ constexpr uint32_t make_idesc(int M, int N) {
  return (1u << 4)                       // D format: F32
         | (1u << 7)                     // A format: BF16
         | (1u << 10)                    // B format: BF16
         | ((uint32_t)(N >> 3) << 17)    // N / 8
         | ((uint32_t)(M >> 4) << 24);   // M / 16
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t now_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  if (mbar_try(bar, parity)) return true;
  const uint64_t t0 = now_ns();
  for (uint32_t it = 0; it < (1u << 30); ++it) {
    if (mbar_try(bar, parity)) return true;
    if ((it & 255u) == 255u && now_ns() - t0 > 2000000000ull) return false;
  }
  return false;
}

// Copies rows [r0, r0+128) x k-block [k0, k0+64) of a row-major bf16 matrix
// with `ld` elements per row into the canonical layout at `dst`.  Rows past
// `rows` are zero-filled.  Each thread moves 16-byte chunks.
__device__ __forceinline__ void load_block(unsigned char* dst, const __nv_bfloat16* src, int rows, int ld, int r0,
                                           int k0) {
  // 128 rows x 8 chunks of 16 B = 1024 chunks; 8 per thread
#pragma unroll
  for (int i = 0; i < (kBM * kBK / 8) / kThreads; ++i) {
    const int c = threadIdx.x + i * kThreads;
    const int r = c >> 3, kc = c & 7;
    uint4 v = make_uint4(0, 0, 0, 0);
    const int gr = r0 + r;
    if (gr < rows) v = *reinterpret_cast<const uint4*>(src + (size_t)gr * ld + k0 + kc * 8);
    const uint32_t off = (uint32_t)(r >> 3) * 1024u + (uint32_t)kc * 128u + (uint32_t)(r & 7) * 16u;
    *reinterpret_cast<uint4*>(dst + off) = v;
  }
}

// M rows of A / C, N rows of B / columns of C, K a multiple of 64; lda, ldb in
// elements (multiples of 8); C row stride ldc (floats).
__global__ void __launch_bounds__(kThreads) gemm_bf16_tn(const __nv_bfloat16* __restrict__ A,
                                                        const __nv_bfloat16* __restrict__ B,
                                                        float* __restrict__ C, const float* __restrict__ bias, int M,
                                                        int N, int K, int lda, int ldb, int ldc, uint32_t* err) {
  extern __shared__ unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t done[2];
  __shared__ uint32_t tmem_base;
  unsigned char* sm = reinterpret_cast<unsigned char*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
  const int warp = threadIdx.x >> 5;

  if (threadIdx.x == 0) {
    mbar_init(&done[0], 1);
    mbar_init(&done[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_base)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;

  const uint32_t idesc = make_idesc(kBM, kBN);
  const int nk = K / kBK;
  uint32_t issued0 = 0, issued1 = 0;  // commits per buffer (parity of the latest = (count - 1) & 1)
  bool ok = true;
  for (int kb = 0; kb < nk && ok; ++kb) {
    const int buf = kb & 1;
    // the buffer's previous MMAs (block kb - 2) must be done before it is overwritten
    if (kb >= 2) ok = mbar_wait(&done[buf], (uint32_t)((kb / 2 - 1) & 1));
    if (__syncthreads_or(!ok)) { ok = false; break; }
    unsigned char* sa = sm + buf * kTileBytes;
    unsigned char* sb = sm + (2 + buf) * kTileBytes;
    load_block(sa, A, M, lda, m0, kb * kBK);
    load_block(sb, B, N, ldb, n0, kb * kBK);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int ks = 0; ks < kBK / 16; ++ks) {
        const uint64_t da = make_desc(smem_addr(sa) + ks * 256u, 128u, 1024u);
        const uint64_t db = make_desc(smem_addr(sb) + ks * 256u, 128u, 1024u);
        const uint32_t acc = (kb > 0 || ks > 0) ? 1u : 0u;
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(tmem),
            "l"(da), "l"(db), "r"(idesc), "r"(acc)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_addr(&done[buf]))
                   : "memory");
    }
    if (buf) issued1 += 1;
    else issued0 += 1;
  }
  // wait for the last block's MMAs (a commit covers every earlier MMA of the thread)
  if (ok && nk > 0) {
    const int last = (nk - 1) & 1;
    ok = mbar_wait(&done[last], ((last ? issued1 : issued0) - 1) & 1);
  }
  ok = !__syncthreads_or(!ok);
  if (ok) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int row = m0 + warp * 32 + (threadIdx.x & 31);
#pragma unroll 1
    for (int c0 = 0; c0 < kBN; c0 += 16) {
      uint32_t r[16];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (row < M) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int col = n0 + c0 + j;
          if (col < N) C[(size_t)row * ldc + col] = __uint_as_float(r[j]) + (bias ? bias[col] : 0.0f);
        }
      }
    }
  } else {
    if (threadIdx.x == 0) atomicOr(err, (uint32_t)KERR_TIMEOUT);
    // let whatever this CTA issued finish (bounded) before the columns are released
    if (issued0) (void)mbar_wait(&done[0], (issued0 - 1) & 1);
    if (issued1) (void)mbar_wait(&done[1], (issued1 - 1) & 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

}  // namespace umma
}  // namespace ech
