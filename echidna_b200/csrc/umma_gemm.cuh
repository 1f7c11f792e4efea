// BF16 GEMM on the sm_100a tensor cores (tcgen05.mma, accumulator in TMEM),
// operands moved by TMA (cp.async.bulk.tensor).
//
//   C[M x N] (fp32) = A[M x K] (bf16, row-major) * B[N x K]^T (bf16, row-major)  (+ bias[N])
//
// One CTA of 128 threads computes a 128 x BN tile of C (BN = 256 when such
// tiles still give every SM one, else 128, or 64 when 128-wide tiles would
// leave most SMs idle).  K advances in blocks of 64 through a shared-memory
// ring of about 192 KiB (4 to 8 stages).  Thread 0 is the producer and the MMA
// issuer: per block it issues one 2-D TMA copy per operand, a box of 64
// K-elements (one 128-byte line per row) x 128 (or BN) rows with the 128-byte
// swizzle, which lands as the canonical K-major SWIZZLE_128B layout (rows 128 B
// apart, 8-row groups 1024 B apart, the 16-byte chunks of row r XOR-permuted by
// r mod 8), waits for the block's transaction bytes on the stage's mbarrier,
// issues four tcgen05.mma (K = 16 each: the descriptor's start advances 32 B
// within the swizzle atom) and commits them to the stage's "empty" mbarrier,
// after which the stage is refilled.  Rows past M / N are zero-filled by the TMA unit.  The epilogue
// reads the accumulator with tcgen05.ld (warp w owns TMEM lanes / rows
// 32w..32w+31).
//
// Every wait is bounded (%globaltimer, 2 s): on a timeout the CTA records
// KERR_TIMEOUT, waits (bounded) for its own outstanding copies and MMAs,
// releases its TMEM columns and returns.  No load uses cluster multicast.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "ech_types.h"

namespace ech {
namespace umma {

constexpr int kBM = 128, kBK = 64;
constexpr int kThreads = 128;
constexpr uint32_t kTileBytesA = kBM * kBK * 2;          // 16 KiB per A block (128 rows x 128 B)
// Stages: as many as fit about 192 KiB, so that the copies in flight cover a
// TMA round trip (6 stages of 32 KiB at BN = 128, 4 of 48 KiB at BN = 256).
template <int BN> struct Tile {
  static constexpr uint32_t kTileBytesB = BN * kBK * 2;
  static constexpr uint32_t kStageBytes = kTileBytesA + kTileBytesB;
  static constexpr int kStages = (int)((192u * 1024u) / kStageBytes) > 8 ? 8 : (int)((192u * 1024u) / kStageBytes);
  static constexpr uint32_t kSmemBytes = kStages * kStageBytes + 1024;  // + alignment slack
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, version 1 (sm_100), K-major with the
// 128-byte swizzle (layout type 2, bits 61-63): rows of one 128-byte line, the
// stride byte offset (SBO) between 8-row groups is 1024 B, the leading byte
// offset is unused for this layout (16 B).  The tile base is 1024-B aligned
// (base offset 0); the start may advance within a line to pick a K slice.
__device__ __forceinline__ uint64_t make_desc_sw128(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)(16u >> 4) << 16;     // LBO
  d |= (uint64_t)(1024u >> 4) << 32;   // SBO
  d |= (uint64_t)1 << 46;              // descriptor version
  d |= (uint64_t)2 << 61;              // SWIZZLE_128B
  return d;
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

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// One 2-D TMA copy (no multicast): the box at (x = K element, y = row) of the
// tensor map into shared memory, completing its bytes on `bar`.  x is a
// multiple of 64 elements (128 bytes; TMA requires 16).
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_addr(bar))
      : "memory");
}

// M rows of A / C, N rows of B / columns of C, K a multiple of 64; the tensor
// maps describe A [M][K] and B [N][K] (bf16, inner dimension K, boxes 64 x 128
// and 64 x BN, 128-byte swizzle); C row stride ldc (floats).
template <int BN>
__global__ void __launch_bounds__(kThreads) gemm_bf16_tn(const __grid_constant__ CUtensorMap tma_a,
                                                        const __grid_constant__ CUtensorMap tma_b,
                                                        float* __restrict__ C, const float* __restrict__ bias, int M,
                                                        int N, int K, int ldc, uint32_t* err) {
  using TL = Tile<BN>;
  static_assert(TL::kStages >= 2, "at least two stages");
  extern __shared__ unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t full[TL::kStages], empty[TL::kStages], fin;
  __shared__ uint32_t tmem_base;
  __shared__ int failed;
  unsigned char* sm = reinterpret_cast<unsigned char*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * BN;
  const int warp = threadIdx.x >> 5;
  const int nk = K / kBK;

  if (threadIdx.x == 0) {
    for (int s = 0; s < TL::kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(&fin, 1);
    failed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tma_a)) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tma_b)) : "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_base)),
                 "r"((uint32_t)BN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;

  if (threadIdx.x == 0) {
    const uint32_t idesc = make_idesc(kBM, BN);
    auto stage_a = [&](int s) { return sm + (size_t)s * TL::kStageBytes; };
    auto stage_b = [&](int s) { return sm + (size_t)s * TL::kStageBytes + kTileBytesA; };
    auto issue = [&](int kb) {  // block kb into stage kb % TL::kStages
      const int s = kb % TL::kStages;
      mbar_expect_tx(&full[s], TL::kStageBytes);
      tma_load_2d(stage_a(s), &tma_a, kb * kBK, m0, &full[s]);
      tma_load_2d(stage_b(s), &tma_b, kb * kBK, n0, &full[s]);
    };
    int loaded = 0, consumed = 0;  // blocks whose copies were issued / whose bytes arrived
    bool ok = true;
    for (; loaded < nk && loaded < TL::kStages; ++loaded) issue(loaded);
    for (int kb = 0; kb < nk && ok; ++kb) {
      const int s = kb % TL::kStages;
      ok = mbar_wait(&full[s], (uint32_t)((kb / TL::kStages) & 1));
      if (!ok) break;
      consumed = kb + 1;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int ks = 0; ks < kBK / 16; ++ks) {
        // K slice ks: 16 elements = 32 B into every row's line
        const uint64_t da = make_desc_sw128(smem_addr(stage_a(s)) + ks * 32u);
        const uint64_t db = make_desc_sw128(smem_addr(stage_b(s)) + ks * 32u);
        const uint32_t acc = (kb > 0 || ks > 0) ? 1u : 0u;
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(tmem),
            "l"(da), "l"(db), "r"(idesc), "r"(acc)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_addr(&empty[s]))
                   : "memory");
      // refill the stage block kb - 1 used, once its MMAs are done (block kb's run meanwhile)
      if (kb >= 1 && loaded < nk) {
        const int sp = (kb - 1) % TL::kStages;
        ok = mbar_wait(&empty[sp], (uint32_t)(((kb - 1) / TL::kStages) & 1));
        if (!ok) break;
        issue(loaded++);
      }
    }
    if (!ok) {
      failed = 1;
      // the copies still in flight land before the CTA's shared memory is given up
      for (int kb = consumed; kb < loaded; ++kb) (void)mbar_wait(&full[kb % TL::kStages], (uint32_t)((kb / TL::kStages) & 1));
    }
    // arrives once every MMA this thread issued has completed
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(&fin))
                 : "memory");
  }
  __syncthreads();
  bool ok = mbar_wait(&fin, 0u);
  ok = !__syncthreads_or(!ok || failed);
  if (ok) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int row = m0 + warp * 32 + (threadIdx.x & 31);
    // 16-byte stores need every row start and the bias 16-byte aligned
    const bool vec_ok = (ldc % 4) == 0 && ((uintptr_t)C & 15u) == 0 && ((uintptr_t)bias & 15u) == 0;
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 16) {
      uint32_t r[16];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (row < M) {
        float* crow = C + (size_t)row * ldc + n0 + c0;
        if (vec_ok && n0 + c0 + 16 <= N) {  // four 16-byte stores
#pragma unroll
          for (int j = 0; j < 16; j += 4) {
            float4 q = make_float4(__uint_as_float(r[j]), __uint_as_float(r[j + 1]), __uint_as_float(r[j + 2]),
                                   __uint_as_float(r[j + 3]));
            if (bias) {
              const float4 bq = *reinterpret_cast<const float4*>(bias + n0 + c0 + j);
              q.x = q.x + bq.x; q.y = q.y + bq.y; q.z = q.z + bq.z; q.w = q.w + bq.w;
            }
            *reinterpret_cast<float4*>(crow + j) = q;
          }
        } else {
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int col = n0 + c0 + j;
            if (col < N) crow[j] = __uint_as_float(r[j]) + (bias ? bias[col] : 0.0f);
          }
        }
      }
    }
  } else if (threadIdx.x == 0) {
    atomicOr(err, (uint32_t)KERR_TIMEOUT);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)BN) : "memory");
}

}  // namespace umma
}  // namespace ech
