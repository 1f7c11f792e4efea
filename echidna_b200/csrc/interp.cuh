// Tape interpreter kernels for sm_100a.
//
// One CTA owns a tile of TILE evaluation points (P per thread).  Every thread
// executes the same lowered instruction stream, so the opcode dispatch is
// warp-uniform while each lane works on its own points.  Per-point values live
// in a two-level slot file laid out [slot][point]:
//   * shared memory registers (hot, liveness-allocated on the host), and
//   * L2-resident global scratch slots (long-lived values, and the reverse
//     sweep's trajectory), one region per CTA reused across its tiles.
// The instruction stream is staged into shared memory chunk by chunk with
// cp.async.bulk (TMA bulk copies) signalled on mbarriers, kStages deep.
//
// Semantics per instruction follow the reference's BytecodeTape sweeps:
// forward_dispatch (src/bytecode_tape/forward.rs:11-43), reverse_sweep_core
// (src/bytecode_tape/reverse.rs:32-105) and the tangent sweeps
// (src/bytecode_tape/tangent.rs:97-262): the zero-adjoint skip, the
// zero-multiplier guard and adjoint accumulation in reverse tape order.
#pragma once
#include <stdint.h>
#include "ech_types.h"
#include "device_math.cuh"

namespace ech {

// ───────────────────────────── launch parameters ────────────────────────────
struct KParams {
  const Ins* fwd;        // forward program
  uint32_t n_fwd;
  const RIns* rev;       // reverse program (gradient / HVP kinds)
  uint32_t n_rev;
  const double* pool;    // reverse-side constant pool
  void* scratch;         // per-CTA global slot regions
  uint64_t scratch_stride_bytes;  // bytes per CTA region
  uint32_t far_slots;    // global slots before the trajectory region
  uint32_t smem_regs;    // shared-memory registers
  uint32_t tile;         // points per CTA tile
  uint64_t n_units;      // evaluation units (points, or point-direction pairs)
  uint32_t ni, no;       // inputs / outputs per unit
  // inputs
  const void* x;         // primal inputs, row-major [unit][ni] (or one row when x_bcast)
  const void* v;         // directions / seeds, row-major [unit][ni] (tangent kinds)
  int x_bcast;           // all units share x row 0
  // outputs
  void* out;             // values (or coefficient-major jets)  [unit][no]
  void* out2;            // tangents / hvp / grads
  void* out3;
  uint32_t* err;         // error word (KErr bits)
  // STDE: units = points * S; directions from host or device RNG
  uint32_t S;            // directions per point (0 = not STDE)
  int dir_mode;          // 0: v per unit, 1: v shared [S][ni], 2: device Rademacher, 3: basis e_s
  uint64_t seed;
};

// ───────────────────────────── bounded mbarrier waits ───────────────────────
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
// Waits for `parity` with a wall-clock bound; false means the wait gave up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (uint32_t it = 0; it < (1u << 30); ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 255u) == 255u && global_ns() - t0 > 2000000000ull) return false;
  }
  return false;
}

// ───────────────────────────── instruction ring ─────────────────────────────
// All threads consume the same chunks in the same order.  `seq` counts chunks
// consumed by this CTA over its lifetime and picks (stage, parity).
struct Ring {
  unsigned char* buf;   // kStages * kChunk * 32 bytes
  uint64_t* full;       // kStages mbarriers
  uint32_t seq;
  uint32_t inflight;    // bitmask of stages with an outstanding copy (thread 0)
};

__device__ __forceinline__ void ring_issue(Ring& rg, const unsigned char* prog, uint32_t nins, uint32_t chunk,
                                           uint32_t stage) {
  const uint32_t first = chunk * kChunk;
  const uint32_t cnt = min((uint32_t)kChunk, nins - first);
  const uint32_t bytes = cnt * 32u;
  uint64_t* bar = rg.full + stage;
  mbar_expect_tx(bar, bytes);
  bulk_g2s(rg.buf + (size_t)stage * kChunk * 32, prog + (size_t)first * 32, bytes, bar);
  rg.inflight |= 1u << stage;
}
// Orders this CTA's earlier generic-proxy reads of the ring before the next
// async-proxy (TMA) write into it.
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Drain outstanding copies before a CTA leaves on an error path.
__device__ __forceinline__ void ring_drain(Ring& rg) {
  if (threadIdx.x != 0) return;
  for (uint32_t k = 0; k < (uint32_t)kStages; ++k) {
    uint32_t s = (rg.seq + k) % kStages;
    if (rg.inflight & (1u << s)) {
      uint32_t parity = ((rg.seq + k) / kStages) & 1u;
      (void)mbar_wait_bounded(rg.full + s, parity);
    }
  }
  rg.inflight = 0;
}

// Runs one program through the ring, calling exec(ins_bytes) for each
// instruction.  Returns false if a wait gave up (all threads agree).
template <class Exec>
__device__ __forceinline__ bool run_program(Ring& rg, const unsigned char* prog, uint32_t nins, uint32_t* err,
                                            Exec&& exec) {
  const uint32_t nchunks = (nins + kChunk - 1) / kChunk;
  if (nchunks == 0) return true;
  if (threadIdx.x == 0) {
    fence_proxy_async();
    const uint32_t pre = min((uint32_t)kStages, nchunks);
    for (uint32_t c = 0; c < pre; ++c) ring_issue(rg, prog, nins, c, (rg.seq + c) % kStages);
  }
  for (uint32_t c = 0; c < nchunks; ++c) {
    const uint32_t stage = rg.seq % kStages;
    const uint32_t parity = (rg.seq / kStages) & 1u;
    const bool ok = mbar_wait_bounded(rg.full + stage, parity);
    if (ok) {
      if (threadIdx.x == 0) rg.inflight &= ~(1u << stage);
      const uint32_t cnt = min((uint32_t)kChunk, nins - c * kChunk);
      const unsigned char* base = rg.buf + (size_t)stage * kChunk * 32;
#pragma unroll 1
      for (uint32_t k = 0; k < cnt; ++k) exec(base + k * 32u);
    }
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) atomicOr(err, (uint32_t)KERR_TIMEOUT);
      ring_drain(rg);
      return false;
    }
    rg.seq += 1;
    if (threadIdx.x == 0 && c + kStages < nchunks) {
      fence_proxy_async();
      ring_issue(rg, prog, nins, c + kStages, stage);
    }
  }
  return true;
}

// ───────────────────────────── slot file access ─────────────────────────────
template <class V, int P> struct Slots {
  V* sm;          // shared registers: sm[reg * tile + col + p]
  V* gs;          // global scratch:   gs[slot * tile + col + p]
  uint32_t tile;
  uint32_t col;

  __device__ __forceinline__ V ld(uint8_t mode, uint32_t idx, int p) const {
    if (mode == M_SMEM) return sm[(size_t)idx * tile + col + p];
    return gs[(size_t)idx * tile + col + p];
  }
  __device__ __forceinline__ void st(uint8_t mode, uint32_t idx, int p, const V& v) const {
    if (mode == M_SMEM) sm[(size_t)idx * tile + col + p] = v;
    else if (mode == M_GLOB) gs[(size_t)idx * tile + col + p] = v;
  }
};

// Per-kind input construction and output handling; the primary template is
// the plain-value kind (forward, gradient).
template <class T> struct Lane {
  using S = T;
  static __device__ __forceinline__ T make_input(const KParams& kp, uint64_t u, uint32_t i, bool valid) {
    if (!valid) return T(0);
    const T* x = (const T*)kp.x;
    return x[(kp.x_bcast ? 0 : u) * kp.ni + i];
  }
  static __device__ __forceinline__ void store_output(const KParams& kp, uint64_t u, uint32_t j, const T& val, bool valid) {
    if (valid) ((T*)kp.out)[u * kp.no + j] = val;
  }
};
template <class T> struct Lane<dm::Dual<T>> {
  using S = T;
  static __device__ __forceinline__ dm::Dual<T> make_input(const KParams& kp, uint64_t u, uint32_t i, bool valid) {
    if (!valid) return {T(0), T(0)};
    const T* x = (const T*)kp.x;
    const T* v = (const T*)kp.v;
    return {x[(kp.x_bcast ? 0 : u) * kp.ni + i], v[u * kp.ni + i]};
  }
  static __device__ __forceinline__ void store_output(const KParams& kp, uint64_t u, uint32_t j, const dm::Dual<T>& val,
                                                      bool valid) {
    if (!valid) return;
    if (kp.out) ((T*)kp.out)[u * kp.no + j] = val.re;
    if (kp.out2) ((T*)kp.out2)[u * kp.no + j] = val.eps;
  }
};

// Direction component for STDE units (point = u / S, direction = u % S).
__device__ __forceinline__ uint32_t philox_bits(uint64_t seed, uint64_t point, uint32_t dir, uint32_t i);

template <class T, int K> struct Lane<dm::Jet<T, K>> {
  using S = T;
  static __device__ __forceinline__ T dir_component(const KParams& kp, uint64_t u, uint32_t i) {
    const T* v = (const T*)kp.v;
    if (kp.S == 0 || kp.dir_mode == 0) return v[u * kp.ni + i];
    const uint64_t pt = u / kp.S;
    const uint32_t s = (uint32_t)(u - pt * kp.S);
    if (kp.dir_mode == 1) return v[(uint64_t)s * kp.ni + i];
    if (kp.dir_mode == 3) return (i == s) ? T(1) : T(0);
    return (philox_bits(kp.seed, pt, s, i) & 1u) ? T(1) : T(-1);
  }
  static __device__ __forceinline__ dm::Jet<T, K> make_input(const KParams& kp, uint64_t u, uint32_t i, bool valid) {
    dm::Jet<T, K> j;
#pragma unroll
    for (int k = 0; k < K; ++k) j.c[k] = T(0);
    if (!valid) return j;
    const T* x = (const T*)kp.x;
    const uint64_t xrow = kp.x_bcast ? 0 : (kp.S ? u / kp.S : u);
    j.c[0] = x[xrow * kp.ni + i];
    if (K > 1) j.c[1] = dir_component(kp, u, i);
    return j;
  }
  static __device__ __forceinline__ void store_output(const KParams& kp, uint64_t u, uint32_t j, const dm::Jet<T, K>& val,
                                                      bool valid) {
    if (!valid) return;
    // coefficient-major layout: out[k][u * no + j] (TaylorKthBatchResult)
    T* o = (T*)kp.out;
    const uint64_t plane = kp.n_units * kp.no;
#pragma unroll
    for (int k = 0; k < K; ++k) o[(uint64_t)k * plane + u * kp.no + j] = val.c[k];
  }
};

// Philox-4x32-10 (Salmon et al., SC'11) keyed by (seed); counter (point, dir, i).
__device__ __forceinline__ uint32_t philox_bits(uint64_t seed, uint64_t point, uint32_t dir, uint32_t i) {
  uint32_t c0 = (uint32_t)point, c1 = (uint32_t)(point >> 32), c2 = dir, c3 = i;
  uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c0;
}

// ───────────────────────────── forward executor ─────────────────────────────
template <class V, int P> struct FwdExec {
  using Kd = typename dm::KindOf<V>::K;
  const KParams& kp;
  Slots<V, P> sl;
  uint64_t unit0;        // unit of point p = unit0 + p
  V* traj;               // trajectory region of this CTA (gs + G*tile)
  bool valid[P];

  __device__ __forceinline__ V opnd(uint8_t mode, uint32_t idx, double imm, int p) const {
    if (mode == M_IMM) return dm::VT<V>::cst(imm);
    return sl.ld(mode, idx, p);
  }
  __device__ __forceinline__ void put(const Ins& in, int p, const V& r) const {
    sl.st(in.md, in.d, p, r);
    if (in.save != kNone) traj[(size_t)in.save * sl.tile + sl.col + p] = r;
  }

  __device__ __forceinline__ void operator()(const unsigned char* raw) const {
    const Ins in = *reinterpret_cast<const Ins*>(raw);
    switch (in.opc) {
      case XI_LDIN:
#pragma unroll
        for (int p = 0; p < P; ++p) put(in, p, Lane<V>::make_input(kp, unit0 + p, (uint32_t)in.aux, valid[p]));
        return;
      case XI_STOUT:
#pragma unroll
        for (int p = 0; p < P; ++p)
          Lane<V>::store_output(kp, unit0 + p, (uint32_t)in.aux, opnd(in.ma, in.a, in.imm, p), valid[p]);
        return;
      case XI_MOV:
#pragma unroll
        for (int p = 0; p < P; ++p) put(in, p, opnd(in.ma, in.a, in.imm, p));
        return;
      default: break;
    }
    V a[P], b[P], r[P];
#pragma unroll
    for (int p = 0; p < P; ++p) {
      a[p] = opnd(in.ma, in.a, in.imm, p);
      b[p] = (in.mb == M_NONE) ? Kd::c(0) : opnd(in.mb, in.b, in.imm, p);
    }
#pragma unroll
    for (int p = 0; p < P; ++p) r[p] = dm::eval_forward<V>(in.opc, a[p], b[p], in.aux);
#pragma unroll
    for (int p = 0; p < P; ++p) put(in, p, r[p]);
  }
};

// ───────────────────────────── reverse executor ─────────────────────────────
// Gradient outputs: plain kind -> out2[u][k]; Dual kind -> out2 (re) and out3 (eps).
template <class V> struct GradOut {
  static __device__ __forceinline__ void store(const KParams& kp, uint64_t u, uint32_t k, const V& g, bool valid) {
    if (valid) ((V*)kp.out2)[u * kp.ni + k] = g;
  }
};
template <class T> struct GradOut<dm::Dual<T>> {
  static __device__ __forceinline__ void store(const KParams& kp, uint64_t u, uint32_t k, const dm::Dual<T>& g,
                                               bool valid) {
    if (!valid) return;
    ((T*)kp.out2)[u * kp.ni + k] = g.re;
    ((T*)kp.out3)[u * kp.ni + k] = g.eps;
  }
};

template <class V, int P> struct RevExec {
  using Kd = typename dm::KindOf<V>::K;
  const KParams& kp;
  Slots<V, P> sl;
  uint64_t unit0;
  const V* traj;
  bool valid[P];

  __device__ __forceinline__ V value(uint32_t idx, bool imm, int p) const {
    if (idx == kNone) return Kd::c(0);
    if (imm) return dm::VT<V>::cst(kp.pool[idx]);
    return traj[(size_t)idx * sl.tile + sl.col + p];
  }

  __device__ __forceinline__ void operator()(const unsigned char* raw) const {
    const RIns in = *reinterpret_cast<const RIns*>(raw);
    const uint8_t mr = (in.flags & RF_R_GLOB) ? M_GLOB : M_SMEM;
    if (in.opc == XI_SEED) {
#pragma unroll
      for (int p = 0; p < P; ++p) sl.st(mr, in.r, p, Kd::c(1));
      return;
    }
    if (in.opc == XI_STGRAD) {
#pragma unroll
      for (int p = 0; p < P; ++p) {
        const V g = (in.r == kNone) ? Kd::c(0) : sl.ld(mr, in.r, p);
        GradOut<V>::store(kp, unit0 + p, (uint32_t)in.aux, g, valid[p]);
      }
      return;
    }
    V adj[P], da[P], db[P];
    bool live[P];
#pragma unroll
    for (int p = 0; p < P; ++p) {
      adj[p] = sl.ld(mr, in.r, p);
      live[p] = !Kd::all_zero(adj[p]);
    }
#pragma unroll
    for (int p = 0; p < P; ++p) {
      const V va = value(in.va, (in.flags & RF_VA_IMM) != 0, p);
      const V vb = value(in.vb, (in.flags & RF_VB_IMM) != 0, p);
      const V vr = value(in.vr, false, p);
      dm::reverse_partials<V>(in.opc, va, vb, vr, in.aux, da[p], db[p]);
    }
    if (in.flags & RF_HAS_A) {
      const uint8_t ma = (in.flags & RF_A_GLOB) ? M_GLOB : M_SMEM;
      const bool init = (in.flags & RF_A_INIT) != 0;
#pragma unroll
      for (int p = 0; p < P; ++p) {
        const bool hit = live[p] && !Kd::all_zero(da[p]);
        if (init) {
          const V z = Kd::c(0);
          sl.st(ma, in.a, p, hit ? Kd::add(z, Kd::mul(da[p], adj[p])) : z);
        } else if (hit) {
          sl.st(ma, in.a, p, Kd::add(sl.ld(ma, in.a, p), Kd::mul(da[p], adj[p])));
        }
      }
    }
    if (in.flags & RF_HAS_B) {
      const uint8_t mb = (in.flags & RF_B_GLOB) ? M_GLOB : M_SMEM;
      const bool init = (in.flags & RF_B_INIT) != 0;
#pragma unroll
      for (int p = 0; p < P; ++p) {
        const bool hit = live[p] && !Kd::all_zero(db[p]);
        if (init) {
          const V z = Kd::c(0);
          sl.st(mb, in.b, p, hit ? Kd::add(z, Kd::mul(db[p], adj[p])) : z);
        } else if (hit) {
          sl.st(mb, in.b, p, Kd::add(sl.ld(mb, in.b, p), Kd::mul(db[p], adj[p])));
        }
      }
    }
  }

};

}  // namespace ech

namespace ech {

// ───────────────────────────── the sweep kernel ─────────────────────────────
// REV = false: forward program only (forward values, JVP, Taylor jets).
// REV = true : forward program with trajectory saves, then the reverse program
//              (gradient for plain values, HVP for Dual values).
template <class V, int P, bool REV>
__global__ void __launch_bounds__(256) sweep_kernel(KParams kp) {
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  __shared__ __align__(8) uint64_t full[kStages];
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) mbar_init(&full[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  Ring rg{smem_dyn, full, 0u, 0u};
  V* regs = reinterpret_cast<V*>(smem_dyn + (size_t)kStages * kChunk * 32);
  const uint32_t tile = kp.tile;
  const uint32_t col = threadIdx.x * P;
  V* gs = reinterpret_cast<V*>(reinterpret_cast<unsigned char*>(kp.scratch) + blockIdx.x * kp.scratch_stride_bytes);
  V* traj = gs + (size_t)kp.far_slots * tile;
  const uint64_t ntiles = (kp.n_units + tile - 1) / tile;
  for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const uint64_t unit0 = t * tile + col;
    FwdExec<V, P> fx{kp, Slots<V, P>{regs, gs, tile, col}, unit0, traj, {}};
#pragma unroll
    for (int p = 0; p < P; ++p) fx.valid[p] = unit0 + p < kp.n_units;
    if (!run_program(rg, reinterpret_cast<const unsigned char*>(kp.fwd), kp.n_fwd, kp.err, fx)) return;
    if (REV) {
      RevExec<V, P> rx{kp, Slots<V, P>{regs, gs, tile, col}, unit0, traj, {}};
#pragma unroll
      for (int p = 0; p < P; ++p) rx.valid[p] = fx.valid[p];
      if (!run_program(rg, reinterpret_cast<const unsigned char*>(kp.rev), kp.n_rev, kp.err, rx)) return;
    }
  }
}

}  // namespace ech
