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
// Instructions carry byte offsets from the thread's column base and, for the
// common shapes, mode-specialised opcodes (see DOp in ech_types.h), so a
// typical op is: two vector loads, the arithmetic, one vector store.
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
#include "rng.cuh"

namespace ech {

// ───────────────────────────── launch parameters ────────────────────────────
struct KParams {
  const DIns* fwd;       // forward program (device encoding; chain terms inline)
  uint32_t n_fwd;        // records
  const DRIns* rev;      // reverse program (gradient / HVP kinds)
  uint32_t n_rev;
  void* scratch;         // per-CTA global slot regions
  uint64_t scratch_stride_bytes;  // bytes per CTA region
  uint32_t far_slots;    // global slots before the trajectory region
  uint32_t smem_regs;    // shared-memory registers
  uint32_t traj_smem;    // 1: the trajectory rows follow the shared registers (else in the global scratch)
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
  int dir_mode;          // 0: v per unit, 1: v shared [S][ni], 2: device Rademacher, 3: basis e_s,
                         // 4: basis e_{v[u]} (v: one uint32 coordinate per unit),
                         // 5: slot-seeded jets (v: one uint32 entry per unit into seed_off / seed_items)
  uint64_t seed;
  const uint32_t* seed_off;  // dir_mode 5: entry e's seeds are seed_items[seed_off[e] .. seed_off[e+1])
  const void* seed_items;    // SlotSeed records
  uint32_t dir_bits;         // dir_mode 2 with input-direct terms: byte offset in shared memory of the
                             // tile's direction signs, [ceil(ni/32) words][tile units] (0: none)
  uint32_t traj_slots;       // trajectory slots (bounds of the checked build)
  uint32_t compensated;      // order-3 jets: Neumaier-compensated additions in fused chains (an FP32
                             // option of the batch Laplacian; results then differ from the
                             // reference's rounding)
};

// ───────────────────────────── device bounds checks ─────────────────────────
// Built with ECH_DEVICE_BOUNDS (the library variant libechidna_b200_bounds.so),
// every slot access of the sweeps checks its offset against its region (shared
// registers, global far slots, trajectory) and every input / output / gradient
// index against the unit's sizes.  An access out of its region sets KERR_BOUNDS
// in the error word and goes to the thread's first shared register instead (no
// fault); ech_ctx_synchronize reports it.  Without the macro the checks compile
// to plain pointer arithmetic.
#ifdef ECH_DEVICE_BOUNDS
constexpr bool kBoundsChecked = true;
#else
constexpr bool kBoundsChecked = false;
#endif
__device__ __forceinline__ unsigned char* bounded(unsigned char* base, uint32_t off, uint64_t limit,
                                                  unsigned char* fallback, uint32_t* err) {
  if constexpr (kBoundsChecked) {
    if ((uint64_t)off >= limit) {
      atomicOr(err, (uint32_t)KERR_BOUNDS);
      return fallback;
    }
  }
  return base + off;
}
__device__ __forceinline__ bool index_ok(uint32_t i, uint32_t n, uint32_t* err) {
  if constexpr (kBoundsChecked) {
    if (i >= n) {
      atomicOr(err, (uint32_t)KERR_BOUNDS);
      return false;
    }
  }
  return true;
}

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
// consumed by this CTA over its lifetime and picks (stage, parity).  Records are
// REC bytes (32 forward, 48 reverse); a stage holds kChunk records.
struct Ring {
  unsigned char* buf;   // kStages stages of kChunk * 48 bytes
  uint64_t* full;       // kStages mbarriers
  uint32_t seq;
  uint32_t inflight;    // bitmask of stages with an outstanding copy (thread 0)
};

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

template <int REC>
__device__ __forceinline__ void ring_issue(Ring& rg, const unsigned char* prog, uint32_t nins, uint32_t chunk,
                                           uint32_t stage) {
  const uint32_t first = chunk * kChunk;
  const uint32_t cnt = min((uint32_t)kChunk, nins - first);
  const uint32_t bytes = cnt * (uint32_t)REC;
  uint64_t* bar = rg.full + stage;
  mbar_expect_tx(bar, bytes);
  bulk_g2s(rg.buf + (size_t)stage * kChunk * 48, prog + (size_t)first * REC, bytes, bar);
  rg.inflight |= 1u << stage;
}

// Drain outstanding copies before a CTA leaves on an error path.
__device__ __forceinline__ void ring_drain(Ring& rg) {
  if (threadIdx.x != 0) return;
  for (uint32_t k = 0; k < (uint32_t)kStages; ++k) {
    const uint32_t s = (rg.seq + k) % kStages;
    if (rg.inflight & (1u << s)) {
      const uint32_t parity = ((rg.seq + k) / kStages) & 1u;
      (void)mbar_wait_bounded(rg.full + s, parity);
    }
  }
  rg.inflight = 0;
}

// Makes chunk `c` of a program current: waits (bounded) for its copy, and
// once every thread has passed the barrier (so all are done with chunk c-1)
// refills chunk c-1's stage with chunk c-1+kStages.  Returns the chunk's
// record count, 0 when a wait gave up or the program ended early (every thread
// sees the same value).  Out of line: it runs once per chunk.
struct Chunk {
  const unsigned char* base;
  uint32_t count;
};
template <int REC>
__device__ __noinline__ Chunk ring_chunk(Ring* rg, const unsigned char* prog, uint32_t nins, uint32_t c,
                                         uint32_t* err) {
  const uint32_t nchunks = (nins + kChunk - 1) / kChunk;
  if (c >= nchunks) {  // a chain ran past the end of its program
    if (threadIdx.x == 0) atomicOr(err, (uint32_t)KERR_BADINS);
    ring_drain(*rg);
    return {nullptr, 0u};
  }
  const uint32_t stage = rg->seq % kStages;
  const bool ok = mbar_wait_bounded(rg->full + stage, (rg->seq / kStages) & 1u);
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x == 0) atomicOr(err, (uint32_t)KERR_TIMEOUT);
    ring_drain(*rg);
    return {nullptr, 0u};
  }
  if (threadIdx.x == 0) {
    rg->inflight &= ~(1u << stage);
    if (c > 0 && c - 1 + kStages < nchunks) {
      fence_proxy_async();
      ring_issue<REC>(*rg, prog, nins, c - 1 + kStages, (rg->seq + kStages - 1) % kStages);
    }
  }
  rg->seq += 1;
  return {rg->buf + (size_t)stage * kChunk * 48, min((uint32_t)kChunk, nins - c * kChunk)};
}

// The records of one program in order, read from the ring.  Executors pull
// the records that follow an instruction (a chain's terms) with next(); every
// thread pulls the same records.  A record's fields must be read before the
// next pull, which may recycle its stage.
template <int REC>
struct Stream {
  Ring* rg;
  const unsigned char* prog;
  uint32_t nins;
  uint32_t* err;
  const unsigned char* rec;  // next record in the current chunk
  uint32_t left;             // records left in the current chunk
  uint32_t chunk;            // chunks made current so far
  bool failed;

  __device__ __forceinline__ const unsigned char* next() {
    if (left == 0) {
      const Chunk ch = ring_chunk<REC>(rg, prog, nins, chunk, err);
      if (ch.count == 0) {
        failed = true;
        return nullptr;
      }
      chunk += 1;
      rec = ch.base;
      left = ch.count;
    }
    const unsigned char* r = rec;
    rec += REC;
    left -= 1;
    return r;
  }
};

// Runs one program through the ring: exec(record, stream) per instruction
// (chain instructions pull their terms from the stream).  Returns false if a
// wait gave up or the program is malformed (all threads agree).
template <int REC, class Exec>
__device__ __forceinline__ bool run_program(Ring& rg, const unsigned char* prog, uint32_t nins, uint32_t* err,
                                            Exec& exec) {
  if (nins == 0) return true;
  if (threadIdx.x == 0) {
    fence_proxy_async();
    const uint32_t pre = min((uint32_t)kStages, (nins + kChunk - 1) / kChunk);
    for (uint32_t c = 0; c < pre; ++c) ring_issue<REC>(rg, prog, nins, c, (rg.seq + c) % kStages);
  }
  Stream<REC> st{&rg, prog, nins, err, nullptr, 0u, 0u, false};
  const uint32_t total_chunks = (nins + kChunk - 1) / kChunk;
#pragma unroll 1
  while (st.chunk < total_chunks || st.left > 0) {
    const unsigned char* r = st.next();
    if (r == nullptr || !exec(r, st)) return false;
  }
  // every thread is done with the last chunk before the ring is refilled
  __syncthreads();
  return true;
}

// ───────────────────────────── column access ────────────────────────────────
// A thread owns P consecutive points of every slot row, so the P values of one
// slot are contiguous and move with the widest aligned vector access.
__host__ __device__ constexpr int gcd_c(int a, int b) { return b == 0 ? a : gcd_c(b, a % b); }

template <class V, int P> struct Col {
  using T = typename dm::VT<V>::S;
  static constexpr int N = (int)(sizeof(V) * P / sizeof(T));  // scalars per column access
  static constexpr int B = N * (int)sizeof(T);
  static __device__ __forceinline__ void ld(const unsigned char* p, V (&v)[P]) {
    T* t = reinterpret_cast<T*>(v);
    if constexpr (sizeof(T) == 4 && B % 16 == 0) {
#pragma unroll
      for (int i = 0; i < N / 4; ++i) {
        const float4 q = reinterpret_cast<const float4*>(p)[i];
        t[4 * i] = q.x; t[4 * i + 1] = q.y; t[4 * i + 2] = q.z; t[4 * i + 3] = q.w;
      }
    } else if constexpr (sizeof(T) == 4 && B % 8 == 0) {
#pragma unroll
      for (int i = 0; i < N / 2; ++i) {
        const float2 q = reinterpret_cast<const float2*>(p)[i];
        t[2 * i] = q.x; t[2 * i + 1] = q.y;
      }
    } else if constexpr (sizeof(T) == 8 && B % 16 == 0) {
#pragma unroll
      for (int i = 0; i < N / 2; ++i) {
        const double2 q = reinterpret_cast<const double2*>(p)[i];
        t[2 * i] = q.x; t[2 * i + 1] = q.y;
      }
    } else {
#pragma unroll
      for (int i = 0; i < N; ++i) t[i] = reinterpret_cast<const T*>(p)[i];
    }
  }
  static __device__ __forceinline__ void st(unsigned char* p, const V (&v)[P]) {
    const T* t = reinterpret_cast<const T*>(v);
    if constexpr (sizeof(T) == 4 && B % 16 == 0) {
#pragma unroll
      for (int i = 0; i < N / 4; ++i)
        reinterpret_cast<float4*>(p)[i] = make_float4(t[4 * i], t[4 * i + 1], t[4 * i + 2], t[4 * i + 3]);
    } else if constexpr (sizeof(T) == 4 && B % 8 == 0) {
#pragma unroll
      for (int i = 0; i < N / 2; ++i) reinterpret_cast<float2*>(p)[i] = make_float2(t[2 * i], t[2 * i + 1]);
    } else if constexpr (sizeof(T) == 8 && B % 16 == 0) {
#pragma unroll
      for (int i = 0; i < N / 2; ++i) reinterpret_cast<double2*>(p)[i] = make_double2(t[2 * i], t[2 * i + 1]);
    } else {
#pragma unroll
      for (int i = 0; i < N; ++i) reinterpret_cast<T*>(p)[i] = t[i];
    }
  }
};

// Constant of a linear-combination term record: programs for f32 values carry
// it already rounded to f32 (the low word of the 8-byte field), f64 programs
// the double.
template <class V>
__device__ __forceinline__ V lc_const(uint32_t lo, uint32_t hi) {
  if constexpr (sizeof(typename dm::VT<V>::S) == 4) return dm::VT<V>::cst_s(__uint_as_float(lo));
  else return dm::VT<V>::cst(__hiloint2double((int)hi, (int)lo));
}

// Scalar constant of a linear-combination term record (see lc_const).
template <class T>
__device__ __forceinline__ T lc_scalar(uint32_t lo, uint32_t hi) {
  if constexpr (sizeof(T) == 4) return __uint_as_float(lo);
  else return __hiloint2double((int)hi, (int)lo);
}

// Order of a jet value kind (0 for the other kinds).
template <class V> struct JetOrder { static constexpr int K = 0; };
template <class T, int K_> struct JetOrder<dm::Jet<T, K_>> { static constexpr int K = K_; };

// x * 0 + z with one rounding: z unchanged (+0 stays +0) when x is finite, NaN otherwise.
__device__ __forceinline__ float fma_zero(float x, float z) { return __fmaf_rn(x, 0.0f, z); }
__device__ __forceinline__ double fma_zero(double x, double z) { return __fma_rn(x, 0.0, z); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }

// s + x with Neumaier's compensation (Neumaier, 1974): the rounding error of
// the addition accumulates in c.
template <class T>
__device__ __forceinline__ void neumaier_add(T& s, T& c, T x) {
  const T t = s + x;
  c = c + ((fabs(s) >= fabs(x)) ? ((s - t) + x) : ((x - t) + s));
  s = t;
}

// Dual value kind detection (the dense group's shared zero product).
template <class V> struct IsDual { static constexpr bool v = false; };
template <class T> struct IsDual<dm::Dual<T>> { static constexpr bool v = true; };

// Per-kind input construction and output handling; the primary template is
// the plain-value kind (forward, gradient).  `Info` is what a unit's inputs
// depend on beyond the unit index, computed once per tile (empty for plain and
// dual values).
template <class T> struct Lane {
  struct Info {};
  static __device__ __forceinline__ Info info(const KParams&, uint64_t, bool) { return {}; }
  static __device__ __forceinline__ T make_input(const KParams& kp, uint64_t u, const Info&, uint32_t i, bool valid) {
    if (!valid) return T(0);
    const T* x = (const T*)kp.x;
    return x[(kp.x_bcast ? 0 : u) * kp.ni + i];
  }
  static __device__ __forceinline__ void store_output(const KParams& kp, uint64_t u, uint32_t j, const T& val, bool valid) {
    if (valid) ((T*)kp.out)[u * kp.no + j] = val;
  }
};
template <class T> struct Lane<dm::Dual<T>> {
  struct Info {};
  static __device__ __forceinline__ Info info(const KParams&, uint64_t, bool) { return {}; }
  static __device__ __forceinline__ dm::Dual<T> make_input(const KParams& kp, uint64_t u, const Info&, uint32_t i,
                                                           bool valid) {
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


// Direction component for Taylor units; STDE units are (point = u / S, dir = u % S).
template <class T, int K> struct Lane<dm::Jet<T, K>> {
  // STDE units (point, direction): the point and direction index (the unit's
  // inputs would otherwise repeat a 64-bit division per input), and in
  // direction modes 4 / 5 the unit's coordinate or entry.  Points are < 2^32.
  struct Info {
    uint32_t pt, s, ent;
  };
  static __device__ __forceinline__ Info info(const KParams& kp, uint64_t u, bool valid) {
    Info f{(uint32_t)u, 0u, 0u};
    if (!valid) return f;
    if (kp.S) {
      const uint64_t pt = u / kp.S;
      f.pt = (uint32_t)pt;
      f.s = (uint32_t)(u - pt * kp.S);
    }
    if (kp.dir_mode == 4 || kp.dir_mode == 5) f.ent = reinterpret_cast<const uint32_t*>(kp.v)[u];
    return f;
  }
  static __device__ __forceinline__ T dir_component(const KParams& kp, uint64_t u, const Info& f, uint32_t i) {
    const T* v = (const T*)kp.v;
    if (kp.S == 0 || kp.dir_mode == 0) return v[u * kp.ni + i];
    if (kp.dir_mode == 1) return v[(uint64_t)f.s * kp.ni + i];
    if (kp.dir_mode == 3) return (i == f.s) ? T(1) : T(0);
    if (kp.dir_mode == 4) return (i == f.ent) ? T(1) : T(0);
    return (philox_bits(kp.seed, f.pt, f.s, i) & 1u) ? T(1) : T(-1);
  }
  static __device__ __forceinline__ dm::Jet<T, K> make_input(const KParams& kp, uint64_t u, const Info& f, uint32_t i,
                                                             bool valid) {
    dm::Jet<T, K> j;
#pragma unroll
    for (int k = 0; k < K; ++k) j.c[k] = T(0);
    if (!valid) return j;
    const T* x = (const T*)kp.x;
    const uint64_t xrow = kp.x_bcast ? 0 : (kp.S ? (uint64_t)f.pt : u);
    j.c[0] = x[xrow * kp.ni + i];
    if (kp.dir_mode == 5) {
      // the unit's entry seeds coefficient `slot` of each of its active inputs
      // (seed_taylor_dyn_jets, src/taylor_dyn.rs); every other coefficient is 0
      const uint32_t e = f.ent;
      const SlotSeed* it = reinterpret_cast<const SlotSeed*>(kp.seed_items);
      for (uint32_t q = kp.seed_off[e]; q < kp.seed_off[e + 1]; ++q) {
        if (it[q].var != i) continue;
        const T c = (T)it[q].coef;
#pragma unroll
        for (int k = 1; k < K; ++k)
          if ((uint32_t)k == it[q].slot) j.c[k] = c;
      }
      return j;
    }
    if (K > 1) j.c[1] = dir_component(kp, u, f, i);
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

// ───────────────────────────── forward executor ─────────────────────────────
// Instructions are decoded from two 16-byte words straight into registers
// (DIns layout: opc|ma|mb|md, a, b, d | save, aux, imm).
// DN: the executor carries dense groups (D_DENSE).  Their m running values
// raise the kernel's register demand for every program, so programs without
// dense groups run an instantiation without them (DN = false), where D_DENSE is
// an invalid instruction.
// WS (warp-shared point): every warp's 32 units are directions of one point
// (point-direction launches, one unit per thread, S a multiple of 32), so
// coefficient 0 of every jet is the same in all lanes; the dense executor then
// accumulates coefficient 0 of output r in lane r (mod the group size) only and
// broadcasts the results with shuffles, instead of every lane accumulating it
// for every output.
template <class V, int P, bool DN = true, bool WS = false> struct FwdExec {
  using Kd = typename dm::KindOf<V>::K;
  using C = Col<V, P>;
  const KParams& kp;
  unsigned char* sm;     // this thread's column base in the shared slot file
  unsigned char* gs;     // ... in the global slots
  unsigned char* tj;     // ... in the trajectory region
  uint64_t unit0;        // unit of point p = unit0 + p
  const uint32_t* bits;  // this thread's column of the direction-sign words (dir_bits)
  bool valid[P];
  typename Lane<V>::Info ui[P];
  // jets of point-direction launches, per point of the thread (set per tile):
  const void* xrow[P];   // the unit's primal row
  const void* vrow[P];   // dir_mode 1: the unit's direction row
  uint32_t sel[P];       // dir_mode 3 / 4: the coordinate of the basis direction

  // slot addresses (bounds-checked in the checked build; plain pointer
  // arithmetic otherwise)
#ifdef ECH_DEVICE_BOUNDS
  __device__ __forceinline__ uint64_t row_bytes() const { return (uint64_t)kp.tile * sizeof(V); }
  __device__ __forceinline__ unsigned char* sp(uint32_t off) const {
    return bounded(sm, off, (uint64_t)kp.smem_regs * row_bytes(), sm, kp.err);
  }
  __device__ __forceinline__ unsigned char* gp(uint32_t off) const {
    return bounded(gs, off, (uint64_t)kp.far_slots * row_bytes(), sm, kp.err);
  }
  __device__ __forceinline__ unsigned char* tp(uint32_t off) const {
    return bounded(tj, off, (uint64_t)kp.traj_slots * row_bytes(), sm, kp.err);
  }
  __device__ __forceinline__ unsigned char* vp(uint32_t mode, uint32_t off) const {
    return mode == M_GLOB ? gp(off) : sp(off);
  }
#else
  __device__ __forceinline__ unsigned char* sp(uint32_t off) const { return sm + off; }
  __device__ __forceinline__ unsigned char* gp(uint32_t off) const { return gs + off; }
  __device__ __forceinline__ unsigned char* tp(uint32_t off) const { return tj + off; }
  __device__ __forceinline__ unsigned char* vp(uint32_t mode, uint32_t off) const {
    return (mode == M_GLOB ? gs : sm) + off;
  }
#endif

  __device__ __forceinline__ void ld(uint32_t mode, uint32_t off, double imm, V (&v)[P]) const {
    if (mode == M_SMEM) C::ld(sp(off), v);
    else if (mode == M_GLOB) C::ld(gp(off), v);
    else {
      const V c = dm::VT<V>::cst(imm);
#pragma unroll
      for (int p = 0; p < P; ++p) v[p] = c;
    }
  }
  __device__ __forceinline__ void put(uint32_t md, uint32_t d, uint32_t save, const V (&r)[P]) const {
    if (md == M_SMEM) C::st(sp(d), r);
    else if (md == M_GLOB) C::st(gp(d), r);
    if (save != kNone) C::st(tp(save), r);
  }
  __device__ __forceinline__ void put_sm(uint32_t d, uint32_t save, const V (&r)[P]) const {
    C::st(sp(d), r);
    if (save != kNone) C::st(tp(save), r);
  }

  __device__ __forceinline__ void ldv(uint32_t mode, uint32_t off, V (&v)[P]) const {
    C::ld(vp(mode, off), v);
  }

  // Fused chain s_t = s_{t-1} (+|-) term_t, t = 1..n, s_0 = acc0: the same
  // Mul / Add / Sub evaluations, in the same operand order, as the tape ops it
  // replaces.  The n DFTerm records follow in the stream
  // (kind|op|xm|ym, x, y, pad | c, pad).
  __device__ __forceinline__ bool chain(Stream<32>& st, uint32_t ma, uint32_t ao, double imm, uint32_t n,
                                        V (&acc)[P]) const {
    if constexpr (JetOrder<V>::K == 3) {  // the compensated option serves the order-3 batch Laplacian
      if (kp.compensated) return chain_comp(st, ma, ao, imm, n, acc);
    }
    ld(ma, ao, imm, acc);
#pragma unroll 1
    for (uint32_t q = 0; q < n; ++q) {
      const unsigned char* rec = st.next();
      if (rec == nullptr) return false;
      const uint4 w0 = *reinterpret_cast<const uint4*>(rec);
      const uint2 w1 = *reinterpret_cast<const uint2*>(rec + 16);
      const uint32_t kind = w0.x & 0xFFu, op = (w0.x >> 8) & 0xFFu;
      V t[P], x[P];
      if (kind == CK_C) {
        const V c = dm::VT<V>::cst(__hiloint2double((int)w1.y, (int)w1.x));
#pragma unroll
        for (int p = 0; p < P; ++p) t[p] = c;
      } else {
        ldv((w0.x >> 16) & 0xFFu, w0.y, kind == CK_X ? t : x);
        if (kind == CK_CX) {
          const V c = dm::VT<V>::cst(__hiloint2double((int)w1.y, (int)w1.x));
#pragma unroll
          for (int p = 0; p < P; ++p) t[p] = Kd::mul(c, x[p]);
        } else if (kind == CK_XC) {
          const V c = dm::VT<V>::cst(__hiloint2double((int)w1.y, (int)w1.x));
#pragma unroll
          for (int p = 0; p < P; ++p) t[p] = Kd::mul(x[p], c);
        } else if (kind == CK_XY) {
          V y[P];
          ldv(w0.x >> 24, w0.z, y);
#pragma unroll
          for (int p = 0; p < P; ++p) t[p] = Kd::mul(x[p], y[p]);
        }
      }
      switch (op) {
        case 0:
#pragma unroll
          for (int p = 0; p < P; ++p) acc[p] = Kd::add(acc[p], t[p]);
          break;
        case 1:
#pragma unroll
          for (int p = 0; p < P; ++p) acc[p] = Kd::add(t[p], acc[p]);
          break;
        case 2:
#pragma unroll
          for (int p = 0; p < P; ++p) acc[p] = Kd::sub(acc[p], t[p]);
          break;
        default:
#pragma unroll
          for (int p = 0; p < P; ++p) acc[p] = Kd::sub(t[p], acc[p]);
          break;
      }
    }
    return true;
  }

  // The fused chain over jets with compensated additions: every coefficient of
  // the running value carries a Neumaier compensation term, folded in at the
  // end.  A subtraction adds the negated term; t - acc negates the running
  // value and its compensation first (negation is exact).
  __device__ __forceinline__ bool chain_comp(Stream<32>& st, uint32_t ma, uint32_t ao, double imm, uint32_t n,
                                             V (&acc)[P]) const {
    using T = typename dm::VT<V>::S;
    constexpr int K = JetOrder<V>::K;
    ld(ma, ao, imm, acc);
    T cmp[P][K];
#pragma unroll
    for (int p = 0; p < P; ++p)
#pragma unroll
      for (int k = 0; k < K; ++k) cmp[p][k] = T(0);
#pragma unroll 1
    for (uint32_t q = 0; q < n; ++q) {
      const unsigned char* rec = st.next();
      if (rec == nullptr) return false;
      const uint4 w0 = *reinterpret_cast<const uint4*>(rec);
      const uint2 w1 = *reinterpret_cast<const uint2*>(rec + 16);
      const uint32_t kind = w0.x & 0xFFu, op = (w0.x >> 8) & 0xFFu;
      V t[P], x[P];
      if (kind == CK_C) {
        const V c = dm::VT<V>::cst(__hiloint2double((int)w1.y, (int)w1.x));
#pragma unroll
        for (int p = 0; p < P; ++p) t[p] = c;
      } else {
        ldv((w0.x >> 16) & 0xFFu, w0.y, kind == CK_X ? t : x);
        if (kind == CK_CX || kind == CK_XC) {
          const V c = dm::VT<V>::cst(__hiloint2double((int)w1.y, (int)w1.x));
#pragma unroll
          for (int p = 0; p < P; ++p) t[p] = kind == CK_CX ? Kd::mul(c, x[p]) : Kd::mul(x[p], c);
        } else if (kind == CK_XY) {
          V y[P];
          ldv(w0.x >> 24, w0.z, y);
#pragma unroll
          for (int p = 0; p < P; ++p) t[p] = Kd::mul(x[p], y[p]);
        }
      }
#pragma unroll
      for (int p = 0; p < P; ++p) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
          if (op == 3) {
            acc[p].c[k] = -acc[p].c[k];
            cmp[p][k] = -cmp[p][k];
          }
          neumaier_add(acc[p].c[k], cmp[p][k], op == 2 ? -t[p].c[k] : t[p].c[k]);
        }
      }
    }
#pragma unroll
    for (int p = 0; p < P; ++p)
#pragma unroll
      for (int k = 0; k < K; ++k) acc[p].c[k] = acc[p].c[k] + cmp[p][k];
    return true;
  }

  // Linear-combination chain: every term is Mul(c, x) or Mul(x, c) added to the
  // running value, in tape order.  DFPair records carry two terms each
  // (c0, c1 | x0, x1, m0|m1|cx0|cx1, pad).  kLcGroup records at a time: all
  // their operand loads are issued before the arithmetic, so a warp keeps
  // several L2 round trips (global slots) in flight; the additions stay in
  // term order.
  static constexpr int kWords = (int)(sizeof(V) * P / 4);
  static constexpr int kLcGroup = kWords <= 8 ? 4 : (kWords <= 16 ? 2 : 1);
  // One term of a linear-combination chain: acc + Mul(c, x) (or Mul(x, c)).
  // Dual values: the product's eps is c eps + 0 re; the zero products commute
  // with every addition and add up exactly, so they collect in a tracker (one
  // fused step each, started at -0) added once at the end of the chain.
  __device__ __forceinline__ void lc_term(V& a, const V& c, const V& x, bool cx,
                                          typename dm::VT<V>::S& dz) const {
    if constexpr (IsDual<V>::v) {
      a.re = a.re + c.re * x.re;
      a.eps = a.eps + c.re * x.eps;
      dz = fma_zero(x.re, dz);
    } else {
      a = Kd::add(a, cx ? Kd::mul(c, x) : Kd::mul(x, c));
    }
  }
  __device__ __forceinline__ void lc_finish(V (&acc)[P], const typename dm::VT<V>::S (&dz)[P]) const {
    if constexpr (IsDual<V>::v) {
#pragma unroll
      for (int p = 0; p < P; ++p) acc[p].eps = acc[p].eps + dz[p];
    }
  }

  __device__ __forceinline__ bool chain_lc(Stream<32>& st, uint32_t ma, uint32_t ao, double imm, uint32_t n,
                                           V (&acc)[P]) const {
    if constexpr (JetOrder<V>::K > 0) return chain_lc_jet(st, ma, ao, imm, n, acc);
    using S = typename dm::VT<V>::S;
    ld(ma, ao, imm, acc);
    S dz[P];
#pragma unroll
    for (int p = 0; p < P; ++p) dz[p] = -S(0);
    uint32_t q = 0;
    if constexpr (kLcGroup > 1) {
#pragma unroll 1
      for (; q + 2 * kLcGroup <= n; q += 2 * kLcGroup) {
        V xs[2 * kLcGroup][P];
        V cs[2 * kLcGroup];
        bool cx[2 * kLcGroup];
#pragma unroll
        for (int k = 0; k < kLcGroup; ++k) {
          const unsigned char* rec = st.next();
          if (rec == nullptr) return false;
          const uint4 cw = *reinterpret_cast<const uint4*>(rec);
          const uint4 xw = *reinterpret_cast<const uint4*>(rec + 16);
          ldv(xw.z & 0xFFu, xw.x, xs[2 * k]);
          ldv((xw.z >> 8) & 0xFFu, xw.y, xs[2 * k + 1]);
          cs[2 * k] = lc_const<V>(cw.x, cw.y);
          cs[2 * k + 1] = lc_const<V>(cw.z, cw.w);
          cx[2 * k] = ((xw.z >> 16) & 0xFFu) != 0;
          cx[2 * k + 1] = (xw.z >> 24) != 0;
        }
#pragma unroll
        for (int j = 0; j < 2 * kLcGroup; ++j) {
#pragma unroll
          for (int p = 0; p < P; ++p) lc_term(acc[p], cs[j], xs[j][p], cx[j], dz[p]);
        }
      }
    }
#pragma unroll 1
    for (; q < n; q += 2) {
      const unsigned char* rec = st.next();
      if (rec == nullptr) return false;
      const uint4 cw = *reinterpret_cast<const uint4*>(rec);
      const uint4 xw = *reinterpret_cast<const uint4*>(rec + 16);
      const V ca = lc_const<V>(cw.x, cw.y);
      const bool a_cx = ((xw.z >> 16) & 0xFFu) != 0;
      V xa[P];
      ldv(xw.z & 0xFFu, xw.x, xa);
      if (q + 1 < n) {
        V xb[P];
        ldv((xw.z >> 8) & 0xFFu, xw.y, xb);
        const V cb = lc_const<V>(cw.z, cw.w);
        const bool b_cx = (xw.z >> 24) != 0;
#pragma unroll
        for (int p = 0; p < P; ++p) {
          lc_term(acc[p], ca, xa[p], a_cx, dz[p]);
          lc_term(acc[p], cb, xb[p], b_cx, dz[p]);
        }
      } else {
#pragma unroll
        for (int p = 0; p < P; ++p) lc_term(acc[p], ca, xa[p], a_cx, dz[p]);
      }
    }
    lc_finish(acc, dz);
    return true;
  }

  // Linear-combination chain over jets.  The reference multiplies a constant c
  // and a jet x as the truncated Cauchy product of the constant jet (c, 0, ..)
  // with x, in either operand order:
  //   t_k = ((0 + c x_k) + 0 x_{k-1}) + ... + 0 x_0.
  // With x_0..x_{k-1} finite the zero products change nothing and t_k is c x_k
  // with a -0 turned into +0; a non-finite x_j (j < k) makes t_k NaN.  So the
  // running value starts as acc0 + 0 (after which no coefficient is ever -0,
  // and adding c x_k equals adding t_k), each term adds c x_k to coefficient
  // k, and per coefficient j below the top a tracker z_j = x_j * 0 + z_j (one
  // fused, exact step: +0 while every x_j is finite, NaN after) is added to
  // every higher coefficient at the end.  Results equal the per-op product bit
  // for bit; each term costs K multiplies, K adds and K-1 fused steps instead
  // of the product's K(K+1) operations.
  // Primal x_i and direction component v_i of point p's unit: the input jet
  // (x_i, v_i, 0, ..) of an M_INPUT term, read at its source.  Programs with
  // such terms run for point-direction launches (S > 0) with directions shared
  // over points (dir_mode 1), device Rademacher signs (2, from the tile's sign
  // words) or basis vectors (3, 4).
  __device__ __forceinline__ void input_xv(uint32_t i, int p, typename dm::VT<V>::S& x0,
                                           typename dm::VT<V>::S& v) const {
    using T = typename dm::VT<V>::S;
    if (!valid[p]) {
      x0 = T(0);
      v = T(0);
      return;
    }
    if (!index_ok(i, kp.ni, kp.err)) i = 0;
    x0 = reinterpret_cast<const T*>(xrow[p])[i];
    if (kp.dir_mode == 2) v = ((bits[(i >> 5) * kp.tile + p] >> (i & 31u)) & 1u) ? T(1) : T(-1);
    else if (kp.dir_mode == 1) v = reinterpret_cast<const T*>(vrow[p])[i];
    else v = (i == sel[p]) ? T(1) : T(0);
  }
  // An M_INPUT term: coefficients 0 and 1 of the input jet are x_i and v_i, the
  // rest +0, whose products add nothing to a running value that is never -0;
  // only the trackers of x_i and v_i remain for the higher coefficients.
  template <bool COMP>
  __device__ __forceinline__ void lc_jet_input_term(V (&acc)[P], typename dm::VT<V>::S (&z)[P][JetOrder<V>::K],
                                                    typename dm::VT<V>::S (&cmp)[P][JetOrder<V>::K],
                                                    const V (&x)[P], typename dm::VT<V>::S c) const {
    constexpr int K = JetOrder<V>::K;
#pragma unroll
    for (int p = 0; p < P; ++p) {
      if constexpr (COMP) neumaier_add(acc[p].c[0], cmp[p][0], c * x[p].c[0]);
      else acc[p].c[0] = acc[p].c[0] + c * x[p].c[0];
      if constexpr (K > 1) {
        if constexpr (COMP) neumaier_add(acc[p].c[1], cmp[p][1], c * x[p].c[1]);
        else acc[p].c[1] = acc[p].c[1] + c * x[p].c[1];
        z[p][0] = fma_zero(x[p].c[0], z[p][0]);
      }
      if constexpr (K > 2) z[p][1] = fma_zero(x[p].c[1], z[p][1]);
    }
  }
  // Operand j of a linear-combination term record into x: a slot load, or the
  // input jet at its source (returns true for M_INPUT).
  __device__ __forceinline__ bool lc_jet_operand(uint32_t mode, uint32_t off, V (&x)[P]) const {
    if constexpr (kBoundsChecked) {
      if (mode != M_INPUT && mode != M_SMEM && mode != M_GLOB) {
        atomicOr(kp.err, (uint32_t)KERR_BOUNDS);
        mode = M_SMEM;
        off = 0;
      }
    }
    if (mode == M_INPUT) {
#pragma unroll
      for (int p = 0; p < P; ++p) {
        typename dm::VT<V>::S x0, v;
        input_xv(off, p, x0, v);
        x[p].c[0] = x0;
        if constexpr (JetOrder<V>::K > 1) x[p].c[1] = v;
      }
      return true;
    }
    ldv(mode, off, x);
    return false;
  }
  template <bool COMP>
  __device__ __forceinline__ void lc_jet_term(V (&acc)[P], typename dm::VT<V>::S (&z)[P][JetOrder<V>::K],
                                              typename dm::VT<V>::S (&cmp)[P][JetOrder<V>::K],
                                              const V (&x)[P], typename dm::VT<V>::S c) const {
    constexpr int K = JetOrder<V>::K;
#pragma unroll
    for (int p = 0; p < P; ++p) {
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if constexpr (COMP) neumaier_add(acc[p].c[k], cmp[p][k], c * x[p].c[k]);
        else acc[p].c[k] = acc[p].c[k] + c * x[p].c[k];
      }
#pragma unroll
      for (int k = 0; k + 1 < K; ++k) z[p][k] = fma_zero(x[p].c[k], z[p][k]);
    }
  }
  __device__ __forceinline__ bool chain_lc_jet(Stream<32>& st, uint32_t ma, uint32_t ao, double imm, uint32_t n,
                                               V (&acc)[P]) const {
    if constexpr (JetOrder<V>::K == 3) {  // the compensated option serves the order-3 batch Laplacian
      if (kp.compensated) return chain_lc_jet_impl<true>(st, ma, ao, imm, n, acc);
    }
    return chain_lc_jet_impl<false>(st, ma, ao, imm, n, acc);
  }
  // COMP: every coefficient's additions carry a Neumaier compensation term
  // (the FP32 compensated option), folded in before the trackers.
  template <bool COMP>
  __device__ __forceinline__ bool chain_lc_jet_impl(Stream<32>& st, uint32_t ma, uint32_t ao, double imm, uint32_t n,
                                                    V (&acc)[P]) const {
    using T = typename dm::VT<V>::S;
    constexpr int K = JetOrder<V>::K;
    ld(ma, ao, imm, acc);
    T z[P][K], cmp[P][K];
#pragma unroll
    for (int p = 0; p < P; ++p) {
#pragma unroll
      for (int k = 0; k < K; ++k) {
        acc[p].c[k] = acc[p].c[k] + T(0);
        z[p][k] = T(0);
        cmp[p][k] = T(0);
      }
    }
    uint32_t q = 0;
    if constexpr (kLcGroup > 1) {
#pragma unroll 1
      for (; q + 2 * kLcGroup <= n; q += 2 * kLcGroup) {
        V xs[2 * kLcGroup][P];
        T cs[2 * kLcGroup];
        bool direct[2 * kLcGroup];
#pragma unroll
        for (int k = 0; k < kLcGroup; ++k) {
          const unsigned char* rec = st.next();
          if (rec == nullptr) return false;
          const uint4 cw = *reinterpret_cast<const uint4*>(rec);
          const uint4 xw = *reinterpret_cast<const uint4*>(rec + 16);
          direct[2 * k] = lc_jet_operand(xw.z & 0xFFu, xw.x, xs[2 * k]);
          direct[2 * k + 1] = lc_jet_operand((xw.z >> 8) & 0xFFu, xw.y, xs[2 * k + 1]);
          cs[2 * k] = lc_scalar<T>(cw.x, cw.y);
          cs[2 * k + 1] = lc_scalar<T>(cw.z, cw.w);
        }
#pragma unroll
        for (int j = 0; j < 2 * kLcGroup; ++j) {
          if (direct[j]) lc_jet_input_term<COMP>(acc, z, cmp, xs[j], cs[j]);
          else lc_jet_term<COMP>(acc, z, cmp, xs[j], cs[j]);
        }
      }
    }
#pragma unroll 1
    for (; q < n; q += 2) {
      const unsigned char* rec = st.next();
      if (rec == nullptr) return false;
      const uint4 cw = *reinterpret_cast<const uint4*>(rec);
      const uint4 xw = *reinterpret_cast<const uint4*>(rec + 16);
      V xa[P];
      if (lc_jet_operand(xw.z & 0xFFu, xw.x, xa)) lc_jet_input_term<COMP>(acc, z, cmp, xa, lc_scalar<T>(cw.x, cw.y));
      else lc_jet_term<COMP>(acc, z, cmp, xa, lc_scalar<T>(cw.x, cw.y));
      if (q + 1 < n) {
        V xb[P];
        if (lc_jet_operand((xw.z >> 8) & 0xFFu, xw.y, xb))
          lc_jet_input_term<COMP>(acc, z, cmp, xb, lc_scalar<T>(cw.z, cw.w));
        else
          lc_jet_term<COMP>(acc, z, cmp, xb, lc_scalar<T>(cw.z, cw.w));
      }
    }
    if constexpr (COMP) {
#pragma unroll
      for (int p = 0; p < P; ++p)
#pragma unroll
        for (int k = 0; k < K; ++k) acc[p].c[k] = acc[p].c[k] + cmp[p][k];
    }
#pragma unroll
    for (int p = 0; p < P; ++p) {
      T zs = T(0);
#pragma unroll
      for (int k = 1; k < K; ++k) {
        zs = zs + z[p][k - 1];
        acc[p].c[k] = acc[p].c[k] + zs;
      }
    }
    return true;
  }

  // Dense group (D_DENSE): m linear-combination chains over the same n
  // operands, outputs j = 0..m-1:  z_j = acc0_j + c_j0 x_0 + .. + c_j,n-1 x_n-1,
  // each added in term order as the chains do, but with one operand load per
  // term for the whole group.  The m running values live in registers; the
  // results are stored after every operand has been read (a result may take an
  // operand's register).  Products follow the kinds' exact forms:
  //   plain  c x;
  //   Dual   (c re, c eps + 0 re), the zero product shared by the group;
  //   jets   the scaled, normalised form with per-term trackers (chain_lc_jet).
  static constexpr int kDenseMax = DN ? (int)dense_group_max((uint32_t)sizeof(V), (uint32_t)P) : 1;
  __device__ __forceinline__ bool dense(Stream<32>& st, uint32_t m, uint32_t n) const {
    if constexpr (kDenseMax < 2) {
      if (threadIdx.x == 0) atomicOr(kp.err, (uint32_t)KERR_BADINS);
      ring_drain(*st.rg);
      return false;
    } else {
      // (launches with compensated chains run plans without dense groups; the
      // lowering forms only full groups, m == kDenseMax)
      if constexpr (JetOrder<V>::K > 1) {
        // device Rademacher signs and basis directions: every direction
        // component is +-1 or 0
        if (kp.dir_mode >= 2 && kp.dir_mode <= 4) return dense_impl<true, true>(st, m, n);
      }
      return dense_impl<true, false>(st, m, n);
    }
  }
  // FULL: the group has kDenseMax outputs, so no output needs a bound (the
  // per-output bounds of the general form cost registers and instructions in
  // every group).  UNITV: the direction components of input-direct operands
  // are +-1 or 0, so c * v is exact and c1 + c * v rounds like one fused
  // multiply-add.
  template <bool FULL, bool UNITV>
  __device__ __forceinline__ bool dense_impl(Stream<32>& st, uint32_t m, uint32_t n) const {
    using T = typename dm::VT<V>::S;
    constexpr int MX = kDenseMax > 1 ? kDenseMax : 2;
    constexpr int KJ = JetOrder<V>::K > 0 ? JetOrder<V>::K : 1;
    constexpr int PER = sizeof(T) == 4 ? 8 : 4;  // constants per record
    if (m < 1 || m > (uint32_t)kDenseMax || (FULL && m != (uint32_t)kDenseMax)) {
      if (threadIdx.x == 0) atomicOr(kp.err, (uint32_t)KERR_BADINS);
      ring_drain(*st.rg);
      return false;
    }
    V acc[MX][P];
#pragma unroll
    for (int jj = 0; jj < MX; jj += 2) {
      if (FULL || (uint32_t)jj < m) {
        const unsigned char* rec = st.next();
        if (rec == nullptr) return false;
        const double2 imm = *reinterpret_cast<const double2*>(rec);
        const uint4 w = *reinterpret_cast<const uint4*>(rec + 16);
        ld(w.z & 0xFFu, w.x, imm.x, acc[jj]);
        if (FULL || (uint32_t)jj + 1 < m) ld((w.z >> 8) & 0xFFu, w.y, imm.y, acc[jj + 1]);
      }
    }
    // Dual: the eps part of c x is c eps + 0 re; the zero products commute with
    // every addition and add up exactly, so one tracker per point, started at
    // -0 (the identity of +), collects them for the whole group: dz = fma(re, 0, dz).
    T z[P][KJ], dz[P];
#pragma unroll
    for (int p = 0; p < P; ++p) dz[p] = -T(0);
    if constexpr (JetOrder<V>::K > 0) {
#pragma unroll
      for (int p = 0; p < P; ++p)
#pragma unroll
        for (int k = 0; k < KJ; ++k) z[p][k] = T(0);
#pragma unroll
      for (int j = 0; j < MX; ++j)
#pragma unroll
        for (int p = 0; p < P; ++p)
#pragma unroll
          for (int k = 0; k < KJ; ++k) acc[j][p].c[k] = acc[j][p].c[k] + T(0);
    }
    // warp-shared point: this lane accumulates coefficient 0 of output `myrow`
    // (every lane holds the same starting values, so a select picks it)
    constexpr bool kWS = WS && JetOrder<V>::K > 1 && P == 1;
    const int myrow = kWS ? (int)((threadIdx.x & 31u) % (uint32_t)MX) : 0;
    T c0m = T(0);
    if constexpr (kWS) {
#pragma unroll
      for (int j = 0; j < MX; ++j)
        if (j == myrow) c0m = acc[j][0].c[0];
    }
#pragma unroll 1
    for (uint32_t q0 = 0; q0 < n; q0 += 4) {
      const unsigned char* orec = st.next();
      if (orec == nullptr) return false;
      const uint4 xw = *reinterpret_cast<const uint4*>(orec);
      const uint32_t mw = *reinterpret_cast<const uint32_t*>(orec + 16);
      const uint32_t xo[4] = {xw.x, xw.y, xw.z, xw.w};
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        if (q0 + t >= n) break;
        const uint32_t mode = (mw >> (8 * t)) & 0xFFu;
        V x[P];
        bool direct = false;
        if constexpr (JetOrder<V>::K > 0) direct = lc_jet_operand(mode, xo[t], x);
        else ldv(mode, xo[t], x);
        if constexpr (IsDual<V>::v) {
#pragma unroll
          for (int p = 0; p < P; ++p) dz[p] = fma_zero(x[p].re, dz[p]);
        }
        T mycs = T(0);  // warp-shared point: this lane's output's constant of the term
#pragma unroll
        for (int jj = 0; jj < MX; jj += PER) {
          if (FULL || (uint32_t)jj < m) {
            const unsigned char* crec = st.next();
            if (crec == nullptr) return false;
            T cs[PER];
#pragma unroll
            for (int j = 0; j < PER; ++j) cs[j] = reinterpret_cast<const T*>(crec)[j];
            if constexpr (kWS) {
              // read before the next pull, which may recycle the record's stage
              const T mine = reinterpret_cast<const T*>(crec)[myrow % PER];
              if (myrow / PER == jj / PER) mycs = mine;
            }
            // an input jet (x_i, v_i, 0, ..) read at its source changes
            // coefficients 0 and 1 only (its zero products add nothing)
            if constexpr (JetOrder<V>::K > 0) {
              if (direct) {
#pragma unroll
                for (int j = 0; j < PER; ++j) {
                  if (jj + j < MX && (FULL || (uint32_t)(jj + j) < m)) {
#pragma unroll
                    for (int p = 0; p < P; ++p) {
                      V& a = acc[jj + j < MX ? jj + j : 0][p];
                      if constexpr (!kWS) a.c[0] = a.c[0] + cs[j] * x[p].c[0];
                      if constexpr (KJ > 1) {
                        if constexpr (UNITV) a.c[1] = fma_rn(cs[j], x[p].c[1], a.c[1]);
                        else a.c[1] = a.c[1] + cs[j] * x[p].c[1];
                      }
                    }
                  }
                }
                continue;
              }
            }
#pragma unroll
            for (int j = 0; j < PER; ++j) {
              if (jj + j < MX && (FULL || (uint32_t)(jj + j) < m)) {
                const T c = cs[j];
#pragma unroll
                for (int p = 0; p < P; ++p) {
                  V& a = acc[jj + j < MX ? jj + j : 0][p];
                  if constexpr (JetOrder<V>::K > 0) {
#pragma unroll
                    for (int k = kWS ? 1 : 0; k < KJ; ++k) a.c[k] = a.c[k] + c * x[p].c[k];
                  } else if constexpr (IsDual<V>::v) {
                    a.re = a.re + c * x[p].re;
                    a.eps = a.eps + c * x[p].eps;
                  } else {
                    a = a + c * x[p];
                  }
                }
              }
            }
          }
        }
        if constexpr (kWS) c0m = c0m + mycs * x[0].c[0];
        if constexpr (JetOrder<V>::K > 1) {
#pragma unroll
          for (int p = 0; p < P; ++p) {
            if (direct) {
              z[p][0] = fma_zero(x[p].c[0], z[p][0]);
              if constexpr (KJ > 2) z[p][1] = fma_zero(x[p].c[1], z[p][1]);
            } else {
#pragma unroll
              for (int k = 0; k + 1 < KJ; ++k) z[p][k] = fma_zero(x[p].c[k], z[p][k]);
            }
          }
        }
      }
    }
    if constexpr (kWS) {
#pragma unroll
      for (int j = 0; j < MX; ++j) acc[j][0].c[0] = __shfl_sync(0xffffffffu, c0m, j);
    }
#pragma unroll
    for (int jj = 0; jj < MX; jj += 2) {
      if (FULL || (uint32_t)jj < m) {
        const unsigned char* rec = st.next();
        if (rec == nullptr) return false;
        const uint4 w0 = *reinterpret_cast<const uint4*>(rec);
        const uint32_t mdw = *reinterpret_cast<const uint32_t*>(rec + 16);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int j = jj + h;
          if (j >= MX || (!FULL && (uint32_t)j >= m)) continue;
          if constexpr (JetOrder<V>::K > 0) {
#pragma unroll
            for (int p = 0; p < P; ++p) {
              T zs = T(0);
#pragma unroll
              for (int k = 0; k < KJ; ++k) {
                if (k > 0) {
                  zs = zs + z[p][k - 1];
                  acc[j][p].c[k] = acc[j][p].c[k] + zs;
                }
              }
            }
          } else if constexpr (IsDual<V>::v) {
#pragma unroll
            for (int p = 0; p < P; ++p) acc[j][p].eps = acc[j][p].eps + dz[p];
          }
          put((mdw >> (8 * h)) & 0xFFu, h == 0 ? w0.x : w0.y, h == 0 ? w0.z : w0.w, acc[j]);
        }
      }
    }
    return true;
  }

  __device__ __forceinline__ bool operator()(const unsigned char* raw, Stream<32>& st) const {
    const uint4 w0 = *reinterpret_cast<const uint4*>(raw);
    const uint4 w1 = *reinterpret_cast<const uint4*>(raw + 16);
    const uint32_t opc = w0.x & 0xFFu;
    const uint32_t ao = w0.y, bo = w0.z, dof = w0.w, save = w1.x;
    const int32_t aux = (int32_t)w1.y;
    const double imm = __hiloint2double((int)w1.w, (int)w1.z);
    V a[P], b[P], r[P];
    switch (opc) {
      case D_LDIN:
#pragma unroll
        for (int p = 0; p < P; ++p)
          r[p] = Lane<V>::make_input(kp, unit0 + p, ui[p], (uint32_t)aux,
                                     valid[p] && index_ok((uint32_t)aux, kp.ni, kp.err));
        put(w0.x >> 24, dof, save, r);
        return true;
      case D_STOUT:
        ld((w0.x >> 8) & 0xFFu, ao, imm, a);
#pragma unroll
        for (int p = 0; p < P; ++p)
          Lane<V>::store_output(kp, unit0 + p, (uint32_t)aux, a[p], valid[p] && index_ok((uint32_t)aux, kp.no, kp.err));
        return true;
      case D_MOV:
        ld((w0.x >> 8) & 0xFFu, ao, imm, a);
        put(w0.x >> 24, dof, save, a);
        return true;
      case D_CHAIN:
        if (!chain(st, (w0.x >> 8) & 0xFFu, ao, imm, (uint32_t)aux, r)) return false;
        put(w0.x >> 24, dof, save, r);
        return true;
      case D_CHAIN_LC:
        if (!chain_lc(st, (w0.x >> 8) & 0xFFu, ao, imm, (uint32_t)aux, r)) return false;
        put(w0.x >> 24, dof, save, r);
        return true;
      case D_DENSE:
        return dense(st, (uint32_t)aux, ao);
#define ECH_FB(NAME, FN)                                                     \
  case D_##NAME##_RR:                                                        \
    C::ld(sp(ao), a);                                                        \
    C::ld(sp(bo), b);                                                        \
    _Pragma("unroll") for (int p = 0; p < P; ++p) r[p] = Kd::FN(a[p], b[p]); \
    put_sm(dof, save, r);                                                    \
    return true;                                                                  \
  case D_##NAME##_IR: {                                                      \
    const V c = dm::VT<V>::cst(imm);                                         \
    C::ld(sp(bo), b);                                                        \
    _Pragma("unroll") for (int p = 0; p < P; ++p) r[p] = Kd::FN(c, b[p]);    \
    put_sm(dof, save, r);                                                    \
    return true;                                                                  \
  }                                                                          \
  case D_##NAME##_RI: {                                                      \
    const V c = dm::VT<V>::cst(imm);                                         \
    C::ld(sp(ao), a);                                                        \
    _Pragma("unroll") for (int p = 0; p < P; ++p) r[p] = Kd::FN(a[p], c);    \
    put_sm(dof, save, r);                                                    \
    return true;                                                                  \
  }
      ECH_FB(ADD, add)
      ECH_FB(SUB, sub)
      ECH_FB(MUL, mul)
      ECH_FB(DIV, div)
#undef ECH_FB
#define ECH_FU(OP)                                                                               \
  case D_FU_BASE + (OP - OP_NEG):                                                                \
    C::ld(sp(ao), a);                                                                            \
    _Pragma("unroll") for (int p = 0; p < P; ++p) r[p] = dm::eval_forward<V>(OP, a[p], a[p], aux); \
    put_sm(dof, save, r);                                                                        \
    return true;
      ECH_FU(OP_NEG) ECH_FU(OP_RECIP) ECH_FU(OP_SQRT) ECH_FU(OP_CBRT) ECH_FU(OP_POWI) ECH_FU(OP_EXP)
      ECH_FU(OP_EXP2) ECH_FU(OP_EXPM1) ECH_FU(OP_LN) ECH_FU(OP_LOG2) ECH_FU(OP_LOG10) ECH_FU(OP_LN1P)
      ECH_FU(OP_SIN) ECH_FU(OP_COS) ECH_FU(OP_TAN) ECH_FU(OP_ASIN) ECH_FU(OP_ACOS) ECH_FU(OP_ATAN)
      ECH_FU(OP_SINH) ECH_FU(OP_COSH) ECH_FU(OP_TANH) ECH_FU(OP_ASINH) ECH_FU(OP_ACOSH) ECH_FU(OP_ATANH)
      ECH_FU(OP_ABS) ECH_FU(OP_SIGNUM) ECH_FU(OP_FLOOR) ECH_FU(OP_CEIL) ECH_FU(OP_ROUND) ECH_FU(OP_TRUNC)
      ECH_FU(OP_FRACT)
#undef ECH_FU
      default:
        break;
    }
    // generic path: any operand modes
    const uint32_t mb = (w0.x >> 16) & 0xFFu;
    ld((w0.x >> 8) & 0xFFu, ao, imm, a);
    if (mb == M_NONE) {
#pragma unroll
      for (int p = 0; p < P; ++p) b[p] = Kd::c(0);
    } else {
      ld(mb, bo, imm, b);
    }
#pragma unroll
    for (int p = 0; p < P; ++p) r[p] = dm::eval_forward<V>(opc, a[p], b[p], aux);
    put(w0.x >> 24, dof, save, r);
    return true;
  }
};

// ───────────────────────────── reverse executor ─────────────────────────────
// DRIns layout: opc|pad|flags, r, a, b | va, vb, vr, aux | imm, pad.
// DN: the executor carries gather tiles (built with the dense-group executor).
template <class V, int P, bool DN = true> struct RevExec {
  using Kd = typename dm::KindOf<V>::K;
  using C = Col<V, P>;
  const KParams& kp;
  unsigned char* sm;
  unsigned char* gs;
  const unsigned char* tj;
  uint64_t unit0;
  bool valid[P];

  __device__ __forceinline__ void value(uint32_t off, bool imm, double c, V (&v)[P]) const {
    if (imm) {
      const V k = dm::VT<V>::cst(c);
#pragma unroll
      for (int p = 0; p < P; ++p) v[p] = k;
    } else if (off == kNone) {
#pragma unroll
      for (int p = 0; p < P; ++p) v[p] = Kd::c(0);
    } else {
#ifdef ECH_DEVICE_BOUNDS
      C::ld(bounded(const_cast<unsigned char*>(tj), off, (uint64_t)kp.traj_slots * kp.tile * sizeof(V), sm, kp.err),
            v);
#else
      C::ld(tj + off, v);
#endif
    }
  }
#ifdef ECH_DEVICE_BOUNDS
  __device__ __forceinline__ unsigned char* loc(bool glob, uint32_t off) const {
    const uint64_t row = (uint64_t)kp.tile * sizeof(V);
    return glob ? bounded(gs, off, (uint64_t)kp.far_slots * row, sm, kp.err)
                : bounded(sm, off, (uint64_t)kp.smem_regs * row, sm, kp.err);
  }
#else
  __device__ __forceinline__ unsigned char* loc(bool glob, uint32_t off) const { return (glob ? gs : sm) + off; }
#endif

  template <bool FAST>
  __device__ __forceinline__ void accumulate(unsigned char* ptr, bool init, const V (&adj)[P], const V (&d)[P]) const {
    V cur[P];
    if (init) {
#pragma unroll
      for (int p = 0; p < P; ++p) cur[p] = Kd::c(0);
    } else {
      C::ld(ptr, cur);
    }
#pragma unroll
    for (int p = 0; p < P; ++p) {
      const bool hit = !Kd::all_zero(adj[p]) && !Kd::all_zero(d[p]);
      if (hit) cur[p] = Kd::add(cur[p], Kd::mul(d[p], adj[p]));
    }
    C::st(ptr, cur);
  }

  // Adjoint of a single-use intermediate after its only contribution.
  __device__ __forceinline__ void internal(const V (&adj)[P], const V (&d)[P], V (&out)[P]) const {
#pragma unroll
    for (int p = 0; p < P; ++p) {
      const bool hit = !Kd::all_zero(adj[p]) && !Kd::all_zero(d[p]);
      out[p] = hit ? Kd::add(Kd::c(0), Kd::mul(d[p], adj[p])) : Kd::c(0);
    }
  }

  // Reverse of a fused chain: for t = n..1 the Add/Sub (its two operands in
  // operand order), then the absorbed Mul, exactly as the per-op sweep visits
  // them.  Adjoints of the chain's intermediates stay in registers.  The n
  // DRTerm records follow in the stream, last term first
  // (kind|op|flags, ax, ay, vx | vy, pad, c | pad).
  __device__ __forceinline__ bool chain(Stream<48>& st, uint32_t flags, uint32_t ro, uint32_t ao, uint32_t n) const {
    V adj[P];
    C::ld(loc(flags & RF_R_GLOB, ro), adj);
    V one[P], mone[P];
    {
      V d0, d1;
      dm::reverse_partials<V>(OP_SUB, Kd::c(0), Kd::c(0), Kd::c(0), 0, d0, d1);
#pragma unroll
      for (int p = 0; p < P; ++p) { one[p] = d0; mone[p] = d1; }
    }
#pragma unroll 1
    for (uint32_t q = n; q-- > 0;) {
      const unsigned char* rec = st.next();
      if (rec == nullptr) return false;
      const uint4 w0 = *reinterpret_cast<const uint4*>(rec);
      const uint4 w1 = *reinterpret_cast<const uint4*>(rec + 16);
      const uint32_t kind = w0.x & 0xFFu, op = (w0.x >> 8) & 0xFFu, tf = w0.x >> 16;
      const bool chain_a = (op & 1u) == 0;
      // partials of the Add / Sub: acc side and term side
      const V (&dacc)[P] = (op == 3) ? mone : one;
      const V (&dterm)[P] = (op == 2) ? mone : one;
      V nadj[P], tadj[P];
      auto acc_side = [&]() {
        if (q == 0) {
          if (flags & RF_HAS_A) accumulate<false>(loc(flags & RF_A_GLOB, ao), (flags & RF_A_INIT) != 0, adj, dacc);
        } else {
          internal(adj, dacc, nadj);
        }
      };
      auto term_side = [&]() {
        if (kind == CK_X) accumulate<false>(loc(tf & CF_X_GLOB, w0.y), (tf & CF_X_INIT) != 0, adj, dterm);
        else if (kind != CK_C) internal(adj, dterm, tadj);
      };
      if (chain_a) { acc_side(); term_side(); } else { term_side(); acc_side(); }
      if (kind == CK_CX || kind == CK_XC) {
        V c[P];
        const V cv = dm::VT<V>::cst(__hiloint2double((int)w1.w, (int)w1.z));
#pragma unroll
        for (int p = 0; p < P; ++p) c[p] = cv;
        accumulate<false>(loc(tf & CF_X_GLOB, w0.y), (tf & CF_X_INIT) != 0, tadj, c);
      } else if (kind == CK_XY) {
        V xv[P], yv[P];
        value(w0.w, false, 0.0, xv);
        value(w1.x, false, 0.0, yv);
        accumulate<false>(loc(tf & CF_X_GLOB, w0.y), (tf & CF_X_INIT) != 0, tadj, yv);
        accumulate<false>(loc(tf & CF_Y_GLOB, w0.z), (tf & CF_Y_INIT) != 0, tadj, xv);
      }
      if (q > 0) {
#pragma unroll
        for (int p = 0; p < P; ++p) adj[p] = nadj[p];
      }
    }
    return true;
  }

  // Reverse of a linear-combination chain (every term Mul(c, x) or Mul(x, c),
  // op acc + term): for t = n..1 the Add (acc side, then the term side), then
  // the Mul's contribution c * adj(term) to adj(x).  Both Add sides see the
  // multiplier 1, so the running adjoint and the term's adjoint are the same
  // value, internal(running).  internal() is idempotent (a value it returns
  // comes back unchanged, NaN stays NaN), so every term sees
  // t = internal(adj(r)), and the first term's acc side sees adj(r) itself when
  // the chain has one term, t otherwise.  DRPair records carry terms
  // (n-1-2k, n-2-2k) (c0, c1 | ax0, ax1, flags0|flags1, pad | pad).
  static constexpr int kWords = (int)(sizeof(V) * P / 4);
  static constexpr int kLcGroup = kWords <= 4 ? 2 : 1;  // records per batch of independent updates
  __device__ __forceinline__ void lc_update(V (&cur)[P], const V (&t)[P], const V& c) const {
#pragma unroll
    for (int p = 0; p < P; ++p)
      if (!Kd::all_zero(t[p]) && !Kd::all_zero(c)) cur[p] = Kd::add(cur[p], Kd::mul(c, t[p]));
  }
  __device__ __forceinline__ void lc_load(unsigned char* ptr, bool init, V (&cur)[P]) const {
    if (init) {
#pragma unroll
      for (int p = 0; p < P; ++p) cur[p] = Kd::c(0);
    } else {
      C::ld(ptr, cur);
    }
  }
  __device__ __forceinline__ bool chain_lc(Stream<48>& st, uint32_t flags, uint32_t ro, uint32_t ao,
                                           uint32_t n) const {
    V adj[P], one[P], t[P];
#pragma unroll
    for (int p = 0; p < P; ++p) one[p] = Kd::c(1);
    C::ld(loc(flags & RF_R_GLOB, ro), adj);
    internal(adj, one, t);
    uint32_t q = n;
    if constexpr (kLcGroup > 1) {
      // The chain's adjoint targets are pairwise distinct (RF_LC_DISTINCT): the
      // updates of 2*kLcGroup terms that are not the first are independent, so
      // all their loads issue before the first store.
      if (flags & RF_LC_DISTINCT) {
#pragma unroll 1
        while (q >= 2 * kLcGroup + 1) {
          unsigned char* pt[2 * kLcGroup];
          V cs[2 * kLcGroup];
          V cur[2 * kLcGroup][P];
#pragma unroll
          for (int k = 0; k < kLcGroup; ++k) {
            const unsigned char* rec = st.next();
            if (rec == nullptr) return false;
            const uint4 cw = *reinterpret_cast<const uint4*>(rec);
            const uint4 aw = *reinterpret_cast<const uint4*>(rec + 16);
            const uint32_t f0 = aw.z & 0xFFFFu, f1 = aw.z >> 16;
            pt[2 * k] = loc(f0 & CF_X_GLOB, aw.x);
            pt[2 * k + 1] = loc(f1 & CF_X_GLOB, aw.y);
            cs[2 * k] = lc_const<V>(cw.x, cw.y);
            cs[2 * k + 1] = lc_const<V>(cw.z, cw.w);
            lc_load(pt[2 * k], (f0 & CF_X_INIT) != 0, cur[2 * k]);
            lc_load(pt[2 * k + 1], (f1 & CF_X_INIT) != 0, cur[2 * k + 1]);
          }
#pragma unroll
          for (int j = 0; j < 2 * kLcGroup; ++j) {
            lc_update(cur[j], t, cs[j]);
            C::st(pt[j], cur[j]);
          }
          q -= 2 * kLcGroup;
        }
      }
    }
#pragma unroll 1
    for (; q > 0; q = q >= 2 ? q - 2 : 0) {
      // this record: terms q-1 and (when q >= 2) q-2
      const unsigned char* rec = st.next();
      if (rec == nullptr) return false;
      const uint4 cw = *reinterpret_cast<const uint4*>(rec);
      const uint4 aw = *reinterpret_cast<const uint4*>(rec + 16);
      const uint32_t fa = aw.z & 0xFFFFu, fb = aw.z >> 16;
      unsigned char* pa = loc(fa & CF_X_GLOB, aw.x);
      unsigned char* pb = loc(fb & CF_X_GLOB, aw.y);
      const V ca = lc_const<V>(cw.x, cw.y);
      const V cb = lc_const<V>(cw.z, cw.w);
      V cura[P], curb[P];
      if (q >= 3 && pa != pb) {
        // neither term is the first and their adjoint targets differ: the two
        // read-modify-writes are independent, so both loads issue first
        lc_load(pa, (fa & CF_X_INIT) != 0, cura);
        lc_load(pb, (fb & CF_X_INIT) != 0, curb);
        lc_update(cura, t, ca);
        lc_update(curb, t, cb);
        C::st(pa, cura);
        C::st(pb, curb);
        continue;
      }
      // one term at a time; the first term's Add also pays adj(acc0)
      if (q == 1 && (flags & RF_HAS_A))
        accumulate<false>(loc(flags & RF_A_GLOB, ao), (flags & RF_A_INIT) != 0, n == 1 ? adj : t, one);
      lc_load(pa, (fa & CF_X_INIT) != 0, cura);
      lc_update(cura, t, ca);
      C::st(pa, cura);
      if (q >= 2) {
        if (q == 2 && (flags & RF_HAS_A))
          accumulate<false>(loc(flags & RF_A_GLOB, ao), (flags & RF_A_INIT) != 0, t, one);
        lc_load(pb, (fb & CF_X_INIT) != 0, curb);
        lc_update(curb, t, cb);
        C::st(pb, curb);
      }
    }
    return true;
  }

  // Reverse gather (D_GATHER): for each target, its adjoint (+0 when this is
  // its first contribution) plus c * t for each contribution in order, with
  // the zero-adjoint skip (the zero-multiplier guard is the encoder's: it
  // leaves zero-constant contributions out), then one store.  t is
  // a chain's adjoint after D_NORM.  Contribution loads are grouped so several
  // are in flight; the updates stay in order.
  static constexpr int kGather = kWords <= 4 ? 4 : (kWords <= 8 ? 2 : 1);
  // c * t into cur unless t is zero (the zero-adjoint skip); gather constants
  // are never zero (the encoder leaves zero contributions out)
  // (Dual values: c t's eps is c eps + 0 re; the zero products go to the
  // target's tracker dz, added once before the store, as in lc_term.)
  __device__ __forceinline__ void gather_update(V (&cur)[P], const V (&t)[P], const V& c,
                                                typename dm::VT<V>::S (&dz)[P]) const {
#pragma unroll
    for (int p = 0; p < P; ++p) {
      if (Kd::all_zero(t[p])) continue;
      if constexpr (IsDual<V>::v) {
        cur[p].re = cur[p].re + c.re * t[p].re;
        cur[p].eps = cur[p].eps + c.re * t[p].eps;
        dz[p] = fma_zero(t[p].re, dz[p]);
      } else {
        cur[p] = Kd::add(cur[p], Kd::mul(c, t[p]));
      }
    }
  }
  // A gather tile (DGatherTargets): kGT targets (the lowering forms only full
  // tiles, so no target needs a bound) whose contributions read the same chain
  // adjoints in the same order, every constant nonzero.  Each source
  // is loaded and zero-tested once for the tile and added to every target, in
  // source order per target, as gather_update does.  Dual values: every target
  // receives the same zero products (one per source that is not skipped), so
  // one tracker per point serves the whole tile.  Records are read into
  // registers before the next pull.
  static constexpr int kGT =
      DN ? (int)gather_tile_max(dense_group_max((uint32_t)sizeof(V), (uint32_t)P), sizeof(typename dm::VT<V>::S) == 8)
         : 1;
  __device__ __forceinline__ bool gather_tile(Stream<48>& st, uint32_t T, uint32_t ns) const {
    if constexpr (kGT < 2) {
      if (threadIdx.x == 0) atomicOr(kp.err, (uint32_t)KERR_BADINS);
      ring_drain(*st.rg);
      return false;
    } else {
      using S = typename dm::VT<V>::S;
      if (T != (uint32_t)kGT) {  // the lowering forms only full tiles
        if (threadIdx.x == 0) atomicOr(kp.err, (uint32_t)KERR_BADINS);
        ring_drain(*st.rg);
        return false;
      }
      const unsigned char* trec = st.next();
      if (trec == nullptr) return false;
      uint32_t tx[kGT];
#pragma unroll
      for (int k = 0; k < kGT; ++k) tx[k] = reinterpret_cast<const uint32_t*>(trec)[k];
      V cur[kGT][P];
#pragma unroll
      for (int k = 0; k < kGT; ++k)
        lc_load(loc((tx[k] & GT_GLOB) != 0, tx[k] & GT_OFF), (tx[k] & GT_INIT) != 0, cur[k]);
      S dz[P];
#pragma unroll
      for (int p = 0; p < P; ++p) dz[p] = -S(0);
#pragma unroll 1
      for (uint32_t s0 = 0; s0 < ns; s0 += 12) {
        const unsigned char* srec = st.next();
        if (srec == nullptr) return false;
        uint32_t ax[12];
#pragma unroll
        for (int j = 0; j < 12; ++j) ax[j] = reinterpret_cast<const uint32_t*>(srec)[j];
#pragma unroll
        for (int j = 0; j < 12; ++j) {
          if (s0 + j >= ns) break;
          V t[P];
          C::ld(loc((ax[j] & GT_GLOB) != 0, ax[j] & GT_OFF), t);
          const unsigned char* crec = st.next();
          if (crec == nullptr) return false;
          S cs[kGT];
#pragma unroll
          for (int k = 0; k < kGT; ++k) cs[k] = reinterpret_cast<const S*>(crec)[k];
#pragma unroll
          for (int p = 0; p < P; ++p) {
            if (Kd::all_zero(t[p])) continue;  // the zero-adjoint skip
            if constexpr (IsDual<V>::v) {
              dz[p] = fma_zero(t[p].re, dz[p]);
#pragma unroll
              for (int k = 0; k < kGT; ++k) {
                cur[k][p].re = cur[k][p].re + cs[k] * t[p].re;
                cur[k][p].eps = cur[k][p].eps + cs[k] * t[p].eps;
              }
            } else {
#pragma unroll
              for (int k = 0; k < kGT; ++k)
                cur[k][p] = Kd::add(cur[k][p], Kd::mul(dm::VT<V>::cst_s(cs[k]), t[p]));
            }
          }
        }
      }
#pragma unroll
      for (int k = 0; k < kGT; ++k) {
        if constexpr (IsDual<V>::v) {
#pragma unroll
          for (int p = 0; p < P; ++p) cur[k][p].eps = cur[k][p].eps + dz[p];
        }
        C::st(loc((tx[k] & GT_GLOB) != 0, tx[k] & GT_OFF), cur[k]);
      }
      return true;
    }
  }

  __device__ __forceinline__ bool gather(Stream<48>& st, uint32_t ntargets) const {
#pragma unroll 1
    for (uint32_t g = 0; g < ntargets; ++g) {
      const unsigned char* rec = st.next();
      if (rec == nullptr) return false;
      const uint4 h = *reinterpret_cast<const uint4*>(rec);
      if ((h.x & 0xFFu) == 1u) {  // a gather tile of (h.x >> 8) & 0xFF targets, h.z sources
        const uint32_t T = (h.x >> 8) & 0xFFu;
        if (T > ntargets - g) {
          if (threadIdx.x == 0) atomicOr(kp.err, (uint32_t)KERR_BADINS);
          ring_drain(*st.rg);
          return false;
        }
        if (!gather_tile(st, T, h.z)) return false;
        g += T - 1;
        continue;
      }
      const uint32_t hf = h.x >> 16, nc = h.z;
      unsigned char* px = loc(hf & CF_X_GLOB, h.y);
      V cur[P];
      lc_load(px, (hf & CF_X_INIT) != 0, cur);
      typename dm::VT<V>::S dz[P];
#pragma unroll
      for (int p = 0; p < P; ++p) dz[p] = -typename dm::VT<V>::S(0);
      uint32_t q = 0;
      if constexpr (kGather > 1) {
#pragma unroll 1
        for (; q + 2 * kGather <= nc; q += 2 * kGather) {
          V ts[2 * kGather][P];
          V cs[2 * kGather];
#pragma unroll
          for (int k = 0; k < kGather; ++k) {
            const unsigned char* r2 = st.next();
            if (r2 == nullptr) return false;
            const uint4 cw = *reinterpret_cast<const uint4*>(r2);
            const uint4 aw = *reinterpret_cast<const uint4*>(r2 + 16);
            C::ld(loc(aw.z & CF_X_GLOB, aw.x), ts[2 * k]);
            C::ld(loc((aw.z >> 16) & CF_X_GLOB, aw.y), ts[2 * k + 1]);
            cs[2 * k] = lc_const<V>(cw.x, cw.y);
            cs[2 * k + 1] = lc_const<V>(cw.z, cw.w);
          }
#pragma unroll
          for (int j = 0; j < 2 * kGather; ++j) gather_update(cur, ts[j], cs[j], dz);
        }
      }
#pragma unroll 1
      for (; q < nc; q += 2) {
        const unsigned char* r2 = st.next();
        if (r2 == nullptr) return false;
        const uint4 cw = *reinterpret_cast<const uint4*>(r2);
        const uint4 aw = *reinterpret_cast<const uint4*>(r2 + 16);
        V t0[P];
        C::ld(loc(aw.z & CF_X_GLOB, aw.x), t0);
        gather_update(cur, t0, lc_const<V>(cw.x, cw.y), dz);
        if (q + 1 < nc) {
          V t1[P];
          C::ld(loc((aw.z >> 16) & CF_X_GLOB, aw.y), t1);
          gather_update(cur, t1, lc_const<V>(cw.z, cw.w), dz);
        }
      }
      if constexpr (IsDual<V>::v) {
#pragma unroll
        for (int p = 0; p < P; ++p) cur[p].eps = cur[p].eps + dz[p];
      }
      C::st(px, cur);
    }
    return true;
  }

  // One reverse op: adj(a) += da * adj(r), adj(b) += db * adj(r) with the
  // zero-adjoint skip and the zero-multiplier guard.  FAST: every adjoint
  // location is in shared memory.
  template <bool FAST>
  __device__ __forceinline__ void body(uint32_t opc, uint32_t flags, uint32_t ro, uint32_t ao, uint32_t bo,
                                       uint32_t vao, uint32_t vbo, uint32_t vro, int32_t aux, double imm) const {
    V adj[P], va[P], vb[P], vr[P], da[P], db[P];
    C::ld(FAST ? loc(false, ro) : loc(flags & RF_R_GLOB, ro), adj);
    value(vao, (flags & RF_VA_IMM) != 0, imm, va);
    value(vbo, (flags & RF_VB_IMM) != 0, imm, vb);
    value(vro, false, 0.0, vr);
#pragma unroll
    for (int p = 0; p < P; ++p) dm::reverse_partials<V>(opc, va[p], vb[p], vr[p], aux, da[p], db[p]);
    if (flags & RF_HAS_A)
      accumulate<FAST>(FAST ? loc(false, ao) : loc(flags & RF_A_GLOB, ao), (flags & RF_A_INIT) != 0, adj, da);
    if (flags & RF_HAS_B)
      accumulate<FAST>(FAST ? loc(false, bo) : loc(flags & RF_B_GLOB, bo), (flags & RF_B_INIT) != 0, adj, db);
  }

  __device__ __forceinline__ bool operator()(const unsigned char* raw, Stream<48>& st) const {
    const uint4 w0 = *reinterpret_cast<const uint4*>(raw);
    const uint4 w1 = *reinterpret_cast<const uint4*>(raw + 16);
    const uint2 w2 = *reinterpret_cast<const uint2*>(raw + 32);
    const uint32_t opc = w0.x & 0xFFu;
    const uint32_t flags = w0.x >> 16;
    const uint32_t ro = w0.y, ao = w0.z, bo = w0.w;
    const int32_t aux = (int32_t)w1.w;
    const double imm = __hiloint2double((int)w2.y, (int)w2.x);
    switch (opc) {
      case D_SEED: {
        V one[P];
#pragma unroll
        for (int p = 0; p < P; ++p) one[p] = Kd::c(1);
        C::st(loc(flags & RF_R_GLOB, ro), one);
        return true;
      }
      case D_CHAIN:
        return chain(st, flags, ro, ao, (uint32_t)aux);
      case D_CHAIN_LC:
        return chain_lc(st, flags, ro, ao, (uint32_t)aux);
      case D_NORM: {
        V a[P], one[P], t[P];
#pragma unroll
        for (int p = 0; p < P; ++p) one[p] = Kd::c(1);
        unsigned char* pr = loc(flags & RF_R_GLOB, ro);
        C::ld(pr, a);
        internal(a, one, t);
        C::st(pr, t);
        return true;
      }
      case D_GATHER:
        return gather(st, (uint32_t)aux);
      case D_STGRAD: {
        V g[P];
        if (ro == kNone) {
#pragma unroll
          for (int p = 0; p < P; ++p) g[p] = Kd::c(0);
        } else {
          C::ld(loc(flags & RF_R_GLOB, ro), g);
        }
#pragma unroll
        for (int p = 0; p < P; ++p)
          GradOut<V>::store(kp, unit0 + p, (uint32_t)aux, g[p], valid[p] && index_ok((uint32_t)aux, kp.ni, kp.err));
        return true;
      }
#define ECH_RF(OP) \
  case D_RF_BASE + OP: body<true>(OP, flags, ro, ao, bo, w1.x, w1.y, w1.z, aux, imm); return true;
      ECH_RF(OP_ADD) ECH_RF(OP_SUB) ECH_RF(OP_MUL) ECH_RF(OP_DIV) ECH_RF(OP_REM) ECH_RF(OP_POWF)
      ECH_RF(OP_ATAN2) ECH_RF(OP_HYPOT) ECH_RF(OP_MAX) ECH_RF(OP_MIN) ECH_RF(OP_NEG) ECH_RF(OP_RECIP)
      ECH_RF(OP_SQRT) ECH_RF(OP_CBRT) ECH_RF(OP_POWI) ECH_RF(OP_EXP) ECH_RF(OP_EXP2) ECH_RF(OP_EXPM1)
      ECH_RF(OP_LN) ECH_RF(OP_LOG2) ECH_RF(OP_LOG10) ECH_RF(OP_LN1P) ECH_RF(OP_SIN) ECH_RF(OP_COS)
      ECH_RF(OP_TAN) ECH_RF(OP_ASIN) ECH_RF(OP_ACOS) ECH_RF(OP_ATAN) ECH_RF(OP_SINH) ECH_RF(OP_COSH)
      ECH_RF(OP_TANH) ECH_RF(OP_ASINH) ECH_RF(OP_ACOSH) ECH_RF(OP_ATANH) ECH_RF(OP_ABS) ECH_RF(OP_SIGNUM)
      ECH_RF(OP_FLOOR) ECH_RF(OP_CEIL) ECH_RF(OP_ROUND) ECH_RF(OP_TRUNC) ECH_RF(OP_FRACT)
#undef ECH_RF
      default:
        body<false>(opc, flags, ro, ao, bo, w1.x, w1.y, w1.z, aux, imm);
        return true;
    }
  }
};

// ───────────────────────────── the sweep kernels ────────────────────────────
// One tile of `kp.tile` units: the forward program (with trajectory saves when
// REV), then the reverse program.  `gbase` is the CTA's global scratch region.
// Returns false when a bounded wait gave up (every thread sees the same value).
template <class V, int P, bool REV, bool DN, bool WS = false>
__device__ __forceinline__ bool sweep_tile(const KParams& kp, Ring& rg, unsigned char* sm, unsigned char* gbase,
                                           uint64_t t) {
  const uint32_t tile = kp.tile;
  const size_t colb = (size_t)threadIdx.x * P * sizeof(V);
  unsigned char* gs = gbase + colb;
  unsigned char* tj = kp.traj_smem ? sm + (size_t)kp.smem_regs * tile * sizeof(V)
                                   : gbase + (size_t)kp.far_slots * tile * sizeof(V) + colb;
  const uint64_t unit0 = t * tile + (uint64_t)threadIdx.x * P;
  uint32_t* bits = kp.dir_bits ? reinterpret_cast<uint32_t*>(rg.buf + kp.dir_bits) + threadIdx.x * P : nullptr;
  FwdExec<V, P, DN, WS> fx{kp, sm, gs, tj, unit0, bits, {}, {}, {}, {}, {}};
#pragma unroll
  for (int p = 0; p < P; ++p) {
    fx.valid[p] = unit0 + p < kp.n_units;
    fx.ui[p] = Lane<V>::info(kp, unit0 + p, fx.valid[p]);
  }
  if constexpr (JetOrder<V>::K > 0) {
    // source rows of the input jets that input-direct terms read (S > 0 launches)
    using T = typename dm::VT<V>::S;
#pragma unroll
    for (int p = 0; p < P; ++p) {
      const uint64_t row = kp.x_bcast ? 0 : (kp.S ? (uint64_t)fx.ui[p].pt : unit0 + p);
      fx.xrow[p] = reinterpret_cast<const T*>(kp.x) + row * kp.ni;
      fx.vrow[p] = kp.dir_mode == 1 ? reinterpret_cast<const T*>(kp.v) + (uint64_t)fx.ui[p].s * kp.ni : nullptr;
      fx.sel[p] = kp.dir_mode == 3 ? fx.ui[p].s : fx.ui[p].ent;
    }
    // the tile's Rademacher signs, one bit per input and unit (the same stream
    // as the per-input draw); each thread writes and reads its own units' words
    if (bits) {
      const uint32_t nw = (kp.ni + 31) / 32;
#pragma unroll
      for (int p = 0; p < P; ++p) {
#pragma unroll 1
        for (uint32_t w = 0; w < nw; ++w) {
          uint32_t word = 0;
          if (fx.valid[p]) {
#pragma unroll 1
            for (uint32_t b = 0; b < 32 && w * 32 + b < kp.ni; ++b)
              word |= (philox_bits(kp.seed, fx.ui[p].pt, fx.ui[p].s, w * 32 + b) & 1u) << b;
          }
          bits[w * tile + p] = word;
        }
      }
    }
  }
  if (!run_program<32>(rg, reinterpret_cast<const unsigned char*>(kp.fwd), kp.n_fwd, kp.err, fx)) return false;
  if (REV) {
    RevExec<V, P, DN> rx{kp, sm, gs, tj, unit0, {}};
#pragma unroll
    for (int p = 0; p < P; ++p) rx.valid[p] = fx.valid[p];
    if (!run_program<48>(rg, reinterpret_cast<const unsigned char*>(kp.rev), kp.n_rev, kp.err, rx)) return false;
  }
  return true;
}

// REV = false: forward program only (forward values, JVP, Taylor jets).
// REV = true : forward program with trajectory saves, then the reverse program
//              (gradient for plain values, HVP for Dual values).
// DN: with the dense-group executor (programs that hold D_DENSE instructions).
// WS: every warp's units are directions of one point (FwdExec).
template <class V, int P, bool REV, bool DN, bool WS = false>
__global__ void __launch_bounds__(256) sweep_kernel(KParams kp) {
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  __shared__ __align__(8) uint64_t full[kStages];
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) mbar_init(&full[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  Ring rg{smem_dyn, full, 0u, 0u};
  unsigned char* sm = smem_dyn + kRingBytes + (size_t)threadIdx.x * P * sizeof(V);
  unsigned char* gbase = reinterpret_cast<unsigned char*>(kp.scratch) + blockIdx.x * kp.scratch_stride_bytes;
  const uint64_t ntiles = (kp.n_units + kp.tile - 1) / kp.tile;
  for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x)
    if (!sweep_tile<V, P, REV, DN, WS>(kp, rg, sm, gbase, t)) return;
}

// ───────────────────────────── many tapes, one launch ───────────────────────
// Uneven batches of tapes (different programs, input sizes and point counts)
// as one persistent launch: the global tile list is the concatenation of every
// job's tiles (jobs ordered by the host, most expensive tile first), and CTAs
// take tiles from a global counter, so long and short tapes balance across
// SMs.  Each job is a complete parameter block; all jobs share the launch's
// tile size, shared-register budget and per-CTA scratch stride.
struct MultiJob {
  KParams kp;
  uint64_t first_tile;   // global id of the job's first tile
  uint64_t pad;
};

struct MultiParams {
  const MultiJob* jobs;
  uint32_t n_jobs;
  uint32_t total_tiles;
  uint32_t* next_tile;   // tile counter, zero at launch
  void* scratch;
  uint64_t stride;       // scratch bytes per CTA
};

template <class V, int P, bool DN>
__global__ void __launch_bounds__(256) multi_sweep_kernel(MultiParams mp) {
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  __shared__ __align__(8) uint64_t full[kStages];
  __shared__ __align__(16) KParams job;
  __shared__ uint32_t s_tile;
  __shared__ uint64_t s_local;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) mbar_init(&full[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  Ring rg{smem_dyn, full, 0u, 0u};
  unsigned char* sm = smem_dyn + kRingBytes + (size_t)threadIdx.x * P * sizeof(V);
  unsigned char* gbase = reinterpret_cast<unsigned char*>(mp.scratch) + blockIdx.x * mp.stride;
  for (;;) {
    if (threadIdx.x == 0) {
      const uint32_t g = atomicAdd(mp.next_tile, 1u);
      s_tile = g;
      if (g < mp.total_tiles) {
        uint32_t lo = 0, hi = mp.n_jobs - 1;   // last job with first_tile <= g
        while (lo < hi) {
          const uint32_t mid = (lo + hi + 1) / 2;
          if (mp.jobs[mid].first_tile <= g) lo = mid;
          else hi = mid - 1;
        }
        job = mp.jobs[lo].kp;
        s_local = g - mp.jobs[lo].first_tile;
      }
    }
    __syncthreads();
    if (s_tile >= mp.total_tiles) break;
    if (!sweep_tile<V, P, true, DN>(job, rg, sm, gbase, s_local)) return;
    __syncthreads();  // every thread is done with `job` before thread 0 replaces it
  }
}

}  // namespace ech
