// C ABI of the engine: context, tape upload, per-kind programs and dispatch.
//
// Reference boundary: echidna's CudaContext (src/gpu/cuda_backend.rs) and the
// GpuBackend trait (src/gpu/mod.rs:92-225); the declarations and the per-call
// reference citations are in include/echidna_b200.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <map>
#include <cmath>
#include <memory>
#include <atomic>
#include <condition_variable>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "../../include/echidna_b200.h"
#include "abi_internal.h"
#include "interp.cuh"
#include "launch.h"
#include "plan.h"

using namespace ech;

// ───────────────────────────── errors ───────────────────────────────────────
static thread_local std::string g_last_error;

static ech_status fail(ech_status st, const std::string& msg) {
  g_last_error = msg;
  return st;
}
static ech_status cuda_fail(cudaError_t e, const char* what) {
  if (e == cudaErrorMemoryAllocation) return fail(ECH_ERR_OUT_OF_MEMORY, "GPU out of memory");
  return fail(ECH_ERR_OTHER, std::string(what) + ": " + cudaGetErrorString(e));
}
#define CU(call)                                           \
  do {                                                     \
    cudaError_t e_ = (call);                               \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);    \
  } while (0)

extern "C" ECH_API const char* ech_last_error(void) { return g_last_error.c_str(); }
extern "C" ECH_API const char* ech_version(void) { return "echidna_b200 0.1.0 (sm_100a)"; }

// ───────────────────────────── device buffers ───────────────────────────────
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  ~DevBuf() { if (p) cudaFree(p); }
  cudaError_t ensure(size_t n) {
    if (n <= bytes) return cudaSuccess;
    if (p) { cudaFree(p); p = nullptr; bytes = 0; }
    size_t want = std::max<size_t>(n, 256);
    cudaError_t e = cudaMalloc(&p, want);
    if (e == cudaSuccess) bytes = want;
    return e;
  }
};

// Page-locked host staging memory (cudaHostAlloc), grown on demand.
struct PinnedBuf {
  void* p = nullptr;
  size_t bytes = 0;
  ~PinnedBuf() { if (p) cudaFreeHost(p); }
  cudaError_t ensure(size_t n) {
    if (n <= bytes) return cudaSuccess;
    if (p) { cudaFreeHost(p); p = nullptr; bytes = 0; }
    cudaError_t e = cudaHostAlloc(&p, n, cudaHostAllocDefault);
    if (e == cudaSuccess) bytes = n;
    return e;
  }
};

struct DevPlan {
  Plan host;
  DIns* d_fwd = nullptr;
  DRIns* d_rev = nullptr;
  uint32_t n_fwd = 0, n_rev = 0;  // records of the device programs (chain terms inline)
  uint32_t gather_tiles = 0;      // gather tiles in the reverse program
  // the program needs the kernel build with the dense-group executor
  bool needs_dense() const { return !host.dense.empty() || gather_tiles > 0; }
  ~DevPlan() {
    if (d_fwd) cudaFree(d_fwd);
    if (d_rev) cudaFree(d_rev);
  }
};

struct ech_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int sm_count = 0;
  size_t smem_optin = 0;
  size_t smem_per_sm = 0;      // shared memory per SM
  size_t smem_reserved = 0;    // shared memory the runtime reserves per block
  bool autotune = true;        // pick launch shapes by timing (per tape, kind, batch size)
  std::mutex mu;
  DevBuf scratch, io_in, io_in2, io_out, io_out2, io_out3, stde_tmp;
  // host-buffer sweeps of large batches run as pipe_chunks chunks, one stream
  // each (4, or ECHIDNA_B200_PIPE_CHUNKS in 1..8, read at context creation)
  static constexpr int kPipeMax = 8;
  int pipe_chunks = 4;
  cudaStream_t pipe[kPipeMax] = {};
  cudaEvent_t pipe_ev = nullptr;
  DevBuf pipe_scratch[kPipeMax];
  PinnedBuf pipe_stage[kPipeMax];   // staging for chunks of pageable host arrays
  uint32_t* d_err = nullptr;
  // resident CTAs per SM of a sweep kernel: (value kind, f64, order, points per
  // thread, reverse, dense build | warp-shared point << 1, threads, dynamic
  // shared memory) -> blocks
  std::map<std::tuple<int, int, int, int, int, int, int, size_t>, int> occupancy;
  // launch overrides (0 = automatic)
  uint32_t ov_threads = 0, ov_ppt = 0, ov_cap = 0;
  uint32_t ov_dense = 0;  // 1: the dense-group kernel build for every program (ech_ctx_set_dense_kernel)
  // ECH_FP32_* options of the FP32 batch STDE calls (0: reference rounding, FP64 reduction)
  uint32_t fp32_mode = 0;
};

// Launch shape: block size, points per thread, and how many CTAs should share
// an SM (which sets the shared-register cap).
struct Shape {
  uint32_t threads = 128, P = 1, ctas = 2;
  // 1: run the kernel build with the dense-group executor even for programs
  // without dense groups.  Both builds compute bit-identical results; the
  // tuner keeps the faster (the build without the executor needs fewer
  // registers, which pays where occupancy binds, not in one-warp launches).
  uint32_t dense_kernel = 0;
};

struct ech_tape {
  ech_ctx* ctx = nullptr;
  bool f64 = true;
  HostTape host;
  std::mutex mu;
  std::map<std::tuple<int, int, uint32_t, uint32_t, uint32_t, uint32_t>, std::unique_ptr<DevPlan>> plans;  // (kind, K, cap, tile, vbytes, P)
  // host-encoded programs for entry points that place them in their own memory
  struct HostProgram {
    Plan plan;
    DevProgram prog;
    uint64_t id = 0;  // process-unique, never reused: identifies the program's bytes
  };
  std::map<std::tuple<int, int, uint32_t, uint32_t, uint32_t, uint32_t>, std::unique_ptr<HostProgram>> host_programs;
  // autotuned launch shapes, keyed (kind, K, log2 of the unit count)
  std::map<std::tuple<int, int, int>, Shape> shapes;
  // for a step map x -> step(x): the tape of sum_j w_j step(x)_j over inputs (x, w)
  std::unique_ptr<ech_tape> vjp;
};

// ───────────────────────────── context ──────────────────────────────────────
extern "C" ECH_API ech_status ech_ctx_create(int device, ech_ctx** out) {
  if (!out) return fail(ECH_ERR_INVALID_ARG, "out is null");
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= device || device < 0)
    return fail(ECH_ERR_NO_DEVICE, "no suitable GPU device found");
  std::unique_ptr<ech_ctx> c(new ech_ctx());
  c->device = device;
  CU(cudaSetDevice(device));
  cudaDeviceProp prop;
  CU(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10) return fail(ECH_ERR_NO_DEVICE, "no suitable GPU device found (sm_100a required)");
  c->sm_count = prop.multiProcessorCount;
  c->smem_optin = prop.sharedMemPerBlockOptin;
  c->smem_per_sm = prop.sharedMemPerMultiprocessor;
  c->smem_reserved = prop.reservedSharedMemPerBlock;
  if (const char* e = std::getenv("ECHIDNA_B200_PIPE_CHUNKS")) {
    const long v = std::strtol(e, nullptr, 10);
    if (v >= 1 && v <= ech_ctx::kPipeMax) c->pipe_chunks = (int)v;
  }
  CU(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  CU(cudaMalloc(&c->d_err, sizeof(uint32_t)));
  CU(cudaMemset(c->d_err, 0, sizeof(uint32_t)));
  *out = c.release();
  return ECH_OK;
}

extern "C" ECH_API void ech_ctx_destroy(ech_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (cudaStream_t s : ctx->pipe)
    if (s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  if (ctx->pipe_ev) cudaEventDestroy(ctx->pipe_ev);
  if (ctx->d_err) cudaFree(ctx->d_err);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

extern "C" ECH_API ech_status ech_ctx_set_launch(ech_ctx* ctx, uint32_t threads, uint32_t ppt, uint32_t cap) {
  if (!ctx) return fail(ECH_ERR_INVALID_ARG, "ctx is null");
  if (threads && (threads % 32 || threads > 256)) return fail(ECH_ERR_INVALID_ARG, "threads must be a multiple of 32, <= 256");
  if (ppt && ppt != 1 && ppt != 2 && ppt != 4) return fail(ECH_ERR_INVALID_ARG, "points_per_thread must be 1, 2 or 4");
  ctx->ov_threads = threads;
  ctx->ov_ppt = ppt;
  ctx->ov_cap = cap;
  return ECH_OK;
}

extern "C" ECH_API ech_status ech_ctx_set_dense_kernel(ech_ctx* ctx, int always) {
  if (!ctx) return fail(ECH_ERR_INVALID_ARG, "ctx is null");
  ctx->ov_dense = always ? 1u : 0u;
  return ECH_OK;
}

extern "C" ECH_API ech_status ech_ctx_set_fp32_mode(ech_ctx* ctx, uint32_t flags) {
  if (!ctx) return fail(ECH_ERR_INVALID_ARG, "ctx is null");
  if (flags & ~(uint32_t)(ECH_FP32_COMPENSATED_JETS | ECH_FP32_COMPENSATED_MEANS | ECH_FP32_PLAIN_MEANS))
    return fail(ECH_ERR_INVALID_ARG, "unknown FP32 mode flag");
  if ((flags & ECH_FP32_COMPENSATED_MEANS) && (flags & ECH_FP32_PLAIN_MEANS))
    return fail(ECH_ERR_INVALID_ARG, "ECH_FP32_COMPENSATED_MEANS and ECH_FP32_PLAIN_MEANS exclude each other");
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->fp32_mode = flags;
  return ECH_OK;
}

extern "C" ECH_API ech_status ech_ctx_set_autotune(ech_ctx* ctx, int enable) {
  if (!ctx) return fail(ECH_ERR_INVALID_ARG, "ctx is null");
  ctx->autotune = enable != 0;
  return ECH_OK;
}

// ───────────────────────────── validation ───────────────────────────────────
extern "C" ECH_API ech_status ech_validate_bytecode_tape(const uint32_t* op, const uint32_t* a0, const uint32_t* a1,
                                                         uint32_t nv, uint32_t ni, uint32_t output_index,
                                                         const uint32_t* outs, uint32_t nouts, int has_custom) {
  if ((nv && (!op || !a0 || !a1)) || (nouts && !outs)) return fail(ECH_ERR_INVALID_ARG, "null tape array");
  std::string m = validate_bytecode_tape(op, a0, a1, nv, ni, output_index, outs, nouts, has_custom != 0);
  if (!m.empty()) return fail(ECH_ERR_OTHER, "invalid bytecode tape: " + m);
  return ECH_OK;
}

extern "C" ECH_API ech_status ech_validate_gpu_tape_data(const uint32_t* op, uint32_t n_op, const uint32_t* a0,
                                                         uint32_t n_a0, const uint32_t* a1, uint32_t n_a1,
                                                         uint32_t n_const, uint32_t num_ops, uint32_t num_inputs,
                                                         uint32_t num_variables, uint32_t output_index,
                                                         const uint32_t* outs, uint32_t nouts) {
  if ((n_op && !op) || (n_a0 && !a0) || (n_a1 && !a1) || (nouts && !outs))
    return fail(ECH_ERR_INVALID_ARG, "null tape array");
  std::string m = validate_gpu_tape_data(op, a0, a1, n_op, n_a0, n_a1, n_const, num_ops, num_inputs, num_variables,
                                         output_index, outs, nouts);
  if (!m.empty()) return fail(ECH_ERR_OTHER, "GPU error: invalid GpuTapeData: " + m);
  return ECH_OK;
}

// ───────────────────────────── upload ───────────────────────────────────────
static ech_status make_tape(ech_ctx* ctx, bool f64, HostTape&& h, ech_tape** out) {
  std::unique_ptr<ech_tape> t(new ech_tape());
  t->ctx = ctx;
  t->f64 = f64;
  t->host = std::move(h);
  *out = t.release();
  return ECH_OK;
}

extern "C" ECH_API ech_status ech_upload_tape_f32(ech_ctx* ctx, const uint32_t* op, uint32_t n_op, const uint32_t* a0,
                                                  uint32_t n_a0, const uint32_t* a1, uint32_t n_a1,
                                                  const float* consts, uint32_t n_const, uint32_t num_ops,
                                                  uint32_t num_inputs, uint32_t num_variables, uint32_t output_index,
                                                  const uint32_t* outs, uint32_t nouts, ech_tape** out) {
  if (!ctx || !out) return fail(ECH_ERR_INVALID_ARG, "ctx/out is null");
  *out = nullptr;
  if ((n_const && !consts)) return fail(ECH_ERR_INVALID_ARG, "null constants");
  ech_status st = ech_validate_gpu_tape_data(op, n_op, a0, n_a0, a1, n_a1, n_const, num_ops, num_inputs, num_variables,
                                             output_index, outs, nouts);
  if (st != ECH_OK) return fail(ECH_ERR_OTHER, "refusing to upload invalid GpuTapeData: " + g_last_error);
  HostTape h;
  h.nv = num_variables;
  h.ni = num_inputs;
  h.out_index = output_index;
  h.op.assign(op, op + n_op);
  h.a0.assign(a0, a0 + n_a0);
  h.a1.assign(a1, a1 + n_a1);
  h.vals.resize(n_const);
  for (uint32_t i = 0; i < n_const; ++i) h.vals[i] = (double)consts[i];
  // empty output_indices -> [output_index] (src/gpu/cuda_backend.rs:632-648)
  if (nouts == 0) h.outs.assign(1, output_index);
  else h.outs.assign(outs, outs + nouts);
  return make_tape(ctx, false, std::move(h), out);
}

extern "C" ECH_API ech_status ech_upload_tape_f64(ech_ctx* ctx, const uint32_t* op, const uint32_t* a0,
                                                  const uint32_t* a1, const double* values, uint32_t nv, uint32_t ni,
                                                  uint32_t output_index, const uint32_t* outs, uint32_t nouts,
                                                  int has_custom, ech_tape** out) {
  if (!ctx || !out) return fail(ECH_ERR_INVALID_ARG, "ctx/out is null");
  *out = nullptr;
  if (has_custom) return fail(ECH_ERR_CUSTOM_OPS_NOT_SUPPORTED, "tape contains custom ops which cannot run on GPU");
  if (nv && !values) return fail(ECH_ERR_INVALID_ARG, "null values");
  ech_status st = ech_validate_bytecode_tape(op, a0, a1, nv, ni, output_index, outs, nouts, 0);
  if (st != ECH_OK) return fail(ECH_ERR_OTHER, "GPU error: refusing to upload invalid tape: " + g_last_error);
  for (uint32_t i = 0; i < nv; ++i)
    if (op[i] == OP_CUSTOM) return fail(ECH_ERR_CUSTOM_OPS_NOT_SUPPORTED, "tape contains custom ops which cannot run on GPU");
  HostTape h;
  h.nv = nv;
  h.ni = ni;
  h.out_index = output_index;
  h.op.assign(op, op + nv);
  h.a0.assign(a0, a0 + nv);
  h.a1.assign(a1, a1 + nv);
  h.vals.assign(values, values + nv);
  if (nouts == 0) h.outs.assign(1, output_index);
  else h.outs.assign(outs, outs + nouts);
  return make_tape(ctx, true, std::move(h), out);
}

extern "C" ECH_API void ech_tape_destroy(ech_tape* t) { delete t; }
extern "C" ECH_API uint32_t ech_tape_num_outputs(const ech_tape* t) { return t ? (uint32_t)t->host.outs.size() : 0; }
extern "C" ECH_API uint32_t ech_tape_num_inputs(const ech_tape* t) { return t ? t->host.ni : 0; }
extern "C" ECH_API uint32_t ech_tape_num_variables(const ech_tape* t) { return t ? t->host.nv : 0; }

// ───────────────────────────── plans and launch configuration ───────────────

struct LaunchCfg {
  LaunchReq req;
  int threads = 128;
  uint32_t tile = 128;
  uint32_t cap = 0;
  size_t smem = 0;
  size_t smem_full = 0;  // the shape's whole per-CTA share of shared memory
  size_t vbytes = 0;
  bool dense_kernel = false;  // Shape::dense_kernel
};

static Kind kind_of(int k) {
  switch (k) {
    case 0: return Kind::Forward;
    case 1: return Kind::Gradient;
    case 2: return Kind::Hvp;
    case 3: return Kind::Jvp;
    case 5: return Kind::TaylorDirect;
    default: return Kind::Taylor;
  }
}

// The shared-register cap follows from the shape: the ring plus `cap`
// registers of `tile` values per CTA, `ctas` CTAs per SM.
static LaunchCfg cfg_for(ech_ctx* ctx, const ech_tape* t, int kind, int K, Shape sh) {
  LaunchCfg c;
  c.req.f64 = t->f64;
  c.req.K = K;
  c.req.vk = (kind == 2 || kind == 3) ? VKind::Dual : (kind == 4 ? VKind::Jet : VKind::Plain);
  c.req.rev = (kind == 1 || kind == 2);
  c.req.P = (int)sh.P;
  c.threads = (int)sh.threads;
  c.tile = sh.threads * sh.P;
  c.vbytes = value_bytes(c.req);
  c.dense_kernel = sh.dense_kernel != 0;
  // per-SM shared memory split between `ctas` CTAs, each paying the
  // per-block reservation and the kernel's static barriers
  const size_t per_sm = ctx->smem_per_sm ? ctx->smem_per_sm : 233472;
  size_t per_cta = per_sm / std::max<uint32_t>(sh.ctas, 1);
  per_cta = per_cta > ctx->smem_reserved + 128 ? per_cta - ctx->smem_reserved - 128 : 0;
  per_cta = std::min(per_cta, ctx->smem_optin);
  size_t cap = per_cta > (size_t)kRingBytes ? (per_cta - kRingBytes) / (c.tile * c.vbytes) : 0;
  if (ctx->ov_cap) cap = std::min<size_t>(cap, ctx->ov_cap);
  c.cap = (uint32_t)std::max<size_t>(cap, 1);
  c.smem_full = per_cta;
  return c;
}

// The fixed shape used with launch overrides, for small batches, and when
// autotuning is off: 128 threads, one point per thread, two CTAs per SM.
static LaunchCfg choose_cfg(ech_ctx* ctx, const ech_tape* t, int kind, int K) {
  Shape sh;
  sh.threads = ctx->ov_threads ? ctx->ov_threads : 128;
  sh.P = ctx->ov_ppt ? ctx->ov_ppt : 1;
  sh.ctas = ctx->ov_cap ? 1 : 2;
  sh.dense_kernel = ctx->ov_dense;
  return cfg_for(ctx, t, kind, K, sh);
}

// `dense`: form dense groups (up to dense_group_max(vbytes, P) chains); launches
// with compensated jet chains use plans without them.
static ech_status get_plan(ech_tape* t, int kind, int K, uint32_t cap, uint32_t tile, uint32_t vbytes, uint32_t P,
                           bool dense, DevPlan** out) {
  std::lock_guard<std::mutex> lk(t->mu);
  const uint32_t dmax = dense ? dense_group_max(vbytes, P) : 1u;
  auto key = std::make_tuple(kind, K, cap, tile, vbytes, dmax);
  auto it = t->plans.find(key);
  if (it != t->plans.end()) {
    *out = it->second.get();
    return ECH_OK;
  }
  std::unique_ptr<DevPlan> dp(new DevPlan());
  dp->host = build_plan(t->host, kind_of(kind), cap, dmax);
  DevProgram prog;
  std::string err;
  if (!encode_plan(dp->host, tile, vbytes, !t->f64, prog, err)) return fail(ECH_ERR_OTHER, err);
  CU(cudaMalloc(&dp->d_fwd, std::max<size_t>(prog.fwd.size(), 1) * sizeof(DIns)));
  if (!prog.fwd.empty())
    CU(cudaMemcpy(dp->d_fwd, prog.fwd.data(), prog.fwd.size() * sizeof(DIns), cudaMemcpyHostToDevice));
  CU(cudaMalloc(&dp->d_rev, std::max<size_t>(prog.rev.size(), 1) * sizeof(DRIns)));
  if (!prog.rev.empty())
    CU(cudaMemcpy(dp->d_rev, prog.rev.data(), prog.rev.size() * sizeof(DRIns), cudaMemcpyHostToDevice));
  dp->n_fwd = (uint32_t)prog.fwd.size();
  dp->n_rev = (uint32_t)prog.rev.size();
  dp->gather_tiles = prog.gather_tiles;
  *out = dp.get();
  t->plans[key] = std::move(dp);
  return ECH_OK;
}

// Enqueues one sweep.  All pointers are device pointers.
struct SweepIO {
  const void* x = nullptr;
  const void* v = nullptr;
  int x_bcast = 0;
  void* out = nullptr;
  void* out2 = nullptr;
  void* out3 = nullptr;
  uint32_t S = 0;
  int dir_mode = 0;
  uint64_t seed = 0;
  const uint32_t* seed_off = nullptr;  // dir_mode 5
  const void* seed_items = nullptr;
  int compensated = 0;                 // jets: compensated sums in linear chains (FP32 batch STDE option)
};

// Point-direction jet launches whose directions the kernel can evaluate per
// input (shared host directions, device Rademacher signs, basis vectors) run
// the input-direct program (Kind::TaylorDirect, plan kind 5): linear
// combinations of inputs read each input jet at its source instead of from a
// slot.  Device Rademacher signs are drawn once per tile into shared memory,
// ceil(ni/32) words per unit, taken from the shared-register budget.
static bool input_direct(int kind, const SweepIO& io) {
  return kind == 4 && io.S > 0 && io.dir_mode >= 1 && io.dir_mode <= 4;
}

static ech_status launch_cfg(ech_ctx* ctx, ech_tape* t, int kind, int K, uint64_t n_units, const SweepIO& io,
                             cudaStream_t st, LaunchCfg c, DevBuf* scratch = nullptr) {
  if (!scratch) scratch = &ctx->scratch;
  const bool direct = input_direct(kind, io);
  const size_t bits_bytes = (direct && io.dir_mode == 2) ? (size_t)((t->host.ni + 31) / 32) * c.tile * 4 : 0;
  if (bits_bytes) {
    const uint32_t reserve = (uint32_t)((bits_bytes + (size_t)c.tile * c.vbytes - 1) / ((size_t)c.tile * c.vbytes));
    c.cap = c.cap > reserve ? c.cap - reserve : 1;
  }
  DevPlan* dp = nullptr;
  ech_status s = get_plan(t, direct ? 5 : kind, K, c.cap, c.tile, (uint32_t)c.vbytes, (uint32_t)c.req.P,
                          io.compensated == 0, &dp);
  if (s != ECH_OK) return s;
  const Plan& p = dp->host;
  c.req.dense = dp->needs_dense() || c.dense_kernel;
  // every warp's 32 units are directions of one point: units u = point * S + s,
  // one per thread, warps start at multiples of 32
  c.req.warp_point = direct && K == 3 && c.req.P == 1 && io.S % 32u == 0;
  const uint32_t regs = std::max<uint32_t>(p.smem_regs, 1);
  c.smem = kRingBytes + (size_t)regs * c.tile * c.vbytes;
  const uint32_t dir_bits = bits_bytes ? (uint32_t)c.smem : 0u;
  c.smem += bits_bytes;
  if (c.smem > ctx->smem_optin) return fail(ECH_ERR_OTHER, "tape live set does not fit the shared-memory slot file");
  // the trajectory goes to shared memory when it fits the shape's share beside
  // the registers (narrow CTAs on small batches): the reverse then reads it at
  // shared-memory latency
  const size_t smem_traj = c.smem + (size_t)p.traj_slots * c.tile * c.vbytes;
  const bool traj_smem = p.traj_slots > 0 && smem_traj <= std::min(c.smem_full, ctx->smem_optin);
  if (traj_smem) c.smem = smem_traj;
  KParams kp{};
  kp.fwd = dp->d_fwd;
  kp.n_fwd = dp->n_fwd;
  kp.rev = dp->d_rev;
  kp.n_rev = c.req.rev ? dp->n_rev : 0u;
  kp.far_slots = p.far_slots;
  kp.traj_slots = p.traj_slots;
  kp.smem_regs = regs;
  kp.traj_smem = traj_smem ? 1u : 0u;
  kp.tile = c.tile;
  kp.n_units = n_units;
  kp.ni = t->host.ni;
  kp.no = (uint32_t)t->host.outs.size();
  kp.x = io.x;
  kp.v = io.v;
  kp.x_bcast = io.x_bcast;
  kp.out = io.out;
  kp.out2 = io.out2;
  kp.out3 = io.out3;
  kp.err = ctx->d_err;
  kp.S = io.S;
  kp.dir_mode = io.dir_mode;
  kp.seed = io.seed;
  kp.seed_off = io.seed_off;
  kp.seed_items = io.seed_items;
  kp.dir_bits = dir_bits;
  kp.compensated = (uint32_t)io.compensated;
  // occupancy per kernel and launch shape, queried once per context (callers hold ctx->mu)
  const auto okey = std::make_tuple((int)c.req.vk, (int)c.req.f64, c.req.K, c.req.P, (int)c.req.rev,
                                    (int)c.req.dense | ((int)c.req.warp_point << 1), (int)c.threads, c.smem);
  int bps = 0;
  cudaError_t e = cudaSuccess;
  auto oit = ctx->occupancy.find(okey);
  if (oit != ctx->occupancy.end()) {
    bps = oit->second;
  } else {
    e = launch_sweep(c.req, kp, 0, c.threads, c.smem, st, &bps);
    if (e != cudaSuccess) return cuda_fail(e, "occupancy query");
    ctx->occupancy[okey] = bps;
  }
  if (bps <= 0) return fail(ECH_ERR_OTHER, "tape live set does not fit the shared-memory slot file");
  const uint64_t ntiles = (n_units + c.tile - 1) / c.tile;
  const uint64_t grid = std::min<uint64_t>(ntiles, (uint64_t)bps * ctx->sm_count);
  const uint64_t slots = (uint64_t)p.far_slots + (traj_smem ? 0 : p.traj_slots);
  uint64_t stride = slots * c.tile * c.vbytes;
  stride = (stride + 255) & ~(uint64_t)255;
  CU(scratch->ensure(std::max<uint64_t>(stride * grid, 256)));
  kp.scratch = scratch->p;
  kp.scratch_stride_bytes = stride;
  if (grid == 0) return ECH_OK;
  e = launch_sweep(c.req, kp, (int)grid, c.threads, c.smem, st, &bps);
  if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
  return ECH_OK;
}

// Autotuning applies from this many units up; smaller batches use the fixed shape.
static constexpr uint64_t kTuneMinUnits = 512;

static int size_bucket(uint64_t n) {
  int b = 0;
  while ((1ull << (b + 1)) <= n && b < 40) ++b;
  return b;
}

// Candidate shapes, timed on the call's own inputs (every shape computes
// bit-identical results: a point's arithmetic does not depend on the launch).
// The narrow shapes (32 / 64 threads) spread batches of fewer than two
// 128-point tiles per SM over more SMs; they are only tried for such batches.
static const Shape kShapes[] = {
    {128, 1, 1}, {128, 1, 2}, {128, 1, 3}, {128, 1, 4}, {128, 2, 1}, {128, 2, 2},
    {128, 2, 3}, {128, 4, 1}, {128, 4, 2}, {256, 1, 1}, {256, 1, 2}, {64, 2, 4},
    {64, 1, 2}, {64, 1, 4}, {32, 1, 2}, {32, 1, 4}, {64, 1, 1}, {32, 1, 1},
};

static ech_status tune(ech_ctx* ctx, ech_tape* t, int kind, int K, uint64_t n_units, const SweepIO& io,
                       cudaStream_t st, Shape* best) {
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  ech_status first_err = ECH_OK;
  std::string first_msg;
  // one warm launch (plan build + upload), then one timed; < 0 when the shape fails
  auto time_shape = [&](const Shape& sh, bool warm) -> float {
    const LaunchCfg c = cfg_for(ctx, t, kind, K, sh);
    if (c.cap < 1 || kRingBytes + (size_t)c.tile * c.vbytes > ctx->smem_optin) return -1.0f;
    ech_status s = warm ? launch_cfg(ctx, t, kind, K, n_units, io, st, c) : ECH_OK;
    if (s == ECH_OK) {
      cudaEventRecord(e0, st);
      s = launch_cfg(ctx, t, kind, K, n_units, io, st, c);
      cudaEventRecord(e1, st);
    }
    if (s != ECH_OK) {
      if (first_err == ECH_OK) { first_err = s; first_msg = g_last_error; }
      return -1.0f;
    }
    if (cudaEventSynchronize(e1) != cudaSuccess) return -2.0f;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    return ms;
  };
  float best_ms = -1.0f;
  const bool small_batch = n_units < (uint64_t)2 * 128 * ctx->sm_count;
  for (const Shape& sh : kShapes) {
    if (sh.threads * sh.P < 128 && !small_batch) continue;
    const float ms = time_shape(sh, true);
    if (ms == -2.0f) break;
    if (ms < 0.0f) continue;
    if (best_ms < 0.0f || ms < best_ms) {
      best_ms = ms;
      *best = sh;
    }
  }
  if (best_ms >= 0.0f) {
    // the best shape on the other kernel build: three timings of each, interleaved; the
    // dense-group build (more registers, more instructions per record for programs
    // without dense groups) must win by 2 % to be kept
    Shape alt = *best;
    alt.dense_kernel = 1;
    float a_ms = time_shape(alt, true);
    if (a_ms >= 0.0f) {
      float b_ms = best_ms;
      for (int r = 0; r < 2; ++r) {
        const float b2 = time_shape(*best, false);
        const float a2 = time_shape(alt, false);
        if (b2 >= 0.0f) b_ms = std::min(b_ms, b2);
        if (a2 >= 0.0f) a_ms = std::min(a_ms, a2);
      }
      if (a_ms < 0.98f * b_ms) *best = alt;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (best_ms < 0.0f) return first_err != ECH_OK ? fail(first_err, first_msg) : fail(ECH_ERR_OTHER, "no launch shape fits");
  return ECH_OK;
}

static ech_status enqueue(ech_ctx* ctx, ech_tape* t, int kind, int K, uint64_t n_units, const SweepIO& io,
                          cudaStream_t st) {
  const bool overridden = ctx->ov_threads || ctx->ov_ppt || ctx->ov_cap || ctx->ov_dense;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (!overridden && ctx->autotune && n_units >= kTuneMinUnits && cudaStreamIsCapturing(st, &cap) == cudaSuccess &&
      cap == cudaStreamCaptureStatusNone) {
    const auto key = std::make_tuple(kind, K, size_bucket(n_units));
    Shape sh;
    bool have = false;
    {
      std::lock_guard<std::mutex> lk(t->mu);
      auto it = t->shapes.find(key);
      if (it != t->shapes.end()) { sh = it->second; have = true; }
    }
    if (!have) {
      ech_status s = tune(ctx, t, kind, K, n_units, io, st, &sh);
      if (s != ECH_OK) return s;
      std::lock_guard<std::mutex> lk(t->mu);
      t->shapes[key] = sh;
    }
    return launch_cfg(ctx, t, kind, K, n_units, io, st, cfg_for(ctx, t, kind, K, sh));
  }
  return launch_cfg(ctx, t, kind, K, n_units, io, st, choose_cfg(ctx, t, kind, K));
}

// ── host-buffer sweeps in chunks ──
// A host-buffer call on a large batch whose launch shape is already tuned runs
// as ctx->pipe_chunks chunks, each on its own stream: copy its inputs in, sweep,
// copy its outputs out, so the copies of one chunk overlap the sweeps of the
// others.  Every chunk uses the whole batch's tuned shape (the chunks' kernels
// run side by side and together fill the GPU like one launch) and its own
// per-CTA scratch.  Results are the same as one launch (a point's arithmetic
// does not depend on the launch).  The first call of a (tape, kind, batch
// octave) runs whole and tunes the shape.
struct PipeArray {
  void* dev;          // device base (inputs: destination; outputs: source)
  void* host;         // host base
  size_t unit_bytes;  // bytes per unit
  bool in;
};
static constexpr uint64_t kPipeMinUnits = 16384;

// True for host memory the CUDA runtime has not page-locked (ordinary allocations).
static bool host_pageable(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // clear the sticky-free error of an unknown pointer
    return true;
  }
  return a.type == cudaMemoryTypeUnregistered;
}

// memcpy on a few host threads for large copies (staging of pageable arrays).
// Host memcpy of staged chunks, split over a process-wide pool of copy threads
// (started on first use and kept, so a copy costs no thread creation): the
// caller copies parts too, and returns when every part is done.  One copy runs
// at a time; calls from several threads queue on the pool's mutex.
class CopyPool {
 public:
  static CopyPool& get() {
    static CopyPool pool;
    return pool;
  }
  void copy(void* dst, const void* src, size_t bytes) {
    constexpr size_t kPart = 1u << 20;
    const size_t parts = std::min<size_t>(workers_.size() + 1, (bytes + kPart - 1) / kPart);
    if (parts <= 1) {
      memcpy(dst, src, bytes);
      return;
    }
    std::lock_guard<std::mutex> one(job_mu_);
    {
      std::lock_guard<std::mutex> lk(mu_);
      dst_ = (char*)dst;
      src_ = (const char*)src;
      bytes_ = bytes;
      step_ = (bytes + parts - 1) / parts;
      parts_ = parts;
      next_.store(0);
      left_ = parts;
      ++generation_;
    }
    cv_.notify_all();
    work();
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [&] { return left_ == 0; });
  }

 private:
  // min(hardware threads, 16) copiers in all (the caller and the workers), or
  // ECHIDNA_B200_COPY_THREADS (1..64) when set
  CopyPool() {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    unsigned n = std::min(hw, 16u);
    if (const char* e = std::getenv("ECHIDNA_B200_COPY_THREADS")) {
      const long v = std::strtol(e, nullptr, 10);
      if (v >= 1 && v <= 64) n = (unsigned)v;
    }
    for (unsigned i = 1; i < n; ++i) workers_.emplace_back([this] { loop(); });
  }
  ~CopyPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (std::thread& t : workers_) t.join();
  }
  // copies parts until none is left
  void work() {
    for (;;) {
      const size_t i = next_.fetch_add(1);
      if (i >= parts_) return;
      const size_t b = i * step_;
      if (b < bytes_) memcpy(dst_ + b, src_ + b, std::min(step_, bytes_ - b));
      std::lock_guard<std::mutex> lk(mu_);
      if (--left_ == 0) done_cv_.notify_all();
    }
  }
  void loop() {
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return stop_ || generation_ != seen; });
        if (stop_) return;
        seen = generation_;
      }
      work();
    }
  }
  std::vector<std::thread> workers_;
  std::mutex job_mu_, mu_;
  std::condition_variable cv_, done_cv_;
  char* dst_ = nullptr;
  const char* src_ = nullptr;
  size_t bytes_ = 0, step_ = 0, parts_ = 0, left_ = 0;
  std::atomic<size_t> next_{0};
  uint64_t generation_ = 0;
  bool stop_ = false;
};

static void host_copy(void* dst, const void* src, size_t bytes) { CopyPool::get().copy(dst, src, bytes); }

static ech_status run_pipelined(ech_ctx* ctx, ech_tape* t, int kind, uint64_t n_units, const SweepIO& io,
                                const size_t io_unit_bytes[5], const std::vector<PipeArray>& arrays, bool* done) {
  *done = false;
  const bool overridden = ctx->ov_threads || ctx->ov_ppt || ctx->ov_cap || ctx->ov_dense;
  if (overridden || !ctx->autotune || n_units < kPipeMinUnits) return ECH_OK;
  Shape sh;
  {
    std::lock_guard<std::mutex> lk(t->mu);
    auto it = t->shapes.find(std::make_tuple(kind, 0, size_bucket(n_units)));
    if (it == t->shapes.end()) return ECH_OK;
    sh = it->second;
  }
  const LaunchCfg c = cfg_for(ctx, t, kind, 0, sh);
  if (!ctx->pipe_ev) CU(cudaEventCreateWithFlags(&ctx->pipe_ev, cudaEventDisableTiming));
  const int nc = ctx->pipe_chunks;
  for (int k = 0; k < nc; ++k)
    if (!ctx->pipe[k]) CU(cudaStreamCreateWithFlags(&ctx->pipe[k], cudaStreamNonBlocking));
  // the chunks start after the context stream's earlier work
  CU(cudaEventRecord(ctx->pipe_ev, ctx->stream));
  uint64_t per = (n_units + nc - 1) / nc;
  per = (per + c.tile - 1) / c.tile * c.tile;
  // Pageable host arrays (what a caller's ordinary allocations are) go through
  // the context's page-locked staging buffers, one per chunk: the host copies a
  // chunk's inputs in while earlier chunks' copies and sweeps run, and copies
  // each chunk's outputs out as soon as its stream is done.
  std::vector<uint8_t> staged(arrays.size(), 0);
  size_t stage_bytes = 0;
  for (size_t q = 0; q < arrays.size(); ++q) {
    staged[q] = host_pageable(arrays[q].host) ? 1 : 0;
    if (staged[q]) stage_bytes += per * arrays[q].unit_bytes;
  }
  if (stage_bytes)
    for (PinnedBuf& b : ctx->pipe_stage) CU(b.ensure(stage_bytes));
  auto stage_at = [&](int k, size_t q) {
    size_t o = 0;
    for (size_t r = 0; r < q; ++r)
      if (staged[r]) o += per * arrays[r].unit_bytes;
    return (unsigned char*)ctx->pipe_stage[k].p + o;
  };
  ech_status first = ECH_OK;
  int issued = 0;
  for (int k = 0; k < nc; ++k) {
    const uint64_t off = (uint64_t)k * per;
    if (off >= n_units) break;
    const uint64_t n = std::min<uint64_t>(per, n_units - off);
    cudaStream_t st = ctx->pipe[k];
    cudaError_t e = cudaStreamWaitEvent(st, ctx->pipe_ev, 0);
    issued = k + 1;
    for (size_t q = 0; q < arrays.size(); ++q) {
      const PipeArray& a = arrays[q];
      if (e != cudaSuccess || !a.in) continue;
      const unsigned char* src = (const unsigned char*)a.host + off * a.unit_bytes;
      if (staged[q]) {
        host_copy(stage_at(k, q), src, n * a.unit_bytes);
        src = stage_at(k, q);
      }
      e = cudaMemcpyAsync((unsigned char*)a.dev + off * a.unit_bytes, src, n * a.unit_bytes, cudaMemcpyHostToDevice,
                          st);
    }
    if (e != cudaSuccess) {
      first = cuda_fail(e, "chunk copy");
      break;
    }
    SweepIO ck = io;
    auto shift = [&](const void* p, size_t ub) -> const void* {
      return (p && ub) ? (const void*)((const unsigned char*)p + off * ub) : p;
    };
    ck.x = shift(io.x, io_unit_bytes[0]);
    ck.v = shift(io.v, io_unit_bytes[1]);
    ck.out = const_cast<void*>(shift(io.out, io_unit_bytes[2]));
    ck.out2 = const_cast<void*>(shift(io.out2, io_unit_bytes[3]));
    ck.out3 = const_cast<void*>(shift(io.out3, io_unit_bytes[4]));
    ech_status s = launch_cfg(ctx, t, kind, 0, n, ck, st, c, &ctx->pipe_scratch[k]);
    if (s != ECH_OK) {
      first = s;
      break;
    }
    for (size_t q = 0; q < arrays.size(); ++q) {
      const PipeArray& a = arrays[q];
      if (e != cudaSuccess || a.in) continue;
      unsigned char* dst = staged[q] ? stage_at(k, q) : (unsigned char*)a.host + off * a.unit_bytes;
      e = cudaMemcpyAsync(dst, (const unsigned char*)a.dev + off * a.unit_bytes, n * a.unit_bytes,
                          cudaMemcpyDeviceToHost, st);
    }
    if (e != cudaSuccess) {
      first = cuda_fail(e, "chunk copy");
      break;
    }
  }
  // every chunk's copies finish before the host buffers are handed back;
  // staged outputs are copied out chunk by chunk as their streams finish
  for (int k = 0; k < nc; ++k) {
    cudaError_t e = cudaStreamSynchronize(ctx->pipe[k]);
    if (e != cudaSuccess && first == ECH_OK) first = cuda_fail(e, "chunk sync");
    if (e != cudaSuccess || first != ECH_OK || k >= issued) continue;
    const uint64_t off = (uint64_t)k * per;
    const uint64_t n = std::min<uint64_t>(per, n_units - off);
    for (size_t q = 0; q < arrays.size(); ++q) {
      const PipeArray& a = arrays[q];
      if (a.in || !staged[q]) continue;
      host_copy((unsigned char*)a.host + off * a.unit_bytes, stage_at(k, q), n * a.unit_bytes);
    }
  }
  if (first != ECH_OK) return first;
  *done = true;
  return ECH_OK;
}

static ech_status check_err_word(ech_ctx* ctx) {
  uint32_t h = 0;
  CU(cudaMemcpy(&h, ctx->d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost));
  if (h) {
    CU(cudaMemset(ctx->d_err, 0, sizeof(uint32_t)));
    if (h & KERR_TIMEOUT) return fail(ECH_ERR_TIMEOUT, "device-side wait timed out");
    if (h & KERR_BOUNDS) return fail(ECH_ERR_OTHER, "device bounds check failed: a slot or index out of its region");
    return fail(ECH_ERR_OTHER, "device reported a malformed instruction");
  }
  return ECH_OK;
}

// validate_batch_args (src/gpu/mod.rs:572-582)
static ech_status batch_args(const ech_tape* t, uint64_t batch) {
  if (batch == 0) return fail(ECH_ERR_OTHER, "batch_size must be non-zero");
  if (t->host.ni == 0)
    return fail(ECH_ERR_OTHER, "tape has no inputs (constant function); evaluate it on the CPU instead");
  return ECH_OK;
}

static ech_status common_checks(ech_ctx* ctx, const ech_tape* t, bool f64) {
  if (!ctx || !t) return fail(ECH_ERR_INVALID_ARG, "ctx/tape is null");
  if (t->ctx != ctx) return fail(ECH_ERR_INVALID_ARG, "tape was uploaded on a different context");
  if (t->f64 != f64)
    return fail(ECH_ERR_INVALID_ARG, f64 ? "tape was uploaded with f32 constants" : "tape was uploaded with f64 constants");
  return ECH_OK;
}

#define CHECK(x)                      \
  do {                                \
    ech_status s_ = (x);              \
    if (s_ != ECH_OK) return s_;      \
  } while (0)

static ech_status len_check(size_t got, uint64_t want, const char* what) {
  if (got != want) {
    char buf[160];
    snprintf(buf, sizeof buf, "%s length mismatch: got %zu, expected %llu", what, got, (unsigned long long)want);
    return fail(ECH_ERR_INVALID_ARG, buf);
  }
  return ECH_OK;
}

// ───────────────────────────── host-buffer entry points ─────────────────────
template <class T>
static ech_status do_forward(ech_ctx* ctx, const ech_tape* tc, const T* in, size_t n_in, uint32_t B, T* out,
                             size_t n_out) {
  const bool f64 = sizeof(T) == 8;
  CHECK(common_checks(ctx, tc, f64));
  ech_tape* t = const_cast<ech_tape*>(tc);
  CHECK(batch_args(t, B));
  const uint64_t ni = t->host.ni, no = t->host.outs.size();
  CHECK(len_check(n_in, (uint64_t)B * ni, "inputs"));
  CHECK(len_check(n_out, (uint64_t)B * no, "outputs"));
  if (!in || !out) return fail(ECH_ERR_INVALID_ARG, "null buffer");
  std::lock_guard<std::mutex> lk(ctx->mu);
  CU(cudaSetDevice(ctx->device));
  CU(ctx->io_in.ensure(n_in * sizeof(T)));
  CU(ctx->io_out.ensure(n_out * sizeof(T)));
  CU(cudaMemcpyAsync(ctx->io_in.p, in, n_in * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
  SweepIO io;
  io.x = ctx->io_in.p;
  io.out = ctx->io_out.p;
  CHECK(enqueue(ctx, t, 0, 0, B, io, ctx->stream));
  CU(cudaMemcpyAsync(out, ctx->io_out.p, n_out * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  return check_err_word(ctx);
}

template <class T>
static ech_status do_gradient(ech_ctx* ctx, const ech_tape* tc, const T* in, size_t n_in, uint32_t B, T* out,
                              size_t n_out, T* grads, size_t n_grads) {
  const bool f64 = sizeof(T) == 8;
  CHECK(common_checks(ctx, tc, f64));
  ech_tape* t = const_cast<ech_tape*>(tc);
  CHECK(batch_args(t, B));
  const uint64_t ni = t->host.ni, no = t->host.outs.size();
  CHECK(len_check(n_in, (uint64_t)B * ni, "inputs"));
  CHECK(len_check(n_out, (uint64_t)B * no, "outputs"));
  CHECK(len_check(n_grads, (uint64_t)B * ni, "grads"));
  if (!in || !out || !grads) return fail(ECH_ERR_INVALID_ARG, "null buffer");
  std::lock_guard<std::mutex> lk(ctx->mu);
  CU(cudaSetDevice(ctx->device));
  CU(ctx->io_in.ensure(n_in * sizeof(T)));
  CU(ctx->io_out.ensure(n_out * sizeof(T)));
  CU(ctx->io_out2.ensure(n_grads * sizeof(T)));
  SweepIO io;
  io.x = ctx->io_in.p;
  io.out = ctx->io_out.p;
  io.out2 = ctx->io_out2.p;
  {
    const size_t ub[5] = {ni * sizeof(T), 0, no * sizeof(T), ni * sizeof(T), 0};
    const std::vector<PipeArray> arr = {{ctx->io_in.p, const_cast<T*>(in), ni * sizeof(T), true},
                                        {ctx->io_out.p, out, no * sizeof(T), false},
                                        {ctx->io_out2.p, grads, ni * sizeof(T), false}};
    bool done = false;
    CHECK(run_pipelined(ctx, t, 1, B, io, ub, arr, &done));
    if (done) return check_err_word(ctx);
  }
  CU(cudaMemcpyAsync(ctx->io_in.p, in, n_in * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
  CHECK(enqueue(ctx, t, 1, 0, B, io, ctx->stream));
  CU(cudaMemcpyAsync(out, ctx->io_out.p, n_out * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaMemcpyAsync(grads, ctx->io_out2.p, n_grads * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  return check_err_word(ctx);
}

template <class T>
static ech_status do_hvp(ech_ctx* ctx, const ech_tape* tc, const T* x, size_t n_x, bool per_point, const T* dirs,
                         size_t n_dirs, uint32_t B, T* grads, size_t n_grads, T* hvps, size_t n_hvps) {
  const bool f64 = sizeof(T) == 8;
  CHECK(common_checks(ctx, tc, f64));
  ech_tape* t = const_cast<ech_tape*>(tc);
  CHECK(batch_args(t, B));
  const uint64_t ni = t->host.ni;
  CHECK(len_check(n_x, per_point ? (uint64_t)B * ni : ni, "x"));
  CHECK(len_check(n_dirs, (uint64_t)B * ni, "tangent_dirs"));
  CHECK(len_check(n_grads, (uint64_t)B * ni, "grads"));
  CHECK(len_check(n_hvps, (uint64_t)B * ni, "hvps"));
  if (!x || !dirs || !grads || !hvps) return fail(ECH_ERR_INVALID_ARG, "null buffer");
  std::lock_guard<std::mutex> lk(ctx->mu);
  CU(cudaSetDevice(ctx->device));
  CU(ctx->io_in.ensure(n_x * sizeof(T)));
  CU(ctx->io_in2.ensure(n_dirs * sizeof(T)));
  CU(ctx->io_out2.ensure(n_grads * sizeof(T)));
  CU(ctx->io_out3.ensure(n_hvps * sizeof(T)));
  SweepIO io;
  io.x = ctx->io_in.p;
  io.v = ctx->io_in2.p;
  io.x_bcast = per_point ? 0 : 1;
  io.out2 = ctx->io_out2.p;
  io.out3 = ctx->io_out3.p;
  if (per_point) {
    const size_t ub[5] = {ni * sizeof(T), ni * sizeof(T), 0, ni * sizeof(T), ni * sizeof(T)};
    const std::vector<PipeArray> arr = {{ctx->io_in.p, const_cast<T*>(x), ni * sizeof(T), true},
                                        {ctx->io_in2.p, const_cast<T*>(dirs), ni * sizeof(T), true},
                                        {ctx->io_out2.p, grads, ni * sizeof(T), false},
                                        {ctx->io_out3.p, hvps, ni * sizeof(T), false}};
    bool done = false;
    CHECK(run_pipelined(ctx, t, 2, B, io, ub, arr, &done));
    if (done) return check_err_word(ctx);
  }
  CU(cudaMemcpyAsync(ctx->io_in.p, x, n_x * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaMemcpyAsync(ctx->io_in2.p, dirs, n_dirs * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
  CHECK(enqueue(ctx, t, 2, 0, B, io, ctx->stream));
  CU(cudaMemcpyAsync(grads, ctx->io_out2.p, n_grads * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaMemcpyAsync(hvps, ctx->io_out3.p, n_hvps * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  return check_err_word(ctx);
}

template <class T>
static ech_status do_tangent(ech_ctx* ctx, const ech_tape* tc, const T* x, size_t n_x, const T* seeds, size_t n_seeds,
                             uint32_t B, T* vals, T* tans, size_t n_out) {
  const bool f64 = sizeof(T) == 8;
  CHECK(common_checks(ctx, tc, f64));
  ech_tape* t = const_cast<ech_tape*>(tc);
  CHECK(batch_args(t, B));
  const uint64_t ni = t->host.ni, no = t->host.outs.size();
  CHECK(len_check(n_x, (uint64_t)B * ni, "primal_inputs"));
  CHECK(len_check(n_seeds, (uint64_t)B * ni, "tangent_seeds"));
  CHECK(len_check(n_out, (uint64_t)B * no, "outputs"));
  if (!x || !seeds || !tans) return fail(ECH_ERR_INVALID_ARG, "null buffer");
  std::lock_guard<std::mutex> lk(ctx->mu);
  CU(cudaSetDevice(ctx->device));
  CU(ctx->io_in.ensure(n_x * sizeof(T)));
  CU(ctx->io_in2.ensure(n_seeds * sizeof(T)));
  CU(ctx->io_out.ensure(n_out * sizeof(T)));
  CU(ctx->io_out2.ensure(n_out * sizeof(T)));
  CU(cudaMemcpyAsync(ctx->io_in.p, x, n_x * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaMemcpyAsync(ctx->io_in2.p, seeds, n_seeds * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
  SweepIO io;
  io.x = ctx->io_in.p;
  io.v = ctx->io_in2.p;
  io.out = ctx->io_out.p;
  io.out2 = ctx->io_out2.p;
  CHECK(enqueue(ctx, t, 3, 0, B, io, ctx->stream));
  if (vals) CU(cudaMemcpyAsync(vals, ctx->io_out.p, n_out * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaMemcpyAsync(tans, ctx->io_out2.p, n_out * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  return check_err_word(ctx);
}

template <class T>
static ech_status do_taylor(ech_ctx* ctx, const ech_tape* tc, const T* P, size_t n_p, const T* S, size_t n_s,
                            uint32_t B, uint32_t order, T* coeffs, size_t n_c) {
  const bool f64 = sizeof(T) == 8;
  CHECK(common_checks(ctx, tc, f64));
  ech_tape* t = const_cast<ech_tape*>(tc);
  if (order < 1 || order > 5) {
    char buf[96];
    snprintf(buf, sizeof buf, "unsupported Taylor order %u, must be 1..=5", order);
    return fail(ECH_ERR_OTHER, buf);
  }
  CHECK(batch_args(t, B));
  const uint64_t ni = t->host.ni, no = t->host.outs.size();
  CHECK(len_check(n_p, (uint64_t)B * ni, "primal_inputs"));
  CHECK(len_check(n_s, (uint64_t)B * ni, "direction_seeds"));
  CHECK(len_check(n_c, (uint64_t)order * B * no, "coefficients"));
  if (!P || !S || !coeffs) return fail(ECH_ERR_INVALID_ARG, "null buffer");
  std::lock_guard<std::mutex> lk(ctx->mu);
  CU(cudaSetDevice(ctx->device));
  CU(ctx->io_in.ensure(n_p * sizeof(T)));
  CU(ctx->io_in2.ensure(n_s * sizeof(T)));
  CU(ctx->io_out.ensure(n_c * sizeof(T)));
  CU(cudaMemcpyAsync(ctx->io_in.p, P, n_p * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaMemcpyAsync(ctx->io_in2.p, S, n_s * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
  SweepIO io;
  io.x = ctx->io_in.p;
  io.v = ctx->io_in2.p;
  io.out = ctx->io_out.p;
  CHECK(enqueue(ctx, t, 4, (int)order, B, io, ctx->stream));
  CU(cudaMemcpyAsync(coeffs, ctx->io_out.p, n_c * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  return check_err_word(ctx);
}

extern "C" {

ECH_API ech_status ech_forward_batch_f32(ech_ctx* c, const ech_tape* t, const float* in, size_t n_in, uint32_t B,
                                         float* out, size_t n_out) {
  return do_forward<float>(c, t, in, n_in, B, out, n_out);
}
ECH_API ech_status ech_forward_batch_f64(ech_ctx* c, const ech_tape* t, const double* in, size_t n_in, uint32_t B,
                                         double* out, size_t n_out) {
  return do_forward<double>(c, t, in, n_in, B, out, n_out);
}
ECH_API ech_status ech_gradient_batch_f32(ech_ctx* c, const ech_tape* t, const float* in, size_t n_in, uint32_t B,
                                          float* out, size_t n_out, float* g, size_t n_g) {
  return do_gradient<float>(c, t, in, n_in, B, out, n_out, g, n_g);
}
ECH_API ech_status ech_gradient_batch_f64(ech_ctx* c, const ech_tape* t, const double* in, size_t n_in, uint32_t B,
                                          double* out, size_t n_out, double* g, size_t n_g) {
  return do_gradient<double>(c, t, in, n_in, B, out, n_out, g, n_g);
}
ECH_API ech_status ech_hvp_batch_f32(ech_ctx* c, const ech_tape* t, const float* x, size_t n_x, const float* d,
                                     size_t n_d, uint32_t B, float* g, size_t n_g, float* h, size_t n_h) {
  return do_hvp<float>(c, t, x, n_x, false, d, n_d, B, g, n_g, h, n_h);
}
ECH_API ech_status ech_hvp_batch_f64(ech_ctx* c, const ech_tape* t, const double* x, size_t n_x, const double* d,
                                     size_t n_d, uint32_t B, double* g, size_t n_g, double* h, size_t n_h) {
  return do_hvp<double>(c, t, x, n_x, false, d, n_d, B, g, n_g, h, n_h);
}
ECH_API ech_status ech_hvp_batch_points_f32(ech_ctx* c, const ech_tape* t, const float* x, size_t n_x, const float* d,
                                            size_t n_d, uint32_t B, float* g, size_t n_g, float* h, size_t n_h) {
  return do_hvp<float>(c, t, x, n_x, true, d, n_d, B, g, n_g, h, n_h);
}
ECH_API ech_status ech_hvp_batch_points_f64(ech_ctx* c, const ech_tape* t, const double* x, size_t n_x,
                                            const double* d, size_t n_d, uint32_t B, double* g, size_t n_g, double* h,
                                            size_t n_h) {
  return do_hvp<double>(c, t, x, n_x, true, d, n_d, B, g, n_g, h, n_h);
}
ECH_API ech_status ech_tangent_forward_batch_f32(ech_ctx* c, const ech_tape* t, const float* x, size_t n_x,
                                                 const float* s, size_t n_s, uint32_t B, float* v, float* tn,
                                                 size_t n_o) {
  return do_tangent<float>(c, t, x, n_x, s, n_s, B, v, tn, n_o);
}
ECH_API ech_status ech_tangent_forward_batch_f64(ech_ctx* c, const ech_tape* t, const double* x, size_t n_x,
                                                 const double* s, size_t n_s, uint32_t B, double* v, double* tn,
                                                 size_t n_o) {
  return do_tangent<double>(c, t, x, n_x, s, n_s, B, v, tn, n_o);
}
ECH_API ech_status ech_taylor_forward_kth_batch_f32(ech_ctx* c, const ech_tape* t, const float* p, size_t n_p,
                                                    const float* s, size_t n_s, uint32_t B, uint32_t order,
                                                    float* co, size_t n_co) {
  return do_taylor<float>(c, t, p, n_p, s, n_s, B, order, co, n_co);
}
ECH_API ech_status ech_taylor_forward_kth_batch_f64(ech_ctx* c, const ech_tape* t, const double* p, size_t n_p,
                                                    const double* s, size_t n_s, uint32_t B, uint32_t order,
                                                    double* co, size_t n_co) {
  return do_taylor<double>(c, t, p, n_p, s, n_s, B, order, co, n_co);
}

// ── device-pointer variants ──
ECH_API ech_status ech_forward_batch_device(ech_ctx* ctx, const ech_tape* t, int f64, const void* in, uint32_t B,
                                            void* out, void* stream) {
  CHECK(common_checks(ctx, t, f64 != 0));
  CHECK(batch_args(t, B));
  std::lock_guard<std::mutex> lk(ctx->mu);
  CU(cudaSetDevice(ctx->device));
  SweepIO io;
  io.x = in;
  io.out = out;
  return enqueue(ctx, const_cast<ech_tape*>(t), 0, 0, B, io, stream ? (cudaStream_t)stream : ctx->stream);
}
ECH_API ech_status ech_gradient_batch_device(ech_ctx* ctx, const ech_tape* t, int f64, const void* in, uint32_t B,
                                             void* out, void* grads, void* stream) {
  CHECK(common_checks(ctx, t, f64 != 0));
  CHECK(batch_args(t, B));
  std::lock_guard<std::mutex> lk(ctx->mu);
  CU(cudaSetDevice(ctx->device));
  SweepIO io;
  io.x = in;
  io.out = out;
  io.out2 = grads;
  return enqueue(ctx, const_cast<ech_tape*>(t), 1, 0, B, io, stream ? (cudaStream_t)stream : ctx->stream);
}
ECH_API ech_status ech_hvp_batch_device(ech_ctx* ctx, const ech_tape* t, int f64, const void* xs, int x_per_point,
                                        const void* dirs, uint32_t B, void* grads, void* hvps, void* stream) {
  CHECK(common_checks(ctx, t, f64 != 0));
  CHECK(batch_args(t, B));
  std::lock_guard<std::mutex> lk(ctx->mu);
  CU(cudaSetDevice(ctx->device));
  SweepIO io;
  io.x = xs;
  io.v = dirs;
  io.x_bcast = x_per_point ? 0 : 1;
  io.out2 = grads;
  io.out3 = hvps;
  return enqueue(ctx, const_cast<ech_tape*>(t), 2, 0, B, io, stream ? (cudaStream_t)stream : ctx->stream);
}
ECH_API ech_status ech_taylor_batch_device(ech_ctx* ctx, const ech_tape* t, int f64, const void* p, const void* s,
                                           uint32_t B, uint32_t order, void* coeffs, void* stream) {
  CHECK(common_checks(ctx, t, f64 != 0));
  if (order < 1 || order > 5) return fail(ECH_ERR_OTHER, "unsupported Taylor order, must be 1..=5");
  CHECK(batch_args(t, B));
  std::lock_guard<std::mutex> lk(ctx->mu);
  CU(cudaSetDevice(ctx->device));
  SweepIO io;
  io.x = p;
  io.v = s;
  io.out = coeffs;
  return enqueue(ctx, const_cast<ech_tape*>(t), 4, (int)order, B, io, stream ? (cudaStream_t)stream : ctx->stream);
}
}  // extern "C"

// ── STDE (src/gpu/stde_gpu.rs) ──
// require_scalar_output / require_nonempty_x (src/gpu/stde_gpu.rs:16-40)
static ech_status stde_checks(const ech_tape* t, size_t n, const char* caller, const char* quantity) {
  if (t->host.outs.size() != 1) {
    char buf[160];
    snprintf(buf, sizeof buf, "%s requires a scalar-output tape; got %zu outputs", caller, t->host.outs.size());
    return fail(ECH_ERR_OTHER, buf);
  }
  if (n == 0) {
    return fail(ECH_ERR_OTHER, std::string(caller) + " requires a non-empty x (a zero-input tape has no " + quantity +
                                   "); zero-sized GPU buffers would panic");
  }
  if (n != t->host.ni) return fail(ECH_ERR_INVALID_ARG, "x length must match the tape's num_inputs");
  return ECH_OK;
}

// Taylor order K (default 3) over npoints*S units, then the per-point
// reduction of scale*c_kk (default 2*c2).
// dir_mode: 0 dirs per unit, 1 shared [S][n], 2 device Rademacher, 3 basis e_s.
// reduce: 0 Welford in the sample type (the reference's), 1 Welford in FP64,
// 2 FP32 compensated sums (FP32 samples, no control term).
// comp_jets: FP32 jets with compensated linear chains.
template <class T>
static ech_status stde_run(ech_ctx* ctx, ech_tape* t, const T* d_x, bool x_bcast, uint64_t npoints, uint32_t S,
                           const T* d_dirs, int dir_mode, uint64_t seed, int reduce, const T* d_cv, double trace,
                           int control, ech_estimator_result* d_res, T* d_c0_out, T* d_c2_out, int K = 3,
                           int kk = 2, double scale = 2.0, const T* d_wmul = nullptr, bool comp_jets = false) {
  const uint64_t units = npoints * S;
  CU(ctx->stde_tmp.ensure(units * (uint64_t)K * sizeof(T)));
  SweepIO io;
  io.x = d_x;
  io.x_bcast = x_bcast ? 1 : 0;
  io.v = d_dirs;
  io.out = ctx->stde_tmp.p;
  io.S = S;
  io.dir_mode = dir_mode;
  io.seed = seed;
  io.compensated = (comp_jets && sizeof(T) == 4) ? 1 : 0;
  CHECK(enqueue(ctx, t, 4, K, units, io, ctx->stream));
  const T* c0 = (const T*)ctx->stde_tmp.p;
  const T* c2 = c0 + (uint64_t)kk * units;
  if (d_res) {
    if (reduce == 2 && sizeof(T) == 4 && !control)
      CU(launch_stde_reduce_comp(c0, c2, scale, npoints, S, d_wmul, d_res, ctx->stream));
    else
      CU(launch_stde_reduce_t(sizeof(T) == 8, reduce != 0, c0, c2, scale, npoints, S, d_cv, trace, control, d_wmul,
                              d_res, ctx->stream));
  }
  if (d_c0_out) CU(cudaMemcpyAsync(d_c0_out, c0, units * sizeof(T), cudaMemcpyDeviceToDevice, ctx->stream));
  if (d_c2_out) CU(cudaMemcpyAsync(d_c2_out, c2, units * sizeof(T), cudaMemcpyDeviceToDevice, ctx->stream));
  return ECH_OK;
}

ECH_API ech_status ech_laplacian_gpu_f32(ech_ctx* ctx, const ech_tape* tc, const float* x, size_t n,
                                         const float* dirs, uint32_t S, ech_estimator_result* out) {
  CHECK(common_checks(ctx, tc, false));
  ech_tape* t = const_cast<ech_tape*>(tc);
  CHECK(stde_checks(t, n, "laplacian_gpu", "Laplacian"));
  if (S == 0) return fail(ECH_ERR_OTHER, "no directions provided");
  if (!x || !dirs || !out) return fail(ECH_ERR_INVALID_ARG, "null buffer");
  std::lock_guard<std::mutex> lk(ctx->mu);
  CU(cudaSetDevice(ctx->device));
  CU(ctx->io_in.ensure(n * sizeof(float)));
  CU(ctx->io_in2.ensure((size_t)S * n * sizeof(float)));
  CU(ctx->io_out3.ensure(sizeof(ech_estimator_result)));
  CU(cudaMemcpyAsync(ctx->io_in.p, x, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaMemcpyAsync(ctx->io_in2.p, dirs, (size_t)S * n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  CHECK(stde_run<float>(ctx, t, (const float*)ctx->io_in.p, true, 1, S, (const float*)ctx->io_in2.p, 0, 0, false,
                        nullptr, 0.0, 0, (ech_estimator_result*)ctx->io_out3.p, nullptr, nullptr));
  CU(cudaMemcpyAsync(out, ctx->io_out3.p, sizeof(ech_estimator_result), cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  return check_err_word(ctx);
}

ECH_API ech_status ech_hessian_diagonal_gpu_f32(ech_ctx* ctx, const ech_tape* tc, const float* x, size_t n,
                                                float* value, float* diag) {
  CHECK(common_checks(ctx, tc, false));
  ech_tape* t = const_cast<ech_tape*>(tc);
  CHECK(stde_checks(t, n, "hessian_diagonal_gpu", "Hessian diagonal"));
  if (!x || !value || !diag) return fail(ECH_ERR_INVALID_ARG, "null buffer");
  std::lock_guard<std::mutex> lk(ctx->mu);
  CU(cudaSetDevice(ctx->device));
  CU(ctx->io_in.ensure(n * sizeof(float)));
  CU(ctx->io_out.ensure(n * sizeof(float)));
  CU(ctx->io_out2.ensure(n * sizeof(float)));
  CU(cudaMemcpyAsync(ctx->io_in.p, x, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  CHECK(stde_run<float>(ctx, t, (const float*)ctx->io_in.p, true, 1, (uint32_t)n, nullptr, 3, 0, false, nullptr, 0.0,
                        0, nullptr, (float*)ctx->io_out.p, (float*)ctx->io_out2.p));
  std::vector<float> c0(n), c2(n);
  CU(cudaMemcpyAsync(c0.data(), ctx->io_out.p, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaMemcpyAsync(c2.data(), ctx->io_out2.p, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  CHECK(check_err_word(ctx));
  *value = c0[0];
  for (size_t j = 0; j < n; ++j) diag[j] = 2.0f * c2[j];
  return ECH_OK;
}

ECH_API ech_status ech_laplacian_with_control_gpu_f32(ech_ctx* ctx, const ech_tape* tc, const float* x, size_t n,
                                                      const float* dirs, uint32_t S, const float* control,
                                                      ech_estimator_result* out) {
  CHECK(common_checks(ctx, tc, false));
  ech_tape* t = const_cast<ech_tape*>(tc);
  CHECK(stde_checks(t, n, "laplacian_with_control_gpu", "Laplacian"));
  if (S == 0) return fail(ECH_ERR_OTHER, "no directions provided");
  if (!x || !dirs || !control || !out) return fail(ECH_ERR_INVALID_ARG, "null buffer");
  std::lock_guard<std::mutex> lk(ctx->mu);
  CU(cudaSetDevice(ctx->device));
  float trace = 0.0f;
  for (size_t j = 0; j < n; ++j) trace = trace + control[j];
  CU(ctx->io_in.ensure(n * sizeof(float)));
  CU(ctx->io_in2.ensure((size_t)S * n * sizeof(float)));
  CU(ctx->io_out.ensure(n * sizeof(float) + S * sizeof(float)));
  CU(ctx->io_out3.ensure(sizeof(ech_estimator_result)));
  float* d_diag = (float*)ctx->io_out.p;
  float* d_cv = d_diag + n;
  CU(cudaMemcpyAsync(ctx->io_in.p, x, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaMemcpyAsync(ctx->io_in2.p, dirs, (size_t)S * n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaMemcpyAsync(d_diag, control, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  CU(launch_control_term(false, ctx->io_in2.p, d_diag, S, (uint32_t)n, d_cv, ctx->stream));
  CHECK(stde_run<float>(ctx, t, (const float*)ctx->io_in.p, true, 1, S, (const float*)ctx->io_in2.p, 0, 0, false,
                        d_cv, (double)trace, 1, (ech_estimator_result*)ctx->io_out3.p, nullptr, nullptr));
  CU(cudaMemcpyAsync(out, ctx->io_out3.p, sizeof(ech_estimator_result), cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  return check_err_word(ctx);
}

// Reduction of the FP32 batch STDE calls: FP64 Welford unless the context
// asks for FP32 (compensated or plain) sample means.  FP64 samples always
// reduce in FP64.
static int batch_reduce(const ech_ctx* ctx) {
  if (ctx->fp32_mode & ECH_FP32_COMPENSATED_MEANS) return 2;
  if (ctx->fp32_mode & ECH_FP32_PLAIN_MEANS) return 0;
  return 1;
}

template <class T>
static ech_status do_laplacian_batch(ech_ctx* ctx, const ech_tape* tc, const T* xs, size_t n_xs, uint32_t B,
                                     const T* dirs, size_t n_dirs, uint32_t S, int dir_mode, uint64_t seed,
                                     ech_estimator_result* res) {
  CHECK(common_checks(ctx, tc, sizeof(T) == 8));
  ech_tape* t = const_cast<ech_tape*>(tc);
  CHECK(stde_checks(t, t->host.ni, "laplacian_batch", "Laplacian"));
  CHECK(batch_args(t, B));
  if (S == 0) return fail(ECH_ERR_OTHER, "no directions provided");
  const uint64_t n = t->host.ni;
  CHECK(len_check(n_xs, (uint64_t)B * n, "xs"));
  if (dir_mode == 0) CHECK(len_check(n_dirs, (uint64_t)B * S * n, "directions"));
  else if (dir_mode == 1) CHECK(len_check(n_dirs, (uint64_t)S * n, "directions"));
  else if (dir_mode != 2) return fail(ECH_ERR_INVALID_ARG, "dir_mode must be 0, 1 or 2");
  if (!xs || !res || (dir_mode != 2 && !dirs)) return fail(ECH_ERR_INVALID_ARG, "null buffer");
  std::lock_guard<std::mutex> lk(ctx->mu);
  CU(cudaSetDevice(ctx->device));
  CU(ctx->io_in.ensure(n_xs * sizeof(T)));
  CU(ctx->io_out3.ensure((size_t)B * sizeof(ech_estimator_result)));
  CU(cudaMemcpyAsync(ctx->io_in.p, xs, n_xs * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
  const T* d_dirs = nullptr;
  if (dir_mode != 2) {
    CU(ctx->io_in2.ensure(n_dirs * sizeof(T)));
    CU(cudaMemcpyAsync(ctx->io_in2.p, dirs, n_dirs * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
    d_dirs = (const T*)ctx->io_in2.p;
  }
  CHECK(stde_run<T>(ctx, t, (const T*)ctx->io_in.p, false, B, S, d_dirs, dir_mode, seed, batch_reduce(ctx), nullptr,
                    0.0, 0, (ech_estimator_result*)ctx->io_out3.p, nullptr, nullptr, 3, 2, 2.0, nullptr,
                    (ctx->fp32_mode & ECH_FP32_COMPENSATED_JETS) != 0));
  CU(cudaMemcpyAsync(res, ctx->io_out3.p, (size_t)B * sizeof(ech_estimator_result), cudaMemcpyDeviceToHost,
                     ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  return check_err_word(ctx);
}

ECH_API ech_status ech_laplacian_batch_device(ech_ctx* ctx, const ech_tape* tc, int f64, const void* xs, uint32_t B,
                                              const void* dirs, uint32_t S, int dir_mode, uint64_t seed,
                                              ech_estimator_result* results, void* stream) {
  CHECK(common_checks(ctx, tc, f64 != 0));
  ech_tape* t = const_cast<ech_tape*>(tc);
  CHECK(stde_checks(t, t->host.ni, "laplacian_batch", "Laplacian"));
  CHECK(batch_args(t, B));
  if (S == 0) return fail(ECH_ERR_OTHER, "no directions provided");
  if (dir_mode < 0 || dir_mode > 2) return fail(ECH_ERR_INVALID_ARG, "dir_mode must be 0, 1 or 2");
  if (!xs || !results || (dir_mode != 2 && !dirs)) return fail(ECH_ERR_INVALID_ARG, "null buffer");
  std::lock_guard<std::mutex> lk(ctx->mu);
  CU(cudaSetDevice(ctx->device));
  cudaStream_t saved = ctx->stream;
  ctx->stream = stream ? (cudaStream_t)stream : ctx->stream;  // stde_run enqueues on the context's stream
  ech_status s;
  if (f64)
    s = stde_run<double>(ctx, t, (const double*)xs, false, B, S, (const double*)dirs, dir_mode, seed, 1, nullptr,
                         0.0, 0, results, nullptr, nullptr);
  else
    s = stde_run<float>(ctx, t, (const float*)xs, false, B, S, (const float*)dirs, dir_mode, seed, batch_reduce(ctx),
                        nullptr, 0.0, 0, results, nullptr, nullptr, 3, 2, 2.0, nullptr,
                        (ctx->fp32_mode & ECH_FP32_COMPENSATED_JETS) != 0);
  ctx->stream = saved;
  return s;
}

// Exact Hessian diagonals of many points: order-3 jets along every basis
// direction (dir_mode 3), diag[b][j] = 2 * c2.
ECH_API ech_status ech_hessian_diagonal_batch_device(ech_ctx* ctx, const ech_tape* tc, int f64, const void* xs,
                                                     uint32_t B, void* diag, void* stream) {
  CHECK(common_checks(ctx, tc, f64 != 0));
  ech_tape* t = const_cast<ech_tape*>(tc);
  CHECK(stde_checks(t, t->host.ni, "hessian_diagonal_batch", "Hessian diagonal"));
  CHECK(batch_args(t, B));
  if (!xs || !diag) return fail(ECH_ERR_INVALID_ARG, "null buffer");
  std::lock_guard<std::mutex> lk(ctx->mu);
  CU(cudaSetDevice(ctx->device));
  cudaStream_t saved = ctx->stream;
  ctx->stream = stream ? (cudaStream_t)stream : ctx->stream;
  const uint32_t n = t->host.ni;
  ech_status s;
  if (f64)
    s = stde_run<double>(ctx, t, (const double*)xs, false, B, n, nullptr, 3, 0, true, nullptr, 0.0, 0, nullptr,
                         nullptr, (double*)diag);
  else
    s = stde_run<float>(ctx, t, (const float*)xs, false, B, n, nullptr, 3, 0, true, nullptr, 0.0, 0, nullptr,
                        nullptr, (float*)diag);
  if (s == ECH_OK) {
    cudaError_t e = launch_scale(f64 != 0, diag, 2.0, (size_t)B * n, ctx->stream);
    if (e != cudaSuccess) s = cuda_fail(e, "scale");
  }
  ctx->stream = saved;
  return s;
}

// Sparse STDE trace estimator over many points: per point S coordinates drawn
// from `probs` [B][n] (fp32 rows, e.g. the learned proposal) or uniformly
// (probs == NULL), one order-3 jet along each sampled e_j, samples 2*c2 / p_j,
// FP64 Welford per point.  The estimate is unbiased for sum_j H_jj.
ECH_API ech_status ech_sparse_trace_batch_device(ech_ctx* ctx, const ech_tape* tc, int f64, const void* xs,
                                                 uint32_t B, const float* probs, uint32_t S, uint64_t seed,
                                                 ech_estimator_result* results, void* stream) {
  CHECK(common_checks(ctx, tc, f64 != 0));
  ech_tape* t = const_cast<ech_tape*>(tc);
  CHECK(stde_checks(t, t->host.ni, "sparse_trace_batch", "trace"));
  CHECK(batch_args(t, B));
  if (S == 0) return fail(ECH_ERR_OTHER, "sampled_indices must not be empty");
  if (!xs || !results) return fail(ECH_ERR_INVALID_ARG, "null buffer");
  std::lock_guard<std::mutex> lk(ctx->mu);
  CU(cudaSetDevice(ctx->device));
  const uint64_t units = (uint64_t)B * S;
  const size_t vb = f64 ? 8 : 4;
  CU(ctx->io_in2.ensure(units * (sizeof(uint32_t) + vb) + 256));
  uint32_t* d_idx = (uint32_t*)ctx->io_in2.p;
  void* d_w = (unsigned char*)ctx->io_in2.p + ((units * sizeof(uint32_t) + 255) & ~(uint64_t)255);
  cudaStream_t saved = ctx->stream;
  ctx->stream = stream ? (cudaStream_t)stream : ctx->stream;
  ech_status s = ECH_OK;
  cudaError_t e = launch_sample_coords(f64 != 0, probs, t->host.ni, B, S, seed, d_idx, d_w, ctx->stream);
  if (e != cudaSuccess) s = cuda_fail(e, "coordinate sampling");
  if (s == ECH_OK) {
    if (f64)
      s = stde_run<double>(ctx, t, (const double*)xs, false, B, S, (const double*)(const void*)d_idx, 4, seed, true,
                           nullptr, 0.0, 0, results, nullptr, nullptr, 3, 2, 2.0, (const double*)d_w);
    else
      s = stde_run<float>(ctx, t, (const float*)xs, false, B, S, (const float*)(const void*)d_idx, 4, seed, true,
                          nullptr, 0.0, 0, results, nullptr, nullptr, 3, 2, 2.0, (const float*)d_w);
  }
  ctx->stream = saved;
  return s;
}

ECH_API ech_status ech_laplacian_batch_f32(ech_ctx* ctx, const ech_tape* t, const float* xs, size_t n_xs, uint32_t B,
                                           const float* dirs, size_t n_dirs, uint32_t S, int dir_mode, uint64_t seed,
                                           ech_estimator_result* res) {
  return do_laplacian_batch<float>(ctx, t, xs, n_xs, B, dirs, n_dirs, S, dir_mode, seed, res);
}
ECH_API ech_status ech_laplacian_batch_f64(ech_ctx* ctx, const ech_tape* t, const double* xs, size_t n_xs,
                                           uint32_t B, const double* dirs, size_t n_dirs, uint32_t S, int dir_mode,
                                           uint64_t seed, ech_estimator_result* res) {
  return do_laplacian_batch<double>(ctx, t, xs, n_xs, B, dirs, n_dirs, S, dir_mode, seed, res);
}

// The k range of the k-th order diagonals: the reference's checks
// (higher_order.rs:56 and the factorial-exactness limits at :13-22), then the
// engine's own: jets are instantiated up to order 9, so k <= 8.
static ech_status kth_order_range(uint32_t k, bool f32) {
  if (k < 2) return fail(ECH_ERR_OTHER, "k must be >= 2 (use gradient for k=1)");
  if (k > 18) return fail(ECH_ERR_OTHER, "k must be <= 18 (k! is exact in f64 only up to 18!; 19! exceeds 2^53)");
  if (k > 12 && f32)
    return fail(ECH_ERR_OTHER,
                "k must be <= 12 for f32 (one order of margin: f32 k! exactness first degrades at 14!; use f64)");
  if (k + 1 > 9) {
    char buf[96];
    snprintf(buf, sizeof buf, "unsupported Taylor order %u, must be 1..=9", k + 1);
    return fail(ECH_ERR_OTHER, buf);
  }
  return ECH_OK;
}

// diagonal_kth_order_stochastic (src/stde/higher_order.rs:173-227): one jet of
// order k+1 along e_j per sampled coordinate j, samples k! * c_k, Welford in
// the sample type, then the n / |J| rescaling of the estimate, variance and SE.
template <class T>
static ech_status do_diag_kth(ech_ctx* ctx, const ech_tape* tc, const T* x, size_t n, uint32_t k,
                              const uint32_t* idx, size_t n_idx, ech_estimator_result* out) {
  CHECK(common_checks(ctx, tc, sizeof(T) == 8));
  ech_tape* t = const_cast<ech_tape*>(tc);
  CHECK(stde_checks(t, n, "diagonal_kth_order_stochastic", "diagonal"));
  if (n_idx == 0) return fail(ECH_ERR_OTHER, "sampled_indices must not be empty");
  CHECK(kth_order_range(k, sizeof(T) == 4));
  if (!x || !idx || !out) return fail(ECH_ERR_INVALID_ARG, "null buffer");
  for (size_t s = 0; s < n_idx; ++s) {
    if (idx[s] >= n) {
      char buf[96];
      snprintf(buf, sizeof buf, "sampled index %u out of bounds (n=%zu)", idx[s], n);
      return fail(ECH_ERR_OTHER, buf);
    }
  }
  std::vector<T> dirs(n_idx * n, T(0));
  for (size_t s = 0; s < n_idx; ++s) dirs[s * n + idx[s]] = T(1);
  T kfact = T(1);
  for (uint32_t i = 2; i <= k; ++i) kfact = kfact * (T)i;
  std::lock_guard<std::mutex> lk(ctx->mu);
  CU(cudaSetDevice(ctx->device));
  CU(ctx->io_in.ensure(n * sizeof(T)));
  CU(ctx->io_in2.ensure(dirs.size() * sizeof(T)));
  CU(ctx->io_out3.ensure(sizeof(ech_estimator_result)));
  CU(cudaMemcpyAsync(ctx->io_in.p, x, n * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaMemcpyAsync(ctx->io_in2.p, dirs.data(), dirs.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
  CHECK(stde_run<T>(ctx, t, (const T*)ctx->io_in.p, true, 1, (uint32_t)n_idx, (const T*)ctx->io_in2.p, 1, 0, false,
                    nullptr, 0.0, 0, (ech_estimator_result*)ctx->io_out3.p, nullptr, nullptr, (int)k + 1, (int)k,
                    (double)kfact));
  ech_estimator_result r;
  CU(cudaMemcpyAsync(&r, ctx->io_out3.p, sizeof r, cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  CHECK(check_err_word(ctx));
  const T nf = (T)n;
  r.estimate = (double)((T)r.estimate * nf);
  r.sample_variance = (double)((T)r.sample_variance * nf * nf);
  r.standard_error = (double)((T)r.standard_error * nf);
  *out = r;
  return ECH_OK;
}

ECH_API ech_status ech_diagonal_kth_order_stochastic_f32(ech_ctx* ctx, const ech_tape* t, const float* x, size_t n,
                                                         uint32_t k, const uint32_t* sampled_indices,
                                                         size_t n_indices, ech_estimator_result* out) {
  return do_diag_kth<float>(ctx, t, x, n, k, sampled_indices, n_indices, out);
}
ECH_API ech_status ech_diagonal_kth_order_stochastic_f64(ech_ctx* ctx, const ech_tape* t, const double* x, size_t n,
                                                         uint32_t k, const uint32_t* sampled_indices,
                                                         size_t n_indices, ech_estimator_result* out) {
  return do_diag_kth<double>(ctx, t, x, n, k, sampled_indices, n_indices, out);
}

// diagonal_kth_order (src/stde/higher_order.rs:40-95): diag[j] = k! * c_k of the
// order-(k+1) jet along e_j, all n coordinates in one launch (basis directions
// drawn in the kernel); value = c0.  A zero-input tape returns its recorded
// output value and no diagonal, as the reference does.
template <class T>
static ech_status do_diag_kth_exact(ech_ctx* ctx, const ech_tape* tc, const T* x, size_t n, uint32_t k, T* value,
                                    T* diag) {
  CHECK(common_checks(ctx, tc, sizeof(T) == 8));
  ech_tape* t = const_cast<ech_tape*>(tc);
  if (t->host.outs.size() != 1) {
    char buf[160];
    snprintf(buf, sizeof buf, "diagonal_kth_order requires a scalar-output tape; got %zu outputs", t->host.outs.size());
    return fail(ECH_ERR_OTHER, buf);
  }
  CHECK(kth_order_range(k, sizeof(T) == 4));
  if (!value) return fail(ECH_ERR_INVALID_ARG, "null buffer");
  if (n != t->host.ni) return fail(ECH_ERR_INVALID_ARG, "x length must match the tape's num_inputs");
  if (n == 0) {
    *value = (T)t->host.vals[t->host.out_index];
    return ECH_OK;
  }
  if (!x || !diag) return fail(ECH_ERR_INVALID_ARG, "null buffer");
  T kfact = T(1);
  for (uint32_t i = 2; i <= k; ++i) kfact = kfact * (T)i;
  std::lock_guard<std::mutex> lk(ctx->mu);
  CU(cudaSetDevice(ctx->device));
  CU(ctx->io_in.ensure(n * sizeof(T)));
  CU(ctx->io_out.ensure(n * sizeof(T)));
  CU(ctx->io_out2.ensure(n * sizeof(T)));
  CU(cudaMemcpyAsync(ctx->io_in.p, x, n * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
  CHECK(stde_run<T>(ctx, t, (const T*)ctx->io_in.p, true, 1, (uint32_t)n, nullptr, 3, 0, false, nullptr, 0.0, 0,
                    nullptr, (T*)ctx->io_out.p, (T*)ctx->io_out2.p, (int)k + 1, (int)k));
  std::vector<T> c0(n), ck(n);
  CU(cudaMemcpyAsync(c0.data(), ctx->io_out.p, n * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaMemcpyAsync(ck.data(), ctx->io_out2.p, n * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  CHECK(check_err_word(ctx));
  *value = c0[n - 1];
  for (size_t j = 0; j < n; ++j) diag[j] = kfact * ck[j];
  return ECH_OK;
}

ECH_API ech_status ech_diagonal_kth_order_f32(ech_ctx* ctx, const ech_tape* t, const float* x, size_t n, uint32_t k,
                                              float* value, float* diag) {
  return do_diag_kth_exact<float>(ctx, t, x, n, k, value, diag);
}
ECH_API ech_status ech_diagonal_kth_order_f64(ech_ctx* ctx, const ech_tape* t, const double* x, size_t n,
                                              uint32_t k, double* value, double* diag) {
  return do_diag_kth_exact<double>(ctx, t, x, n, k, value, diag);
}

// stde_sparse (src/stde/sparse.rs:37-78) over the sampling distribution of a
// homogeneous differential operator (SparseSamplingDistribution,
// src/diffop.rs:896-1045), for many points: unit (b, s) runs one jet of order
// jet_order + 1 seeded per entry (input var gets coefficient `slot` =
// input_coeff, every input c0 = x), and sample = sign * Z * prefactor *
// c_{output_coeff_index} enters the point's Welford accumulator in order.
// The entry tables are the distribution's, flattened: entry e's seeds are
// [entry_offsets[e], entry_offsets[e+1]) of vars / slots / input_coeffs.
template <class T>
static ech_status do_stde_sparse(ech_ctx* ctx, const ech_tape* tc, const T* xs, size_t n_xs, uint32_t B,
                                 uint32_t n_entries, const uint32_t* off, const uint32_t* vars, const uint32_t* slots,
                                 const T* coeffs, const uint32_t* kout, const T* pref, const T* sign, T z,
                                 const uint64_t* idx, uint32_t S, ech_estimator_result* results) {
  CHECK(common_checks(ctx, tc, sizeof(T) == 8));
  ech_tape* t = const_cast<ech_tape*>(tc);
  const uint32_t n = t->host.ni;
  CHECK(stde_checks(t, n, "stde_sparse", "derivatives"));
  CHECK(batch_args(t, B));
  if (S == 0) return fail(ECH_ERR_OTHER, "sampled_indices must not be empty");
  if (n_entries == 0) return fail(ECH_ERR_OTHER, "the distribution has no entries");
  if (!xs || !off || !kout || !pref || !sign || !idx || !results) return fail(ECH_ERR_INVALID_ARG, "null buffer");
  if (n_xs != (size_t)B * n) return fail(ECH_ERR_INVALID_ARG, "xs length must be batch_size * num_inputs");
  const uint32_t n_items = off[n_entries];
  if (n_items && (!vars || !slots || !coeffs)) return fail(ECH_ERR_INVALID_ARG, "null buffer");
  uint32_t kmax = 0;
  for (uint32_t e = 0; e < n_entries; ++e) {
    if (off[e] > off[e + 1]) return fail(ECH_ERR_INVALID_ARG, "entry_offsets must be nondecreasing");
    kmax = std::max(kmax, kout[e]);
  }
  const uint32_t K = kmax + 1;  // jet order = dist.jet_order() + 1
  if (K > 9) {
    char buf[128];
    snprintf(buf, sizeof buf, "jet order %u exceeds the GPU jets (at most 9: output coefficient index <= 8)", K);
    return fail(ECH_ERR_OTHER, buf);
  }
  std::vector<SlotSeed> items(std::max<uint32_t>(n_items, 1));
  for (uint32_t q = 0; q < n_items; ++q) {
    if (vars[q] >= n) return fail(ECH_ERR_INVALID_ARG, "seed variable out of range");
    items[q] = SlotSeed{vars[q], slots[q], (double)coeffs[q]};
  }
  const uint64_t units = (uint64_t)B * S;
  std::vector<uint32_t> ent(units);
  for (uint64_t u = 0; u < units; ++u) {
    if (idx[u] >= n_entries) {
      char buf[128];
      snprintf(buf, sizeof buf, "sampled index %llu out of bounds (%u entries)", (unsigned long long)idx[u], n_entries);
      return fail(ECH_ERR_OTHER, buf);
    }
    ent[u] = (uint32_t)idx[u];
  }
  std::lock_guard<std::mutex> lk(ctx->mu);
  CU(cudaSetDevice(ctx->device));
  // io_in: xs | io_in2: unit entries, entry offsets, seeds, kout, prefactor, sign
  auto r256 = [](uint64_t b) { return (b + 255) & ~(uint64_t)255; };
  const uint64_t b_ent = r256(units * 4), b_off = r256((n_entries + 1) * 4ull), b_it = r256(items.size() * 16ull),
                 b_k = r256(n_entries * 4ull), b_t = r256(n_entries * (uint64_t)sizeof(T));
  CU(ctx->io_in.ensure((size_t)n_xs * sizeof(T)));
  CU(ctx->io_in2.ensure(b_ent + b_off + b_it + b_k + 2 * b_t));
  CU(ctx->io_out3.ensure(B * sizeof(ech_estimator_result)));
  unsigned char* base = (unsigned char*)ctx->io_in2.p;
  uint32_t* d_ent = (uint32_t*)base;
  uint32_t* d_off = (uint32_t*)(base + b_ent);
  SlotSeed* d_it = (SlotSeed*)(base + b_ent + b_off);
  uint32_t* d_k = (uint32_t*)(base + b_ent + b_off + b_it);
  T* d_pref = (T*)(base + b_ent + b_off + b_it + b_k);
  T* d_sign = (T*)(base + b_ent + b_off + b_it + b_k + b_t);
  cudaStream_t st = ctx->stream;
  CU(cudaMemcpyAsync(ctx->io_in.p, xs, n_xs * sizeof(T), cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(d_ent, ent.data(), units * 4, cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(d_off, off, (n_entries + 1) * 4ull, cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(d_it, items.data(), items.size() * 16ull, cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(d_k, kout, n_entries * 4ull, cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(d_pref, pref, n_entries * sizeof(T), cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(d_sign, sign, n_entries * sizeof(T), cudaMemcpyHostToDevice, st));
  CU(ctx->stde_tmp.ensure(units * (uint64_t)K * sizeof(T)));
  SweepIO io;
  io.x = ctx->io_in.p;
  io.v = d_ent;
  io.out = ctx->stde_tmp.p;
  io.S = S;
  io.dir_mode = 5;
  io.seed_off = d_off;
  io.seed_items = d_it;
  CHECK(enqueue(ctx, t, 4, (int)K, units, io, st));
  CU(launch_stde_sparse_reduce(sizeof(T) == 8, ctx->stde_tmp.p, units, d_ent, d_k, d_pref, d_sign, (double)z, B, S,
                               ctx->io_out3.p, st));
  CU(cudaMemcpyAsync(results, ctx->io_out3.p, B * sizeof(ech_estimator_result), cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  return check_err_word(ctx);
}

ECH_API ech_status ech_stde_sparse_batch_f32(ech_ctx* ctx, const ech_tape* t, const float* xs, size_t n_xs, uint32_t B,
                                             uint32_t n_entries, const uint32_t* entry_offsets, const uint32_t* vars,
                                             const uint32_t* slots, const float* input_coeffs,
                                             const uint32_t* output_coeff_index, const float* extraction_prefactor,
                                             const float* sign, float normalization, const uint64_t* sampled_indices,
                                             uint32_t n_samples, ech_estimator_result* results) {
  return do_stde_sparse<float>(ctx, t, xs, n_xs, B, n_entries, entry_offsets, vars, slots, input_coeffs,
                               output_coeff_index, extraction_prefactor, sign, normalization, sampled_indices,
                               n_samples, results);
}
ECH_API ech_status ech_stde_sparse_batch_f64(ech_ctx* ctx, const ech_tape* t, const double* xs, size_t n_xs,
                                             uint32_t B, uint32_t n_entries, const uint32_t* entry_offsets,
                                             const uint32_t* vars, const uint32_t* slots, const double* input_coeffs,
                                             const uint32_t* output_coeff_index, const double* extraction_prefactor,
                                             const double* sign, double normalization,
                                             const uint64_t* sampled_indices, uint32_t n_samples,
                                             ech_estimator_result* results) {
  return do_stde_sparse<double>(ctx, t, xs, n_xs, B, n_entries, entry_offsets, vars, slots, input_coeffs,
                                output_coeff_index, extraction_prefactor, sign, normalization, sampled_indices,
                                n_samples, results);
}

// ── estimators built on order-3 jets along host-built directions ──
// (src/stde/laplacian.rs:252-344, src/stde/pde.rs:11-330).  The jets run on the
// GPU; the direction algebra (mat-vecs, projections, Gram-Schmidt) and the
// statistics follow the reference's host code, in the sample type and order.

// Welford's update as WelfordAccumulator (src/stde/types.rs:44-113), host side.
template <class T>
struct HostWelford {
  T mean = T(0), m2 = T(0);
  uint64_t count = 0;
  void update(T s) {
    if (!std::isfinite(s)) return;
    count += 1;
    const T k = (T)count;
    const T d = s - mean;
    mean = mean + d / k;
    const T d2 = s - mean;
    m2 = m2 + d * d2;
  }
  void finalize(T* est, T* var, T* se) const {
    if (count == 0) { *est = std::numeric_limits<T>::quiet_NaN(); *var = T(0); *se = T(0); return; }
    if (count == 1) { *est = mean; *var = T(0); *se = T(0); return; }
    const T v = std::max(m2 / ((T)count - T(1)), T(0));
    *est = mean;
    *var = v;
    *se = std::sqrt(v / (T)count);
  }
};

// c0 and c2 of order-3 jets of the scalar-output tape along S host directions
// [S][n] at one point x.
template <class T>
static ech_status jets_along(ech_ctx* ctx, ech_tape* t, const T* x, size_t n, const T* dirs, uint32_t S,
                             std::vector<T>& c0, std::vector<T>& c2, int kk = 2) {
  c0.assign(S, T(0));
  c2.assign(S, T(0));
  if (S == 0) return ECH_OK;
  std::lock_guard<std::mutex> lk(ctx->mu);
  CU(cudaSetDevice(ctx->device));
  CU(ctx->io_in.ensure(n * sizeof(T)));
  CU(ctx->io_in2.ensure((size_t)S * n * sizeof(T)));
  CU(ctx->io_out.ensure((size_t)S * sizeof(T)));
  CU(ctx->io_out2.ensure((size_t)S * sizeof(T)));
  CU(cudaMemcpyAsync(ctx->io_in.p, x, n * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaMemcpyAsync(ctx->io_in2.p, dirs, (size_t)S * n * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
  CHECK(stde_run<T>(ctx, t, (const T*)ctx->io_in.p, true, 1, S, (const T*)ctx->io_in2.p, 1, 0, false, nullptr, 0.0,
                    0, nullptr, (T*)ctx->io_out.p, (T*)ctx->io_out2.p, 3, kk));
  CU(cudaMemcpyAsync(c0.data(), ctx->io_out.p, (size_t)S * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaMemcpyAsync(c2.data(), ctx->io_out2.p, (size_t)S * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  return check_err_word(ctx);
}

template <class T>
static T fold_dot(const T* a, const T* b, size_t n) {
  T acc = T(0);
  for (size_t i = 0; i < n; ++i) acc = acc + a[i] * b[i];
  return acc;
}

static void put_result(ech_estimator_result* out, double value, double est, double var, double se, uint64_t n) {
  out->value = value;
  out->estimate = est;
  out->sample_variance = var;
  out->standard_error = se;
  out->num_samples = n;
}

// laplacian_hutchpp (src/stde/laplacian.rs:252-344)
template <class T>
static ech_status do_hutchpp(ech_ctx* ctx, const ech_tape* tc, const T* x, size_t n, const T* sketch, uint32_t k,
                             const T* stoch, uint32_t m, ech_estimator_result* out) {
  CHECK(common_checks(ctx, tc, sizeof(T) == 8));
  ech_tape* t = const_cast<ech_tape*>(tc);
  CHECK(stde_checks(t, n, "laplacian_hutchpp", "Laplacian"));
  if (k == 0) return fail(ECH_ERR_OTHER, "sketch_directions must not be empty");
  if (m == 0) return fail(ECH_ERR_OTHER, "stochastic_directions must not be empty");
  if (!x || !sketch || !stoch || !out) return fail(ECH_ERR_INVALID_ARG, "null buffer");
  // 1. sketch: H s for every sketch direction (one HVP batch at one x)
  std::vector<T> grads((size_t)k * n), hs((size_t)k * n);
  CHECK(do_hvp<T>(ctx, t, x, n, false, sketch, (size_t)k * n, k, grads.data(), grads.size(), hs.data(), hs.size()));
  // 2. modified Gram-Schmidt with the reference's drop rule (norm < sqrt(eps))
  const T eps = std::sqrt(std::numeric_limits<T>::epsilon());
  std::vector<std::vector<T>> cols(k);
  for (uint32_t j = 0; j < k; ++j) cols[j].assign(hs.begin() + (size_t)j * n, hs.begin() + (size_t)(j + 1) * n);
  size_t rank = 0, i = 0;
  while (i < cols.size()) {
    for (size_t j = 0; j < rank; ++j) {
      const T dot = fold_dot(cols[j].data(), cols[i].data(), n);
      for (size_t e = 0; e < n; ++e) cols[i][e] = cols[i][e] - dot * cols[j][e];
    }
    T nsq = T(0);
    for (size_t e = 0; e < n; ++e) nsq = nsq + cols[i][e] * cols[i][e];
    const T norm = std::sqrt(nsq);
    if (norm < eps) {
      std::swap(cols[i], cols.back());
      cols.pop_back();
    } else {
      const T inv = T(1) / norm;
      for (size_t e = 0; e < n; ++e) cols[i][e] = cols[i][e] * inv;
      if (i != rank) std::swap(cols[i], cols[rank]);
      ++rank;
      ++i;
    }
  }
  // 3. exact trace on span(Q)
  std::vector<T> qd(rank * n), c0, c2;
  for (size_t j = 0; j < rank; ++j) std::copy(cols[j].begin(), cols[j].end(), qd.begin() + j * n);
  CHECK(jets_along<T>(ctx, t, x, n, qd.data(), (uint32_t)rank, c0, c2));
  T value = T(0), exact = T(0);
  for (size_t j = 0; j < rank; ++j) {
    value = c0[j];
    exact = exact + T(2) * c2[j];
  }
  // 4. Hutchinson on the residual: g' = g - Q (Q^T g), dots with the original g
  std::vector<T> proj((size_t)m * n);
  for (uint32_t g = 0; g < m; ++g) {
    const T* gv = stoch + (size_t)g * n;
    T* pv = proj.data() + (size_t)g * n;
    std::copy(gv, gv + n, pv);
    for (size_t j = 0; j < rank; ++j) {
      const T dot = fold_dot(cols[j].data(), gv, n);
      for (size_t e = 0; e < n; ++e) pv[e] = pv[e] - dot * cols[j][e];
    }
  }
  CHECK(jets_along<T>(ctx, t, x, n, proj.data(), m, c0, c2));
  HostWelford<T> acc;
  for (uint32_t g = 0; g < m; ++g) {
    value = c0[g];
    acc.update(T(2) * c2[g]);
  }
  T mean, var, se;
  acc.finalize(&mean, &var, &se);
  put_result(out, (double)value, (double)(exact + mean), (double)var, (double)se, acc.count);
  return ECH_OK;
}

// parabolic_diffusion (src/stde/pde.rs:128-162): (value, 1/2 sum_i 2 c2 along sigma columns)
template <class T>
static ech_status do_parabolic(ech_ctx* ctx, const ech_tape* tc, const T* x, size_t n, const T* sigma, uint32_t d,
                               T* value, T* estimate) {
  CHECK(common_checks(ctx, tc, sizeof(T) == 8));
  ech_tape* t = const_cast<ech_tape*>(tc);
  CHECK(stde_checks(t, n, "parabolic_diffusion", "diffusion term"));
  if (d == 0) return fail(ECH_ERR_OTHER, "sigma_columns must not be empty");
  if (!x || !sigma || !value || !estimate) return fail(ECH_ERR_INVALID_ARG, "null buffer");
  std::vector<T> c0, c2;
  CHECK(jets_along<T>(ctx, t, x, n, sigma, d, c0, c2));
  T v = T(0), sum = T(0);
  for (uint32_t i = 0; i < d; ++i) {
    v = c0[i];
    sum = sum + T(2) * c2[i];
  }
  *value = v;
  *estimate = T(0.5) * sum;
  return ECH_OK;
}

// parabolic_diffusion_stochastic (src/stde/pde.rs:164-240)
template <class T>
static ech_status do_parabolic_stoch(ech_ctx* ctx, const ech_tape* tc, const T* x, size_t n, const T* sigma,
                                     uint32_t d, const uint32_t* idx, uint32_t m, ech_estimator_result* out) {
  CHECK(common_checks(ctx, tc, sizeof(T) == 8));
  ech_tape* t = const_cast<ech_tape*>(tc);
  CHECK(stde_checks(t, n, "parabolic_diffusion_stochastic", "diffusion term"));
  if (m == 0) return fail(ECH_ERR_OTHER, "sampled_indices must not be empty");
  if (!x || !sigma || !idx || !out) return fail(ECH_ERR_INVALID_ARG, "null buffer");
  std::vector<T> dirs((size_t)m * n);
  for (uint32_t s = 0; s < m; ++s) {
    if (idx[s] >= d) {
      char buf[96];
      snprintf(buf, sizeof buf, "sampled index %u out of bounds (d=%u)", idx[s], d);
      return fail(ECH_ERR_OTHER, buf);
    }
    std::copy(sigma + (size_t)idx[s] * n, sigma + (size_t)(idx[s] + 1) * n, dirs.begin() + (size_t)s * n);
  }
  std::vector<T> c0, c2;
  CHECK(jets_along<T>(ctx, t, x, n, dirs.data(), m, c0, c2));
  HostWelford<T> acc;
  T value = T(0);
  for (uint32_t s = 0; s < m; ++s) {
    value = c0[s];
    acc.update(T(2) * c2[s]);
  }
  T mean, var, se;
  acc.finalize(&mean, &var, &se);
  const T scale = (T)d * T(0.5);
  put_result(out, (double)value, (double)(mean * scale), (double)(var * scale * scale), (double)(se * scale),
             acc.count);
  return ECH_OK;
}

// stde::estimate / estimate_weighted (src/stde/pipeline.rs:20-142) with the
// reference's two estimators (src/stde/estimator.rs): Laplacian samples 2 c2,
// GradientSquaredNorm c1^2.  The order-3 jets along the S host directions run on
// the GPU; the statistics follow the reference's host loop in the sample type:
// Welford without weights, West's weighted update with them (zero weights are
// skipped but counted, non-finite samples skipped and not counted, standard error
// over the effective n = (sum w)^2 / sum w^2).
template <class T>
static ech_status do_estimate(ech_ctx* ctx, const ech_tape* tc, const T* x, size_t n, int estimator, const T* dirs,
                              uint32_t S, const T* weights, ech_estimator_result* out) {
  CHECK(common_checks(ctx, tc, sizeof(T) == 8));
  ech_tape* t = const_cast<ech_tape*>(tc);
  CHECK(stde_checks(t, n, "estimate", "estimator"));
  if (estimator != 0 && estimator != 1) return fail(ECH_ERR_INVALID_ARG, "estimator must be 0 (Laplacian) or 1 (GradientSquaredNorm)");
  if (S == 0) return fail(ECH_ERR_OTHER, "directions must not be empty");
  if (!x || !dirs || !out) return fail(ECH_ERR_INVALID_ARG, "null buffer");
  if (weights)
    for (uint32_t s = 0; s < S; ++s)
      if (!(weights[s] >= T(0))) return fail(ECH_ERR_OTHER, "estimate_weighted: weights must be non-negative and non-NaN");
  std::vector<T> c0, ck;
  CHECK(jets_along<T>(ctx, t, x, n, dirs, S, c0, ck, estimator == 0 ? 2 : 1));
  auto sample = [&](uint32_t s) { return estimator == 0 ? T(2) * ck[s] : ck[s] * ck[s]; };
  T value = T(0);
  if (!weights) {
    HostWelford<T> acc;
    for (uint32_t s = 0; s < S; ++s) {
      value = c0[s];
      acc.update(sample(s));
    }
    T mean, var, se;
    acc.finalize(&mean, &var, &se);
    put_result(out, (double)value, (double)mean, (double)var, (double)se, acc.count);
    return ECH_OK;
  }
  T w_sum = T(0), w_sum2 = T(0), mean = T(0), m2 = T(0);
  uint64_t skips = 0;
  for (uint32_t s = 0; s < S; ++s) {
    value = c0[s];
    const T w = weights[s];
    if (w == T(0)) continue;
    const T v = sample(s);
    if (!std::isfinite(v)) {
      ++skips;
      continue;
    }
    w_sum = w_sum + w;
    w_sum2 = w_sum2 + w * w;
    const T d = v - mean;
    mean = mean + (w / w_sum) * d;
    const T d2 = v - mean;
    m2 = m2 + w * d * d2;
  }
  const T denom = w_sum > T(0) ? w_sum - w_sum2 / w_sum : T(0);
  T var = T(0), se = T(0);
  if (S > 1 && denom > T(0)) {
    var = std::max(m2 / denom, T(0));
    const T n_eff = w_sum * w_sum / w_sum2;
    se = std::sqrt(var / n_eff);
  }
  const T est = (w_sum > T(0) || skips == 0) ? mean : std::numeric_limits<T>::quiet_NaN();
  put_result(out, (double)value, (double)est, (double)var, (double)se, (uint64_t)S - skips);
  return ECH_OK;
}

ECH_API ech_status ech_estimate_f32(ech_ctx* ctx, const ech_tape* t, const float* x, size_t n, int estimator,
                                    const float* dirs, uint32_t S, const float* weights, ech_estimator_result* out) {
  return do_estimate<float>(ctx, t, x, n, estimator, dirs, S, weights, out);
}
ECH_API ech_status ech_estimate_f64(ech_ctx* ctx, const ech_tape* t, const double* x, size_t n, int estimator,
                                    const double* dirs, uint32_t S, const double* weights, ech_estimator_result* out) {
  return do_estimate<double>(ctx, t, x, n, estimator, dirs, S, weights, out);
}

// dense_stde_2nd (src/stde/pde.rs:242-296): samples 2 c2 along v = L z, L lower
// triangular (row-major n x n, entries above the diagonal ignored).
template <class T>
static ech_status do_dense_stde(ech_ctx* ctx, const ech_tape* tc, const T* x, size_t n, const T* L, const T* z,
                                uint32_t m, ech_estimator_result* out) {
  CHECK(common_checks(ctx, tc, sizeof(T) == 8));
  ech_tape* t = const_cast<ech_tape*>(tc);
  CHECK(stde_checks(t, n, "dense_stde_2nd", "operator"));
  if (m == 0) return fail(ECH_ERR_OTHER, "z_vectors must not be empty");
  if (!x || !L || !z || !out) return fail(ECH_ERR_INVALID_ARG, "null buffer");
  std::vector<T> dirs((size_t)m * n);
  for (uint32_t s = 0; s < m; ++s) {
    const T* zs = z + (size_t)s * n;
    for (size_t i = 0; i < n; ++i) {
      T sum = T(0);
      for (size_t j = 0; j <= i; ++j) sum = sum + L[i * n + j] * zs[j];
      dirs[(size_t)s * n + i] = sum;
    }
  }
  std::vector<T> c0, c2;
  CHECK(jets_along<T>(ctx, t, x, n, dirs.data(), m, c0, c2));
  HostWelford<T> acc;
  T value = T(0);
  for (uint32_t s = 0; s < m; ++s) {
    value = c0[s];
    acc.update(T(2) * c2[s]);
  }
  T mean, var, se;
  acc.finalize(&mean, &var, &se);
  put_result(out, (double)value, (double)mean, (double)var, (double)se, acc.count);
  return ECH_OK;
}

// divergence (src/stde/pde.rs:52-106): samples v^T J v from JVPs of a square tape.
template <class T>
static ech_status do_divergence(ech_ctx* ctx, const ech_tape* tc, const T* x, size_t n, const T* dirs, uint32_t m,
                                T* values, ech_estimator_result* out) {
  CHECK(common_checks(ctx, tc, sizeof(T) == 8));
  const ech_tape* t = tc;
  const size_t no = t->host.outs.size();
  if (no != t->host.ni) {
    char buf[128];
    snprintf(buf, sizeof buf, "divergence requires num_outputs (%zu) == num_inputs (%u)", no, t->host.ni);
    return fail(ECH_ERR_OTHER, buf);
  }
  if (m == 0) return fail(ECH_ERR_OTHER, "directions must not be empty");
  if (n != t->host.ni) return fail(ECH_ERR_INVALID_ARG, "x length must match the tape's num_inputs");
  if (!x || !dirs || !out) return fail(ECH_ERR_INVALID_ARG, "null buffer");
  std::vector<T> xs((size_t)m * n), vals((size_t)m * no), tans((size_t)m * no);
  for (uint32_t s = 0; s < m; ++s) std::copy(x, x + n, xs.begin() + (size_t)s * n);
  CHECK(do_tangent<T>(ctx, tc, xs.data(), xs.size(), dirs, (size_t)m * n, m, vals.data(), tans.data(), vals.size()));
  HostWelford<T> acc;
  for (uint32_t s = 0; s < m; ++s) acc.update(fold_dot(dirs + (size_t)s * n, tans.data() + (size_t)s * no, n));
  if (values) std::copy(vals.begin(), vals.begin() + no, values);
  T mean, var, se;
  acc.finalize(&mean, &var, &se);
  put_result(out, 0.0, (double)mean, (double)var, (double)se, acc.count);
  return ECH_OK;
}

#define ECH_STDE_OPS(SUF, T)                                                                                       \
  ECH_API ech_status ech_laplacian_hutchpp_##SUF(ech_ctx* c, const ech_tape* t, const T* x, size_t n,             \
                                                 const T* sketch, uint32_t k, const T* stoch, uint32_t m,          \
                                                 ech_estimator_result* out) {                                      \
    return do_hutchpp<T>(c, t, x, n, sketch, k, stoch, m, out);                                                    \
  }                                                                                                                \
  ECH_API ech_status ech_parabolic_diffusion_##SUF(ech_ctx* c, const ech_tape* t, const T* x, size_t n,           \
                                                   const T* sigma, uint32_t d, T* value, T* estimate) {            \
    return do_parabolic<T>(c, t, x, n, sigma, d, value, estimate);                                                 \
  }                                                                                                                \
  ECH_API ech_status ech_parabolic_diffusion_stochastic_##SUF(ech_ctx* c, const ech_tape* t, const T* x, size_t n, \
                                                              const T* sigma, uint32_t d, const uint32_t* idx,     \
                                                              uint32_t m, ech_estimator_result* out) {             \
    return do_parabolic_stoch<T>(c, t, x, n, sigma, d, idx, m, out);                                               \
  }                                                                                                                \
  ECH_API ech_status ech_dense_stde_2nd_##SUF(ech_ctx* c, const ech_tape* t, const T* x, size_t n, const T* L,    \
                                              const T* z, uint32_t m, ech_estimator_result* out) {                 \
    return do_dense_stde<T>(c, t, x, n, L, z, m, out);                                                             \
  }                                                                                                                \
  ECH_API ech_status ech_divergence_##SUF(ech_ctx* c, const ech_tape* t, const T* x, size_t n, const T* dirs,      \
                                          uint32_t m, T* values, ech_estimator_result* out) {                      \
    return do_divergence<T>(c, t, x, n, dirs, m, values, out);                                                     \
  }
ECH_STDE_OPS(f32, float)
ECH_STDE_OPS(f64, double)
#undef ECH_STDE_OPS

// ── checkpointed gradients of iterated maps (src/checkpoint.rs:67-126, 548-722) ──
// x_{t+1} = step(x_t) for t < T, objective loss(x_T); gradient w.r.t. x_0 for a
// batch of starting points.  Only the states at the checkpoint positions are
// kept; every reverse segment recomputes its states from its checkpoint, then
// pulls the adjoint back through each step with a vector-Jacobian product.
// The VJP of a step is the gradient of s = sum_j w_j step(x)_j over the inputs
// (x, w): the step tape with n extra inputs w and the weighted sum appended.

static HostTape vjp_tape_of(const HostTape& h) {
  const uint32_t n = h.ni, shift = n;
  HostTape v;
  v.ni = 2 * n;
  auto map = [&](uint32_t s) { return s < n ? s : s + shift; };
  for (uint32_t i = 0; i < n; ++i) {
    v.op.push_back(OP_INPUT); v.a0.push_back(kUnused); v.a1.push_back(kUnused); v.vals.push_back(h.vals[i]);
  }
  for (uint32_t i = 0; i < n; ++i) {
    v.op.push_back(OP_INPUT); v.a0.push_back(kUnused); v.a1.push_back(kUnused); v.vals.push_back(0.0);
  }
  for (uint32_t i = n; i < h.nv; ++i) {
    const uint32_t o = h.op[i];
    v.op.push_back(o);
    v.vals.push_back(h.vals[i]);
    if (o == OP_CONST) { v.a0.push_back(kUnused); v.a1.push_back(kUnused); continue; }
    v.a0.push_back(map(h.a0[i]));
    v.a1.push_back((o == OP_POWI || h.a1[i] == kUnused) ? h.a1[i] : map(h.a1[i]));
  }
  uint32_t s = kUnused;
  for (uint32_t j = 0; j < (uint32_t)h.outs.size(); ++j) {
    const uint32_t m = (uint32_t)v.op.size();
    v.op.push_back(OP_MUL); v.a0.push_back(n + j); v.a1.push_back(map(h.outs[j])); v.vals.push_back(0.0);
    if (s == kUnused) {
      s = m;
    } else {
      v.op.push_back(OP_ADD); v.a0.push_back(s); v.a1.push_back(m); v.vals.push_back(0.0);
      s = (uint32_t)v.op.size() - 1;
    }
  }
  v.nv = (uint32_t)v.op.size();
  v.out_index = s;
  v.outs.assign(1, s);
  return v;
}

// Stored positions, spread evenly: j * N / (C + 1) for j = 1..C; every step
// when C >= N (spread_positions / revolve_schedule, src/checkpoint.rs:673-722).
static std::vector<uint32_t> spread_positions(uint32_t steps, uint32_t ckpts) {
  std::vector<uint32_t> p;
  if (ckpts >= steps) {
    for (uint32_t s = 1; s < steps; ++s) p.push_back(s);
    return p;
  }
  for (uint32_t j = 1; j <= ckpts; ++j) p.push_back((uint32_t)((uint64_t)j * steps / (ckpts + 1)));
  std::sort(p.begin(), p.end());
  p.erase(std::unique(p.begin(), p.end()), p.end());
  return p;
}

template <class T>
static ech_status do_grad_ckpt(ech_ctx* ctx, const ech_tape* sc, const ech_tape* lc, const T* x0, uint32_t B,
                               uint32_t steps, uint32_t ckpts, T* grads) {
  const bool f64 = sizeof(T) == 8;
  CHECK(common_checks(ctx, sc, f64));
  CHECK(common_checks(ctx, lc, f64));
  ech_tape* st = const_cast<ech_tape*>(sc);
  ech_tape* lt = const_cast<ech_tape*>(lc);
  const uint32_t n = st->host.ni;
  if (st->host.outs.size() != n) {
    char buf[128];
    snprintf(buf, sizeof buf, "step must preserve dimension: expected %u, got %zu", n, st->host.outs.size());
    return fail(ECH_ERR_OTHER, buf);
  }
  if (lt->host.ni != n || lt->host.outs.size() != 1)
    return fail(ECH_ERR_OTHER, "loss must map the state dimension to one output");
  CHECK(batch_args(st, B));
  if (!x0 || !grads) return fail(ECH_ERR_INVALID_ARG, "null buffer");
  {
    std::lock_guard<std::mutex> lk(st->mu);
    if (!st->vjp) {
      st->vjp.reset(new ech_tape());
      st->vjp->ctx = ctx;
      st->vjp->f64 = st->f64;
      st->vjp->host = vjp_tape_of(st->host);
    }
  }
  ech_tape* vt = st->vjp.get();
  const size_t row = (size_t)B * n * sizeof(T);
  std::lock_guard<std::mutex> lk(ctx->mu);
  CU(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  if (steps == 0) {  // gradient of loss(x0)
    SweepIO io;
    io.x = x0;
    CU(ctx->io_out.ensure((size_t)B * sizeof(T)));
    io.out = ctx->io_out.p;
    io.out2 = grads;
    CHECK(enqueue(ctx, lt, 1, 0, B, io, s));
    CU(cudaStreamSynchronize(s));
    return check_err_word(ctx);
  }
  const uint32_t c = std::min(std::max(ckpts, 1u), steps);
  std::vector<uint32_t> pos = spread_positions(steps, c);
  std::vector<uint32_t> seg_start(1, 0);
  seg_start.insert(seg_start.end(), pos.begin(), pos.end());
  uint32_t max_seg = 0;
  for (size_t k = 0; k < seg_start.size(); ++k) {
    const uint32_t e = k + 1 < seg_start.size() ? seg_start[k + 1] : steps;
    max_seg = std::max(max_seg, e - seg_start[k]);
  }
  // buffers: checkpoints, one segment of states, (x | w) rows and their gradient, adjoint
  DevBuf ck, states, xw, gw, adj, lossv;
  CU(ck.ensure(row * seg_start.size()));
  CU(states.ensure(row * (size_t)(max_seg + 1)));
  CU(xw.ensure(2 * row));
  CU(gw.ensure(2 * row));
  CU(adj.ensure(row));
  CU(lossv.ensure((size_t)B * sizeof(T)));
  auto ckp = [&](size_t k) { return (unsigned char*)ck.p + k * row; };
  auto stp = [&](size_t k) { return (unsigned char*)states.p + k * row; };
  auto fwd = [&](const void* in, void* out) -> ech_status {
    SweepIO io;
    io.x = in;
    io.out = out;
    return enqueue(ctx, st, 0, 0, B, io, s);
  };
  // forward pass: keep the state at every checkpoint position
  CU(cudaMemcpyAsync(ckp(0), x0, row, cudaMemcpyDeviceToDevice, s));
  size_t next_ck = 1;
  const void* cur = x0;
  for (uint32_t t = 0; t < steps; ++t) {
    void* out = stp(t & 1);
    CHECK(fwd(cur, out));
    if (next_ck < seg_start.size() && seg_start[next_ck] == t + 1) {
      CU(cudaMemcpyAsync(ckp(next_ck), out, row, cudaMemcpyDeviceToDevice, s));
      ++next_ck;
    }
    cur = out;
  }
  // the objective's gradient at the final state seeds the adjoint
  {
    SweepIO io;
    io.x = cur;
    io.out = lossv.p;
    io.out2 = adj.p;
    CHECK(enqueue(ctx, lt, 1, 0, B, io, s));
  }
  for (size_t seg = seg_start.size(); seg-- > 0;) {
    const uint32_t a = seg_start[seg];
    const uint32_t e = seg + 1 < seg_start.size() ? seg_start[seg + 1] : steps;
    const uint32_t len = e - a;
    CU(cudaMemcpyAsync(stp(0), ckp(seg), row, cudaMemcpyDeviceToDevice, s));
    for (uint32_t i = 0; i < len; ++i) CHECK(fwd(stp(i), stp(i + 1)));
    for (uint32_t i = len; i-- > 0;) {
      // (x | w) rows = [states[i] | adjoint]
      CU(cudaMemcpy2DAsync(xw.p, 2 * n * sizeof(T), stp(i), n * sizeof(T), n * sizeof(T), B,
                           cudaMemcpyDeviceToDevice, s));
      CU(cudaMemcpy2DAsync((unsigned char*)xw.p + n * sizeof(T), 2 * n * sizeof(T), adj.p, n * sizeof(T),
                           n * sizeof(T), B, cudaMemcpyDeviceToDevice, s));
      SweepIO io;
      io.x = xw.p;
      io.out = lossv.p;
      io.out2 = gw.p;
      CHECK(enqueue(ctx, vt, 1, 0, B, io, s));
      CU(cudaMemcpy2DAsync(adj.p, n * sizeof(T), gw.p, 2 * n * sizeof(T), n * sizeof(T), B,
                           cudaMemcpyDeviceToDevice, s));
    }
  }
  CU(cudaMemcpyAsync(grads, adj.p, row, cudaMemcpyDeviceToDevice, s));
  CU(cudaStreamSynchronize(s));
  return check_err_word(ctx);
}

ECH_API ech_status ech_grad_checkpointed_device(ech_ctx* ctx, const ech_tape* step, const ech_tape* loss, int f64,
                                                const void* x0, uint32_t B, uint32_t num_steps,
                                                uint32_t num_checkpoints, void* grads) {
  if (!ctx || !step || !loss) return fail(ECH_ERR_INVALID_ARG, "null argument");
  return f64 ? do_grad_ckpt<double>(ctx, step, loss, (const double*)x0, B, num_steps, num_checkpoints,
                                    (double*)grads)
             : do_grad_ckpt<float>(ctx, step, loss, (const float*)x0, B, num_steps, num_checkpoints, (float*)grads);
}

extern "C" {

ECH_API ech_status ech_ctx_synchronize(ech_ctx* ctx) {
  if (!ctx) return fail(ECH_ERR_INVALID_ARG, "ctx is null");
  CU(cudaSetDevice(ctx->device));
  CU(cudaStreamSynchronize(ctx->stream));
  CU(cudaDeviceSynchronize());
  return check_err_word(ctx);
}


// Host-only: lowers a tape without a device and copies the programs out, so the
// lowering can be checked on machines without a GPU.  counts[0..5] receive the
// instruction, reverse-instruction and pool counts, shared registers, far slots
// and trajectory slots; arrays are filled up to their capacities.
ECH_API ech_status ech_plan_dump(const uint32_t* op, const uint32_t* a0, const uint32_t* a1, const double* values,
                                 uint32_t nv, uint32_t ni, uint32_t output_index, const uint32_t* outs,
                                 uint32_t nouts, int kind, uint32_t cap, void* fwd, size_t fwd_cap, void* rev,
                                 size_t rev_cap, double* pool, size_t pool_cap, void* terms, size_t terms_cap,
                                 void* gathers, size_t gathers_cap, void* dense, size_t dense_cap,
                                 uint32_t dense_max, uint64_t* counts) {
  if (!op || !a0 || !a1 || !values || !counts) return fail(ECH_ERR_INVALID_ARG, "null argument");
  std::string m = validate_bytecode_tape(op, a0, a1, nv, ni, output_index, outs, nouts, false);
  if (!m.empty()) return fail(ECH_ERR_OTHER, "invalid bytecode tape: " + m);
  if (kind < 0 || kind > 5) return fail(ECH_ERR_INVALID_ARG, "kind must be 0..5");
  HostTape h;
  h.nv = nv;
  h.ni = ni;
  h.out_index = output_index;
  h.op.assign(op, op + nv);
  h.a0.assign(a0, a0 + nv);
  h.a1.assign(a1, a1 + nv);
  h.vals.assign(values, values + nv);
  if (nouts == 0) h.outs.assign(1, output_index);
  else h.outs.assign(outs, outs + nouts);
  Plan p = build_plan(h, kind_of(kind), cap, dense_max);
  counts[8] = p.dense.size();
  if (dense) memcpy(dense, p.dense.data(), std::min(dense_cap, p.dense.size()) * sizeof(PDenseOut));
  counts[0] = p.fwd.size();
  counts[1] = p.rev.size();
  counts[2] = p.pool.size();
  counts[3] = p.smem_regs;
  counts[4] = p.far_slots;
  counts[5] = p.traj_slots;
  counts[6] = p.terms.size();
  counts[7] = p.gathers.size();
  if (gathers) memcpy(gathers, p.gathers.data(), std::min(gathers_cap, p.gathers.size()) * sizeof(GRec));
  if (terms) memcpy(terms, p.terms.data(), std::min(terms_cap, p.terms.size()) * sizeof(PTerm));
  if (fwd) memcpy(fwd, p.fwd.data(), std::min(fwd_cap, p.fwd.size()) * sizeof(Ins));
  if (rev) memcpy(rev, p.rev.data(), std::min(rev_cap, p.rev.size()) * sizeof(RIns));
  if (pool) memcpy(pool, p.pool.data(), std::min(pool_cap, p.pool.size()) * sizeof(double));
  return ECH_OK;
}

ECH_API ech_status ech_tape_plan_stats(ech_ctx* ctx, const ech_tape* tc, int kind, uint32_t order, int f64,
                                       uint64_t* stats) {
  if (!ctx || !tc || !stats) return fail(ECH_ERR_INVALID_ARG, "null argument");
  if (kind < 0 || kind > 5) return fail(ECH_ERR_INVALID_ARG, "kind must be 0..5");
  (void)f64;
  ech_tape* t = const_cast<ech_tape*>(tc);
  LaunchCfg c = choose_cfg(ctx, t, kind, (int)order);
  Plan p = build_plan(t->host, kind_of(kind), c.cap, dense_group_max((uint32_t)c.vbytes, (uint32_t)c.req.P));
  const PlanStats& s = p.stats;
  uint64_t v[12] = {s.fwd_ops, s.rev_ops, s.max_live_fwd, s.max_live_rev, s.traj_values, s.flops_fwd, s.flops_rev,
                    s.specials_fwd, s.specials_rev, p.smem_regs, p.far_slots, p.fwd.size() + p.rev.size()};
  memcpy(stats, v, sizeof v);
  return ECH_OK;
}

ECH_API ech_status ech_tape_program_stats(ech_ctx* ctx, const ech_tape* tc, int kind, uint32_t order,
                                         uint64_t n_units, uint64_t* stats) {
  if (!ctx || !tc || !stats) return fail(ECH_ERR_INVALID_ARG, "null argument");
  if (kind < 0 || kind > 5) return fail(ECH_ERR_INVALID_ARG, "kind must be 0..5");
  ech_tape* t = const_cast<ech_tape*>(tc);
  const int skind = kind == 5 ? 4 : kind;  // input-direct jets use the jets' shapes
  Shape sh;
  bool tuned = false;
  {
    std::lock_guard<std::mutex> lk(t->mu);
    auto it = t->shapes.find(std::make_tuple(skind, (int)order, size_bucket(n_units)));
    if (it != t->shapes.end()) { sh = it->second; tuned = true; }
  }
  const LaunchCfg c = tuned ? cfg_for(ctx, t, skind, (int)order, sh) : choose_cfg(ctx, t, skind, (int)order);
  std::lock_guard<std::mutex> lk(ctx->mu);
  CU(cudaSetDevice(ctx->device));
  DevPlan* dp = nullptr;
  CHECK(get_plan(t, kind, (int)order, c.cap, c.tile, (uint32_t)c.vbytes, (uint32_t)c.req.P, true, &dp));
  uint64_t v[5] = {dp->n_fwd, dp->n_rev, (uint64_t)dp->host.dense.size(), dp->gather_tiles,
                   (dp->needs_dense() || c.dense_kernel) ? 1u : 0u};
  memcpy(stats, v, sizeof v);
  return ECH_OK;
}

ECH_API ech_status ech_tape_launch_shape(ech_ctx* ctx, const ech_tape* tc, int kind, uint32_t order,
                                        uint64_t n_units, uint64_t* shape) {
  if (!ctx || !tc || !shape) return fail(ECH_ERR_INVALID_ARG, "null argument");
  if (kind < 0 || kind > 4) return fail(ECH_ERR_INVALID_ARG, "kind must be 0..4");
  ech_tape* t = const_cast<ech_tape*>(tc);
  Shape sh;
  uint64_t tuned = 0;
  LaunchCfg c;
  {
    std::lock_guard<std::mutex> lk(t->mu);
    auto it = t->shapes.find(std::make_tuple(kind, (int)order, size_bucket(n_units)));
    if (it != t->shapes.end()) { sh = it->second; tuned = 1; }
  }
  c = tuned ? cfg_for(ctx, t, kind, (int)order, sh) : choose_cfg(ctx, t, kind, (int)order);
  Plan p = build_plan(t->host, kind_of(kind), c.cap, dense_group_max((uint32_t)c.vbytes, (uint32_t)c.req.P));
  uint64_t v[8] = {(uint64_t)c.threads, (uint64_t)c.req.P, tuned ? sh.ctas : 0, c.cap, p.smem_regs, p.far_slots,
                   p.traj_slots, tuned | (tuned && sh.dense_kernel ? 2u : 0u)};
  memcpy(shape, v, sizeof v);
  return ECH_OK;
}

}  // extern "C"

namespace ech {
size_t value_bytes(const LaunchReq& r) {
  const size_t s = r.f64 ? 8 : 4;
  switch (r.vk) {
    case VKind::Plain: return s;
    case VKind::Dual: return 2 * s;
    case VKind::Jet: return (size_t)r.K * s;
  }
  return s;
}
}  // namespace ech

// ───────────────────────────── many tapes, one launch ───────────────────────
// A prepared many-tape gradient + per-point HVP launch over caller-owned device
// buffers (extension; the uneven-batch workload).  Preparation lowers every
// tape for one launch shape, orders the jobs by cost, uploads the job table and
// sizes the scratch; a launch is then a counter reset plus one kernel.
struct ech_multi {
  ech_ctx* ctx = nullptr;  // must outlive the handle
  int device = 0;
  bool f64 = false;
  std::vector<ech_multi_item> items;
  Shape shape;
  LaunchCfg cfg;
  DevBuf jobs, next, scratch;
  uint32_t n_jobs = 0;
  uint32_t total_tiles = 0;
  uint64_t stride = 0;
  int grid = 0;
  bool tuned = false;
};

static ech_status multi_prepare(ech_multi* m, Shape sh) {
  ech_ctx* ctx = m->ctx;
  CU(cudaStreamSynchronize(ctx->stream));  // no earlier launch may still read the job table or scratch
  LaunchCfg c = cfg_for(ctx, m->items[0].tape, 2, 0, sh);
  if (c.cap < 1 || kRingBytes + (size_t)c.tile * c.vbytes > ctx->smem_optin)
    return fail(ECH_ERR_OTHER, "launch shape does not fit shared memory");
  struct J {
    MultiJob job;
    uint64_t cost, tiles;
  };
  std::vector<J> js;
  uint32_t regs = 1;
  uint64_t slots = 0;
  for (const ech_multi_item& it : m->items) {
    if (it.n_points == 0) continue;
    ech_tape* t = const_cast<ech_tape*>(it.tape);
    DevPlan* dp = nullptr;
    CHECK(get_plan(t, 2, 0, c.cap, c.tile, (uint32_t)c.vbytes, (uint32_t)c.req.P, true, &dp));
    const Plan& p = dp->host;
    if (dp->needs_dense() || c.dense_kernel) c.req.dense = true;
    regs = std::max<uint32_t>(regs, p.smem_regs);
    slots = std::max<uint64_t>(slots, (uint64_t)p.far_slots + p.traj_slots);
    J j{};
    KParams& kp = j.job.kp;
    kp.fwd = dp->d_fwd;
    kp.n_fwd = dp->n_fwd;
    kp.rev = dp->d_rev;
    kp.n_rev = dp->n_rev;
    kp.far_slots = p.far_slots;
    kp.traj_slots = p.traj_slots;
    kp.tile = c.tile;
    kp.n_units = it.n_points;
    kp.ni = t->host.ni;
    kp.no = (uint32_t)t->host.outs.size();
    kp.x = it.xs;
    kp.v = it.dirs;
    kp.x_bcast = 0;
    kp.out2 = it.grads;
    kp.out3 = it.hvps;
    kp.err = ctx->d_err;
    j.tiles = (it.n_points + c.tile - 1) / c.tile;
    j.cost = (uint64_t)dp->n_fwd + dp->n_rev;
    js.push_back(j);
  }
  if (js.empty()) return fail(ECH_ERR_OTHER, "batch_size must be non-zero");
  // most expensive tiles first, so the tail of the dynamic schedule is short work
  std::stable_sort(js.begin(), js.end(), [](const J& a, const J& b) { return a.cost > b.cost; });
  uint64_t first = 0;
  std::vector<MultiJob> h(js.size());
  for (size_t k = 0; k < js.size(); ++k) {
    h[k] = js[k].job;
    h[k].kp.smem_regs = regs;
    h[k].first_tile = first;
    first += js[k].tiles;
  }
  if (first >= 0xFFFFFFFFull) return fail(ECH_ERR_OTHER, "too many tiles for one launch");
  c.smem = kRingBytes + (size_t)regs * c.tile * c.vbytes;
  uint64_t stride = slots * c.tile * c.vbytes;
  stride = (stride + 255) & ~(uint64_t)255;
  MultiParams mp{};
  int bps = 0;
  cudaError_t e = launch_multi_hvp(c.req.dense, m->f64, c.req.P, mp, 0, c.threads, c.smem, nullptr, &bps);
  if (e != cudaSuccess) return cuda_fail(e, "occupancy query");
  if (bps <= 0) return fail(ECH_ERR_OTHER, "tape live set does not fit the shared-memory slot file");
  const uint64_t grid = std::min<uint64_t>(first, (uint64_t)bps * ctx->sm_count);
  CU(m->jobs.ensure(h.size() * sizeof(MultiJob)));
  CU(m->next.ensure(sizeof(uint32_t)));
  CU(m->scratch.ensure(std::max<uint64_t>(stride * grid, 256)));
  for (MultiJob& j : h) {
    j.kp.scratch = m->scratch.p;
    j.kp.scratch_stride_bytes = stride;
  }
  CU(cudaMemcpy(m->jobs.p, h.data(), h.size() * sizeof(MultiJob), cudaMemcpyHostToDevice));
  m->shape = sh;
  m->cfg = c;
  m->n_jobs = (uint32_t)h.size();
  m->total_tiles = (uint32_t)first;
  m->stride = stride;
  m->grid = (int)grid;
  return ECH_OK;
}

static ech_status multi_enqueue(ech_multi* m, cudaStream_t st) {
  MultiParams mp{};
  mp.jobs = (const MultiJob*)m->jobs.p;
  mp.n_jobs = m->n_jobs;
  mp.total_tiles = m->total_tiles;
  mp.next_tile = (uint32_t*)m->next.p;
  mp.scratch = m->scratch.p;
  mp.stride = m->stride;
  CU(cudaMemsetAsync(m->next.p, 0, sizeof(uint32_t), st));
  int bps = 0;
  cudaError_t e = launch_multi_hvp(m->cfg.req.dense, m->f64, m->cfg.req.P, mp, m->grid, m->cfg.threads, m->cfg.smem,
                                   st, &bps);
  if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
  return ECH_OK;
}

extern "C" {

ECH_API ech_status ech_multi_create(ech_ctx* ctx, int f64, const ech_multi_item* items, uint32_t n_items,
                                    int autotune, ech_multi** out) {
  if (!ctx || !out || (n_items && !items)) return fail(ECH_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  if (n_items == 0) return fail(ECH_ERR_OTHER, "batch_size must be non-zero");
  uint64_t total_points = 0;
  for (uint32_t k = 0; k < n_items; ++k) {
    const ech_multi_item& it = items[k];
    if (!it.tape) return fail(ECH_ERR_INVALID_ARG, "null tape");
    if (it.tape->ctx != ctx) return fail(ECH_ERR_INVALID_ARG, "tape belongs to another context");
    if (it.tape->f64 != (f64 != 0)) return fail(ECH_ERR_INVALID_ARG, "tape precision does not match the call");
    if (it.tape->host.ni == 0) return fail(ECH_ERR_OTHER, "tape has no inputs");
    if (it.n_points && (!it.xs || !it.dirs || !it.grads || !it.hvps))
      return fail(ECH_ERR_INVALID_ARG, "null device buffer");
    total_points += it.n_points;
  }
  if (total_points == 0) return fail(ECH_ERR_OTHER, "batch_size must be non-zero");
  std::unique_ptr<ech_multi> m(new ech_multi());
  m->ctx = ctx;
  m->device = ctx->device;
  m->f64 = f64 != 0;
  m->items.assign(items, items + n_items);
  std::lock_guard<std::mutex> lk(ctx->mu);
  CU(cudaSetDevice(ctx->device));
  Shape best;
  best.dense_kernel = ctx->ov_dense;
  if (autotune && !ctx->ov_dense) {
    cudaEvent_t e0, e1;
    CU(cudaEventCreate(&e0));
    CU(cudaEventCreate(&e1));
    float best_ms = -1.0f;
    for (const Shape& sh : kShapes) {
      if (sh.threads * sh.P < 128) continue;
      if (multi_prepare(m.get(), sh) != ECH_OK) continue;
      if (multi_enqueue(m.get(), ctx->stream) != ECH_OK) continue;  // warm
      cudaEventRecord(e0, ctx->stream);
      const ech_status s = multi_enqueue(m.get(), ctx->stream);
      cudaEventRecord(e1, ctx->stream);
      if (s != ECH_OK || cudaEventSynchronize(e1) != cudaSuccess) continue;
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (best_ms < 0.0f || ms < best_ms) {
        best_ms = ms;
        best = sh;
      }
    }
    if (best_ms >= 0.0f) {
      // the best shape on the other kernel build (bit-identical results)
      Shape alt = best;
      alt.dense_kernel = 1;
      if (multi_prepare(m.get(), alt) == ECH_OK && multi_enqueue(m.get(), ctx->stream) == ECH_OK) {
        float a_ms = -1.0f;
        for (int r = 0; r < 2; ++r) {
          cudaEventRecord(e0, ctx->stream);
          const ech_status s = multi_enqueue(m.get(), ctx->stream);
          cudaEventRecord(e1, ctx->stream);
          if (s != ECH_OK || cudaEventSynchronize(e1) != cudaSuccess) break;
          float ms = 0.0f;
          cudaEventElapsedTime(&ms, e0, e1);
          a_ms = a_ms < 0.0f ? ms : std::min(a_ms, ms);
        }
        if (a_ms >= 0.0f && a_ms < best_ms) best = alt;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CHECK(check_err_word(ctx));
    if (best_ms < 0.0f) return fail(ECH_ERR_OTHER, "no launch shape fits");
    m->tuned = true;
  }
  CHECK(multi_prepare(m.get(), best));
  *out = m.release();
  return ECH_OK;
}

ECH_API ech_status ech_multi_launch(ech_multi* m, void* stream) {
  if (!m) return fail(ECH_ERR_INVALID_ARG, "null multi");
  std::lock_guard<std::mutex> lk(m->ctx->mu);
  CU(cudaSetDevice(m->ctx->device));
  return multi_enqueue(m, stream ? (cudaStream_t)stream : m->ctx->stream);
}

ECH_API ech_status ech_multi_info(const ech_multi* m, uint64_t* info) {
  if (!m || !info) return fail(ECH_ERR_INVALID_ARG, "null argument");
  uint64_t v[9] = {m->shape.threads, m->shape.P, m->shape.ctas, m->cfg.cap, (uint64_t)m->grid, m->total_tiles,
                   m->n_jobs, m->stride, (m->tuned ? 1u : 0u) | (m->shape.dense_kernel ? 2u : 0u)};
  memcpy(info, v, sizeof v);
  return ECH_OK;
}

ECH_API void ech_multi_destroy(ech_multi* m) {
  if (!m) return;
  // only the device is needed here (its buffers' cudaFree waits for work that uses them)
  cudaSetDevice(m->device);
  delete m;
}

}  // extern "C"

// ───────────────────────────── internal hooks ───────────────────────────────
namespace ech {

ech_status set_error(ech_status st, const std::string& msg) { return fail(st, msg); }

ech_status ctx_basics(ech_ctx* ctx, int* device, cudaStream_t* stream, uint32_t** err) {
  if (!ctx) return fail(ECH_ERR_INVALID_ARG, "ctx is null");
  *device = ctx->device;
  *stream = ctx->stream;
  *err = ctx->d_err;
  return ECH_OK;
}

ech_status prepare_gradient_host(ech_ctx* ctx, const ech_tape* tc, int f64, uint32_t B, HostSweep* out) {
  CHECK(common_checks(ctx, tc, f64 != 0));
  CHECK(batch_args(tc, B));
  ech_tape* t = const_cast<ech_tape*>(tc);
  const LaunchCfg c = choose_cfg(ctx, t, 1, 0);
  const ech_tape::HostProgram* hp = nullptr;
  {
    std::lock_guard<std::mutex> lk(t->mu);
    auto key = std::make_tuple(1, 0, c.cap, c.tile, (uint32_t)c.vbytes, (uint32_t)c.req.P);
    auto it = t->host_programs.find(key);
    if (it == t->host_programs.end()) {
      static std::atomic<uint64_t> next_id{1};
      std::unique_ptr<ech_tape::HostProgram> np(new ech_tape::HostProgram());
      np->id = next_id.fetch_add(1);
      np->plan = build_plan(t->host, Kind::Gradient, c.cap, dense_group_max((uint32_t)c.vbytes, (uint32_t)c.req.P));
      std::string err;
      if (!encode_plan(np->plan, c.tile, (uint32_t)c.vbytes, !t->f64, np->prog, err)) return fail(ECH_ERR_OTHER, err);
      it = t->host_programs.emplace(key, std::move(np)).first;
    }
    hp = it->second.get();
  }
  out->req = c.req;
  out->req.dense = !hp->plan.dense.empty() || hp->prog.gather_tiles > 0 || ctx->ov_dense;
  out->threads = c.threads;
  out->tile = c.tile;
  out->vbytes = c.vbytes;
  out->smem = kRingBytes + (size_t)std::max<uint32_t>(hp->plan.smem_regs, 1) * c.tile * c.vbytes;
  out->plan = &hp->plan;
  out->prog = &hp->prog;
  out->prog_id = hp->id;
  out->device = ctx->device;
  out->sm_count = ctx->sm_count;
  out->ni = t->host.ni;
  out->no = (uint32_t)t->host.outs.size();
  out->d_err = ctx->d_err;
  out->stream = ctx->stream;
  out->mu = &ctx->mu;
  return ECH_OK;
}

}  // namespace ech
