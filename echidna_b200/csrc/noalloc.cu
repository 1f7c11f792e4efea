// Gradient sweep that allocates no device memory:
// ech_gradient_batch_device_noalloc (declared in include/echidna_b200.h).
//
// Every device byte the call needs beyond the caller's own buffers comes from
// one fixed region compiled into this library, `g_noalloc_region` below:
//   [forward program | reverse program | per-CTA slot scratch]
// The two programs (fused-chain terms sit inline in their records) are copied
// into the front of the region on the caller's stream when the region does not
// already hold them: each device remembers the id of the program it last
// received, and a call with the same program skips the copy.  The rest holds
// the per-CTA global slot files and trajectories of the sweep kernel (the same
// kernel the ordinary gradient entry points launch).  The grid is shrunk until
// the CTAs' scratch fits, so batches of any size run; a tape whose program or
// single-CTA scratch does not fit is rejected with ECH_ERR_OUT_OF_MEMORY.
//
// Nothing in the region has to start at zero: every slot is written before it
// is read and each adjoint is initialised by its first contribution.  Kernel
// errors are latched in the context's error word (allocated when the context
// was created) and reported by ech_ctx_synchronize, as for the other
// *_device entry points.
//
// The region's address is looked up once per device and kept for the life of
// the process; a device reset (cudaDeviceReset) invalidates it, so the call
// must not be used on a device after a reset.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <mutex>

#include "abi_internal.h"
#include "interp.cuh"

namespace {

constexpr size_t kNoAllocBytes = 64ull << 20;  // 64 MiB, fixed at build time
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_region[kNoAllocBytes];

std::mutex g_setup_mu;
unsigned char* g_region_ptr[kMaxDevices] = {};
uint64_t g_region_prog[kMaxDevices] = {};  // id of the program the region holds (0: none); under g_setup_mu

size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

// Once per device, with that device current: the region's device address.
ech_status region_for_device(int device, unsigned char** out) {
  if (device < 0 || device >= kMaxDevices) return ech::set_error(ECH_ERR_INVALID_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_region_ptr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_region);
    if (e != cudaSuccess || !p)
      return ech::set_error(ECH_ERR_OTHER, std::string("cudaGetSymbolAddress of the no-alloc region: ") +
                                               cudaGetErrorString(e));
    g_region_ptr[device] = static_cast<unsigned char*>(p);
  }
  *out = g_region_ptr[device];
  return ECH_OK;
}

}  // namespace

extern "C" ECH_API size_t ech_noalloc_region_bytes(void) { return kNoAllocBytes; }

extern "C" ECH_API ech_status ech_gradient_batch_device_noalloc(ech_ctx* ctx, const ech_tape* t, int f64,
                                                                const void* in, uint32_t B, void* out, void* grads,
                                                                void* stream) {
  using namespace ech;
  HostSweep hs;
  ech_status s = prepare_gradient_host(ctx, t, f64, B, &hs);
  if (s != ECH_OK) return s;
  std::lock_guard<std::mutex> lk(*hs.mu);
  cudaError_t e = cudaSetDevice(hs.device);
  if (e != cudaSuccess) return set_error(ECH_ERR_OTHER, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  unsigned char* region = nullptr;
  s = region_for_device(hs.device, &region);
  if (s != ECH_OK) return s;

  const DevProgram& pg = *hs.prog;
  const Plan& p = *hs.plan;
  const size_t b_fwd = round256(std::max<size_t>(pg.fwd.size(), 1) * sizeof(DIns));
  const size_t b_rev = round256(std::max<size_t>(pg.rev.size(), 1) * sizeof(DRIns));
  const size_t b_prog = b_fwd + b_rev;
  const uint64_t slots = (uint64_t)p.far_slots + p.traj_slots;
  const uint64_t stride = round256(slots * hs.tile * hs.vbytes);
  if (b_prog + std::max<uint64_t>(stride, 256) > kNoAllocBytes) {
    char buf[256];
    snprintf(buf, sizeof buf,
             "no-alloc region too small: this tape needs %zu program bytes plus %llu scratch bytes per CTA, "
             "the region holds %zu bytes",
             b_prog, (unsigned long long)stride, kNoAllocBytes);
    return set_error(ECH_ERR_OUT_OF_MEMORY, buf);
  }
  cudaStream_t st = stream ? (cudaStream_t)stream : hs.stream;
  unsigned char* d_fwd = region;
  unsigned char* d_rev = d_fwd + b_fwd;
  unsigned char* d_scratch = d_rev + b_rev;
  const size_t scratch_bytes = kNoAllocBytes - b_prog;

  KParams kp{};
  kp.fwd = reinterpret_cast<const DIns*>(d_fwd);
  kp.n_fwd = (uint32_t)pg.fwd.size();
  kp.rev = reinterpret_cast<const DRIns*>(d_rev);
  kp.n_rev = (uint32_t)pg.rev.size();
  kp.far_slots = p.far_slots;
  kp.traj_slots = p.traj_slots;
  kp.smem_regs = std::max<uint32_t>(p.smem_regs, 1);
  kp.tile = hs.tile;
  kp.n_units = B;
  kp.ni = hs.ni;
  kp.no = hs.no;
  kp.x = in;
  kp.out = out;
  kp.out2 = grads;
  kp.err = hs.d_err;
  kp.scratch = d_scratch;
  kp.scratch_stride_bytes = stride;

  int bps = 0;
  e = launch_sweep(hs.req, kp, 0, hs.threads, hs.smem, st, &bps);
  if (e != cudaSuccess) return set_error(ECH_ERR_OTHER, std::string("occupancy query: ") + cudaGetErrorString(e));
  if (bps <= 0) return set_error(ECH_ERR_OTHER, "tape live set does not fit the shared-memory slot file");
  const uint64_t ntiles = ((uint64_t)B + hs.tile - 1) / hs.tile;
  uint64_t grid = std::min<uint64_t>(ntiles, (uint64_t)bps * hs.sm_count);
  if (stride > 0) grid = std::min<uint64_t>(grid, scratch_bytes / stride);
  if (grid == 0) return ECH_OK;

  std::lock_guard<std::mutex> tag_lk(g_setup_mu);
  if (g_region_prog[hs.device] != hs.prog_id) {
    // the region holds another program (or none): copy this one in, stream-ordered
    g_region_prog[hs.device] = 0;
    if (!pg.fwd.empty())
      e = cudaMemcpyAsync(d_fwd, pg.fwd.data(), pg.fwd.size() * sizeof(DIns), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && !pg.rev.empty())
      e = cudaMemcpyAsync(d_rev, pg.rev.data(), pg.rev.size() * sizeof(DRIns), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return set_error(ECH_ERR_OTHER, std::string("program copy: ") + cudaGetErrorString(e));
    g_region_prog[hs.device] = hs.prog_id;
  }
  e = launch_sweep(hs.req, kp, (int)grid, hs.threads, hs.smem, st, &bps);
  if (e != cudaSuccess) return set_error(ECH_ERR_OTHER, std::string("kernel launch: ") + cudaGetErrorString(e));
  return ECH_OK;
}
