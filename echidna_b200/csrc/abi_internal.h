// Engine-internal hooks shared between abi.cu and entry points that manage
// their own device memory (noalloc.cu).  Not part of the C ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <string>

#include "../../include/echidna_b200.h"
#include "launch.h"
#include "plan.h"

namespace ech {

// Everything a gradient sweep needs except device memory: the launch
// geometry the ordinary entry points would choose, the host-encoded program
// (cached on the tape), and the context's stream, error word and lock.
struct HostSweep {
  LaunchReq req;
  int threads = 0;
  uint32_t tile = 0;
  size_t vbytes = 0;
  size_t smem = 0;             // dynamic shared memory per CTA
  const Plan* plan = nullptr;
  const DevProgram* prog = nullptr;
  uint64_t prog_id = 0;        // process-unique id of `prog` (never reused)
  int device = 0;
  int sm_count = 0;
  uint32_t ni = 0, no = 0;
  uint32_t* d_err = nullptr;   // the context's error word (allocated at context creation)
  cudaStream_t stream = nullptr;
  std::mutex* mu = nullptr;
};

// Argument checks of the gradient entry points, then the host-side plan.
ech_status prepare_gradient_host(ech_ctx* ctx, const ech_tape* t, int f64, uint32_t batch, HostSweep* out);
ech_status set_error(ech_status st, const std::string& msg);
// The context's device, stream and device-side error word.
ech_status ctx_basics(ech_ctx* ctx, int* device, cudaStream_t* stream, uint32_t** err);

}  // namespace ech
