// Host-side lowering of a recorded tape into interpreter programs.
#pragma once
#include <stdint.h>
#include <string>
#include <vector>
#include "ech_types.h"

namespace ech {

// A validated tape in host memory.  `vals` holds the constants image in double
// (f32 tapes widen exactly); `outs` is all_output_indices() after the upload
// fallback (empty output_indices -> [output_index]).
struct HostTape {
  std::vector<uint32_t> op, a0, a1;
  std::vector<double> vals;
  uint32_t nv = 0, ni = 0, out_index = 0;
  std::vector<uint32_t> outs;
};

// TaylorDirect: a Taylor program for launches whose input jets are (x, v, 0, ..)
// with v from a direction source the kernel can evaluate per input (shared host
// directions, device Rademacher, basis vectors): linear-combination terms over
// inputs read the input jet at its source (M_INPUT) instead of a slot.
enum class Kind { Forward, Gradient, Hvp, Jvp, Taylor, TaylorDirect };

struct PlanStats {
  uint64_t fwd_ops = 0;        // tape ops executed per unit in the forward program
  uint64_t rev_ops = 0;        // tape ops executed per unit in the reverse program
  uint64_t max_live_fwd = 0;   // peak live values (forward)
  uint64_t max_live_rev = 0;   // peak live adjoints (reverse)
  uint64_t traj_values = 0;    // values saved for the reverse (T_val)
  uint64_t flops_fwd = 0;      // arithmetic ops per unit (forward)
  uint64_t flops_rev = 0;      // arithmetic ops per unit (reverse)
  uint64_t specials_fwd = 0;   // libm-class calls per unit (forward)
  uint64_t specials_rev = 0;
  uint64_t chains = 0;         // fused chains
  uint64_t chain_ops = 0;      // tape ops absorbed into chains
};

// One term of a fused chain (XI_CHAIN) with its resolved locations.
// Packed layout (48 bytes) so the host-only dump can hand it out as-is.
struct PTerm {
  uint8_t kind, op;     // ChainKind / operand position (see ech_types.h)
  uint16_t flags;       // ChainFlag bits (CF_*_INIT, CF_*_ADJ, CF_*_GLOB)
  uint32_t xs, ys;      // slot ids, kNone when absent
  uint8_t fxm, fym;     // forward modes of x, y
  uint8_t rxm, rym;     // reverse modes of adj(x), adj(y)
  uint32_t fxi, fyi;    // forward register / slot indices
  uint32_t rxi, ryi;    // reverse adjoint register / slot indices
  uint32_t vx, vy;      // trajectory slots of the values x*y terms read
  double c;             // constant of c*x / x*c / c terms
};
static_assert(sizeof(PTerm) == 48, "PTerm must be 48 bytes");

// One record of a reverse gather (XI_GATHER): a target header followed by its
// contributions.  Header: s = the target's adjoint slot id, n = contributions
// that follow, flags CF_X_INIT (first contribution to the target); a
// contribution: s = a chain result whose normalised adjoint is multiplied by c.
// mode / idx: the slot after allocation.
struct GRec {
  uint32_t s;
  uint32_t n;
  uint16_t flags;
  uint8_t mode, pad;
  uint32_t idx;
  double c;
  uint64_t pad2;
};
static_assert(sizeof(GRec) == 32, "GRec must be 32 bytes");

// One output of a dense group (XI_DENSE): a linear-combination chain whose
// terms (tb .. tb+tn in Plan::terms) read the same operands in the same order
// as every other output of the group.  Locations after allocation.
struct PDenseOut {
  uint32_t tb, tn;      // the chain's terms
  uint8_t am, dm;       // modes of acc0 (M_SMEM / M_GLOB / M_IMM) and of the result
  uint16_t pad;
  uint32_t ai, di;      // register / slot indices
  uint32_t save;        // trajectory slot of the result, or kNone
  double a_val;         // acc0 when am == M_IMM
};
static_assert(sizeof(PDenseOut) == 32, "PDenseOut must be 32 bytes");

struct Plan {
  std::vector<PTerm> terms;  // fused-chain terms, shared by both programs
  std::vector<PDenseOut> dense;  // outputs of dense groups (XI_DENSE: a = first, aux = count)
  std::vector<GRec> gathers; // reverse gather records (XI_GATHER: va = first header, aux = targets)
  std::vector<Ins> fwd;
  std::vector<RIns> rev;
  std::vector<double> pool;
  uint32_t smem_regs = 0;      // shared registers used
  uint32_t far_slots = 0;      // global registers (max of both sweeps)
  uint32_t traj_slots = 0;     // trajectory slots
  uint32_t dense_max = 1;      // the dense group limit the plan was built for (also bounds gather tiles)
  PlanStats stats;
};

// Builds the programs for `kind` with at most `smem_cap` shared registers.
// `dense_max` > 1 groups up to that many consecutive linear-combination chains
// over one operand list into one XI_DENSE instruction (1: no groups).
Plan build_plan(const HostTape& t, Kind kind, uint32_t smem_cap, uint32_t dense_max = 1);

// Device encoding of a plan for a launch geometry (`tile` points per CTA,
// `vbytes` bytes per slot value).  Returns false (with `err`) if an offset does
// not fit the 32-bit encoding.
// Chain terms are records of the streams (after their chain instruction), so
// the record counts exceed the plan's instruction counts.
struct DevProgram {
  std::vector<DIns> fwd;
  std::vector<DRIns> rev;
  uint32_t gather_tiles = 0;   // gather tiles in rev (the kernel build with the dense-group executor runs them)
};
// `f32`: the program runs on f32 values (their linear-combination constants are stored rounded).
bool encode_plan(const Plan& p, uint32_t tile, uint32_t vbytes, bool f32, DevProgram& out, std::string& err);

// Validation with the reference's messages.  Empty string = valid.
//   BytecodeTape::validate   (src/bytecode_tape/mod.rs:575-705)
//   GpuTapeData::validate    (src/gpu/mod.rs:397-564)
std::string validate_bytecode_tape(const uint32_t* op, const uint32_t* a0, const uint32_t* a1, uint32_t nv,
                                   uint32_t ni, uint32_t output_index, const uint32_t* outs, uint32_t nouts,
                                   bool has_custom_ops);
std::string validate_gpu_tape_data(const uint32_t* op, const uint32_t* a0, const uint32_t* a1, uint32_t n_op,
                                   uint32_t n_a0, uint32_t n_a1, uint32_t n_const, uint32_t num_ops,
                                   uint32_t num_inputs, uint32_t num_variables, uint32_t output_index,
                                   const uint32_t* outs, uint32_t nouts);

bool is_binary(uint32_t op);

}  // namespace ech
