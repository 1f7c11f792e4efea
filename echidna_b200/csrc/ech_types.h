// Shared host/device definitions: opcode numbering, the lowered instruction
// formats the interpreter kernels execute, and launch parameter blocks.
//
// Opcode discriminants are the reference's (src/opcode.rs:21-130, pinned in
// src/gpu/mod.rs:427-472).  Everything else here is this engine's own format.
#pragma once
#include <stdint.h>

namespace ech {

enum OpCode : uint8_t {
  OP_INPUT = 0, OP_CONST, OP_ADD, OP_SUB, OP_MUL, OP_DIV, OP_REM, OP_POWF, OP_ATAN2, OP_HYPOT, OP_MAX, OP_MIN,
  OP_NEG, OP_RECIP, OP_SQRT, OP_CBRT, OP_POWI, OP_EXP, OP_EXP2, OP_EXPM1, OP_LN, OP_LOG2, OP_LOG10, OP_LN1P,
  OP_SIN, OP_COS, OP_TAN, OP_ASIN, OP_ACOS, OP_ATAN, OP_SINH, OP_COSH, OP_TANH, OP_ASINH, OP_ACOSH, OP_ATANH,
  OP_ABS, OP_SIGNUM, OP_FLOOR, OP_CEIL, OP_ROUND, OP_TRUNC, OP_FRACT, OP_CUSTOM,
  // Engine-internal instructions (never appear in a recorded tape).
  XI_LDIN = 64,   // dst <- input[aux] (and direction seed for tangent kinds)
  XI_STOUT = 65,  // output[aux] <- a
  XI_MOV = 66,    // dst <- a (used to materialise a constant operand)
  XI_SEED = 67,   // reverse: adj(r) <- 1
  XI_STGRAD = 68, // reverse: grad[aux] <- adj(r)   (r mode NONE -> 0)
  XI_CHAIN = 69,  // fused linear chain: dst <- acc0 (+|-) term_1 (+|-) ... ; terms in the chain table
  XI_NORM = 84,   // reverse: adj(r) <- adj(r) passed through a unit Add (the chain's term adjoint)
  XI_GATHER = 85, // reverse: each target adjoint accumulated over its chain contributions, stored once
  XI_DENSE = 86,  // forward: m linear-combination chains over one operand list (a dense layer), one pass
                  // over the operands: a = first output in the plan's dense table, aux = m
};

// One term of a fused chain s_t = s_{t-1} (+|-) term_t.  `kind` says how the
// term is formed, `op` where the running value sits in the Add/Sub:
//   kind: 0 x, 1 c*x (Mul(c, x)), 2 x*c (Mul(x, c)), 3 x*y (Mul(x, y)), 4 c (constant)
//   op:   0 acc+term, 1 term+acc, 2 acc-term, 3 term-acc
// Index form (plan): x, y are value vregs (slot ids); ax/ay the same slots for
// the adjoints; flags carry the reverse's first-contribution marks.
enum ChainKind : uint8_t { CK_X = 0, CK_CX = 1, CK_XC = 2, CK_XY = 3, CK_C = 4 };
enum ChainFlag : uint16_t {
  CF_X_INIT = 1 << 0,   // first reverse contribution to adj(x): start from +0
  CF_Y_INIT = 1 << 1,
  CF_X_GLOB = 1 << 2,   // (device) adj(x) lives in global slots
  CF_Y_GLOB = 1 << 3,
  CF_X_ADJ = 1 << 4,    // adj(x) receives contributions (x is not a constant)
  CF_Y_ADJ = 1 << 5,
};

constexpr uint32_t kUnused = 0xFFFFFFFFu;
constexpr uint32_t kNone = 0xFFFFFFFFu;

// Operand modes.
enum Mode : uint8_t {
  M_SMEM = 0,  // register in the block's shared-memory slot file
  M_GLOB = 1,  // slot in the block's L2-resident global scratch ([slot][point])
  M_IMM = 2,   // constant: Ins::imm (forward) or RIns pool index (reverse)
  M_NONE = 3,
  M_INPUT = 4, // (linear-combination term of a jet program) input `x` read from the launch's
               // primal inputs and direction source, never materialised in a slot
};

// Forward instruction, 32 bytes.
//   dst <- op(a, b); optionally also written to the trajectory slot `save`.
struct alignas(16) Ins {
  uint8_t opc;
  uint8_t ma, mb, md;  // modes of a, b, dst
  uint32_t a, b, d;
  uint32_t save;       // trajectory slot or kNone
  int32_t aux;         // powi exponent / input index / output index
  double imm;          // value of the (single) immediate operand
};
static_assert(sizeof(Ins) == 32, "Ins must be 32 bytes");

// Reverse instruction, 32 bytes.  Processes one tape op in reverse:
//   adj(a) += da * adj(r); adj(b) += db * adj(r)
// with the zero-adjoint skip and the zero-multiplier guard.
enum RFlag : uint16_t {
  RF_R_GLOB = 1 << 0,   // adj(r) lives in global scratch
  RF_A_GLOB = 1 << 1,
  RF_B_GLOB = 1 << 2,
  RF_A_INIT = 1 << 3,   // first contribution to adj(a): start from +0
  RF_B_INIT = 1 << 4,
  RF_VA_IMM = 1 << 5,   // value a is a pool constant
  RF_VB_IMM = 1 << 6,
  RF_HAS_A = 1 << 7,    // contribute to adj(a)
  RF_HAS_B = 1 << 8,
  RF_LC_DISTINCT = 1 << 9,  // D_CHAIN_LC: the terms' adjoint targets are pairwise distinct
};
struct alignas(16) RIns {
  uint8_t opc;
  uint8_t pad;
  uint16_t flags;
  uint32_t r, a, b;     // adjoint locations
  uint32_t va, vb, vr;  // trajectory slots (or pool index when *_IMM), kNone if unused
  int32_t aux;          // powi exponent / gradient index
};
static_assert(sizeof(RIns) == 32, "RIns must be 32 bytes");

// ───────── device encoding (what the kernels execute) ─────────
// The plan above is in register-index form; before upload it is encoded for a
// launch geometry: every register / slot becomes a byte offset from the
// thread's column base (slot * tile * sizeof(value)), and ops whose operands
// are all shared-memory registers or immediates get mode-specialised opcodes.
enum DOp : uint8_t {
  // 2..42: generic tape opcode, operand modes in the instruction
  D_LDIN = 64, D_STOUT = 65, D_MOV = 66, D_SEED = 67, D_STGRAD = 68,
  // forward binary fast forms: a, b in {smem register, immediate}, dst smem
  D_ADD_RR = 72, D_ADD_IR, D_ADD_RI, D_SUB_RR, D_SUB_IR, D_SUB_RI,
  D_MUL_RR, D_MUL_IR, D_MUL_RI, D_DIV_RR, D_DIV_IR, D_DIV_RI,  // .. 83
  D_CHAIN = 69,     // fused linear chain (forward and reverse)
  D_CHAIN_LC = 70,  // fused chain whose terms are all c*x or x*c added to the running value
  D_DENSE = 86,     // forward: XI_DENSE; followed by its DDenseInit, term and DDenseFin records
  D_NORM = 84,      // reverse: XI_NORM
  D_GATHER = 85,    // reverse: XI_GATHER; per target a DRTerm header (ax, flags, ay = contributions)
                    // followed by DRPair records (ax = the chain adjoint's offset, c); or, for
                    // targets that read the same chain adjoints, a gather tile (DRTerm kind 1,
                    // see DGatherTargets)
  D_FU_BASE = 96,   // forward unary fast form: 96 + (op - OP_NEG), a and dst smem
  D_RF_BASE = 128,  // reverse fast form: 128 + op, every adjoint location in smem
};

// Forward instruction as executed, 32 bytes.
struct alignas(16) DIns {
  uint8_t opc;
  uint8_t ma, mb, md;
  uint32_t a, b, d;    // byte offsets (smem / global region), unused for M_IMM
  uint32_t save;       // byte offset in the trajectory region, or kNone
  int32_t aux;
  double imm;
};
static_assert(sizeof(DIns) == 32, "DIns must be 32 bytes");

// Reverse instruction as executed, 48 bytes (carries its constant operand).
struct alignas(16) DRIns {
  uint8_t opc;
  uint8_t pad;
  uint16_t flags;      // RFlag bits
  uint32_t r, a, b;    // byte offsets of adjoint locations
  uint32_t va, vb, vr; // byte offsets in the trajectory region, or kNone
  int32_t aux;
  double imm;          // value of the constant operand (RF_VA_IMM / RF_VB_IMM)
  uint64_t pad2;
};
static_assert(sizeof(DRIns) == 48, "DRIns must be 48 bytes");

// Chain terms as executed.  They travel inline in the program stream, right
// after their chain instruction, in the order the executor consumes them, so
// the TMA program ring stages them with the instructions:
//   D_CHAIN    forward: n DFTerm records, term order
//   D_CHAIN    reverse: n DRTerm records, last term first
//   D_CHAIN_LC forward: ceil(n/2) DFPair records, terms (2k, 2k+1)
//   D_CHAIN_LC reverse: ceil(n/2) DRPair records, terms (n-1-2k, n-2-2k)
// Forward: operand locations; reverse: adjoint locations and trajectory
// offsets of the values an x*y term reads.
struct alignas(16) DFTerm {
  uint8_t kind, op, xm, ym;   // xm / ym: M_SMEM or M_GLOB
  uint32_t x, y;              // byte offsets
  uint32_t pad;
  double c;
  uint64_t pad2;
};
static_assert(sizeof(DFTerm) == sizeof(DIns), "forward term records are instruction-sized");
struct alignas(16) DRTerm {
  uint8_t kind, op;
  uint16_t flags;             // ChainFlag bits
  uint32_t ax, ay;            // adjoint byte offsets
  uint32_t vx, vy;            // trajectory byte offsets (x*y terms)
  uint32_t pad;
  double c;
  uint64_t pad2[2];
};
static_assert(sizeof(DRTerm) == sizeof(DRIns), "reverse term records are instruction-sized");
// Two terms of a linear-combination chain (Mul(c, x) or Mul(x, c), added).
struct alignas(16) DFPair {
  double c[2];
  uint32_t x[2];              // operand byte offsets
  uint8_t m[2];               // M_SMEM / M_GLOB, or M_INPUT (x = input index)
  uint8_t cx[2];              // 1: Mul(c, x), 0: Mul(x, c)
  uint32_t pad;
};
static_assert(sizeof(DFPair) == sizeof(DIns), "forward term records are instruction-sized");
struct alignas(16) DRPair {
  double c[2];
  uint32_t ax[2];             // adjoint byte offsets
  uint16_t flags[2];          // ChainFlag bits (CF_X_INIT, CF_X_GLOB)
  uint32_t pad;
  uint64_t pad2[2];
};
static_assert(sizeof(DRPair) == sizeof(DRIns), "reverse term records are instruction-sized");

// A gather tile in a D_GATHER stream: T targets (DRTerm header: kind 1, op = T,
// ay = n sources) whose contributions read the same n chain adjoints in the
// same order (the reverse of a dense layer), all with nonzero constants.  Then
// one DGatherTargets record and, per block of 12 sources, one DGatherSrc record
// followed by one record of constants per source (T values, f32 or f64).  Each
// target still adds its contributions in source order.
struct alignas(16) DGatherTargets {
  uint32_t tx[12];            // target adjoint byte offsets | GT_INIT | GT_GLOB
};
static_assert(sizeof(DGatherTargets) == sizeof(DRIns), "reverse records are instruction-sized");
struct alignas(16) DGatherSrc {
  uint32_t ax[12];            // chain adjoint byte offsets | GT_GLOB
};
static_assert(sizeof(DGatherSrc) == sizeof(DRIns), "reverse records are instruction-sized");
constexpr uint32_t GT_GLOB = 1u << 31;   // the slot is a global (far) slot
constexpr uint32_t GT_INIT = 1u << 30;   // the target's first contribution (starts from +0)
constexpr uint32_t GT_OFF = GT_INIT - 1; // byte offset bits

// Largest gather tile: its running targets stay in registers, as a dense
// group's outputs do; at most one record of constants per source (12 f32, 6 f64).
#if defined(__CUDACC__)
__host__ __device__
#endif
constexpr uint32_t gather_tile_max(uint32_t dense_max, bool f64) {
  return dense_max < (f64 ? 6u : 12u) ? dense_max : (f64 ? 6u : 12u);
}

// A dense group (D_DENSE: aux = m outputs, a = n terms) in the forward stream:
//   ceil(m/2) DDenseInit   the outputs' acc0
//   per block of 4 terms: one DDenseOps (the terms' operands), then for each
//     term of the block its m constants, 8 f32 or 4 f64 to a record
//   ceil(m/2) DDenseFin    the outputs' destinations and trajectory saves
struct alignas(16) DDenseInit {
  double imm[2];
  uint32_t off[2];            // byte offsets (M_SMEM / M_GLOB)
  uint8_t mode[2];            // M_SMEM / M_GLOB / M_IMM
  uint8_t pad[6];
};
static_assert(sizeof(DDenseInit) == 32, "dense records are instruction-sized");
struct alignas(16) DDenseOps {
  uint32_t x[4];              // byte offsets, or the input index (M_INPUT)
  uint8_t m[4];               // M_SMEM / M_GLOB / M_INPUT
  uint32_t pad[3];
};
static_assert(sizeof(DDenseOps) == 32, "dense records are instruction-sized");
struct alignas(16) DDenseFin {
  uint32_t d[2];              // byte offsets of the results
  uint32_t save[2];           // byte offsets in the trajectory region, or kNone
  uint8_t md[2];              // M_SMEM / M_GLOB
  uint8_t pad[14];
};
static_assert(sizeof(DDenseFin) == 32, "dense records are instruction-sized");

// Largest dense group for a value of `vbytes` bytes and `P` points per thread:
// the group's running values stay in registers, 64 words per thread at most;
// an even number, at most 16 (below 2: no groups).
#if defined(__CUDACC__)
__host__ __device__
#endif
constexpr uint32_t dense_group_max(uint32_t vbytes, uint32_t P) {
  return ((256u / (vbytes * P)) > 16u ? 16u : (256u / (vbytes * P))) & ~1u;
}

// One seeded input coefficient of a slot-seeded jet (sparse STDE over a
// differential operator): input `var` gets coefficient `slot` = `coef`.
struct SlotSeed {
  uint32_t var;
  uint32_t slot;
  double coef;
};
static_assert(sizeof(SlotSeed) == 16, "SlotSeed must be 16 bytes");

// Interpreter geometry shared by every kernel.
constexpr int kChunk = 128;   // instructions per staged chunk
constexpr int kStages = 3;    // staged chunks in flight
constexpr int kRingBytes = kStages * kChunk * 48;  // sized for the larger record

// Error word bits written by kernels (never trap).
enum KErr : uint32_t {
  KERR_TIMEOUT = 1u << 0,     // a bounded wait gave up
  KERR_BADINS = 1u << 1,      // malformed instruction
  KERR_BOUNDS = 1u << 2,      // (checked build) a slot or index out of its region
};

}  // namespace ech
