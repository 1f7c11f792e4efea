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
};

constexpr uint32_t kUnused = 0xFFFFFFFFu;
constexpr uint32_t kNone = 0xFFFFFFFFu;

// Operand modes.
enum Mode : uint8_t {
  M_SMEM = 0,  // register in the block's shared-memory slot file
  M_GLOB = 1,  // slot in the block's L2-resident global scratch ([slot][point])
  M_IMM = 2,   // constant: Ins::imm (forward) or RIns pool index (reverse)
  M_NONE = 3,
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

// Interpreter geometry shared by every kernel.
constexpr int kChunk = 128;   // instructions per staged chunk
constexpr int kStages = 3;    // staged chunks in flight

// Error word bits written by kernels (never trap).
enum KErr : uint32_t {
  KERR_TIMEOUT = 1u << 0,     // a bounded wait gave up
  KERR_BADINS = 1u << 1,      // malformed instruction
};

}  // namespace ech
