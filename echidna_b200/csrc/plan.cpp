// Host-side lowering: tape -> forward / reverse interpreter programs.
//
// 1. Liveness.  Ops that reach no requested output are dropped (their values are
//    unobservable, and in the reverse sweep their adjoints are exactly zero, so
//    skipping them matches reverse_sweep_core's zero-adjoint skip bit for bit).
// 2. The reverse program visits the surviving ops in decreasing tape order, so
//    every adjoint receives its contributions in the same order as the CPU
//    sweep (src/bytecode_tape/reverse.rs:32-105).
// 3. Virtual registers (slot values forward, adjoints reverse) get live
//    intervals over instruction positions and are assigned by linear scan
//    (Poletto & Sarkar 1999): up to `smem_cap` shared-memory registers, the
//    intervals ending furthest away spill to L2-resident global slots.
// 4. Values that a reverse partial reads are written once to a trajectory slot
//    by the forward program.
#include "plan.h"

#include <algorithm>
#include <cstdio>
#include <cmath>
#include <cstring>
#include <set>
#include <sstream>
#include <stdexcept>

namespace ech {

bool is_binary(uint32_t op) { return op >= OP_ADD && op <= OP_MIN; }

static const char* kOpNames[] = {
    "Input", "Const", "Add", "Sub", "Mul", "Div", "Rem", "Powf", "Atan2", "Hypot", "Max", "Min",
    "Neg", "Recip", "Sqrt", "Cbrt", "Powi", "Exp", "Exp2", "ExpM1", "Ln", "Log2", "Log10", "Ln1p",
    "Sin", "Cos", "Tan", "Asin", "Acos", "Atan", "Sinh", "Cosh", "Tanh", "Asinh", "Acosh", "Atanh",
    "Abs", "Signum", "Floor", "Ceil", "Round", "Trunc", "Fract", "Custom"};

static std::string arg_pair(uint32_t a, uint32_t b) {
  std::ostringstream o;
  o << "[" << a << ", " << b << "]";
  return o.str();
}

// src/bytecode_tape/mod.rs:575-705
std::string validate_bytecode_tape(const uint32_t* op, const uint32_t* a0, const uint32_t* a1, uint32_t nv,
                                   uint32_t ni, uint32_t output_index, const uint32_t* outs, uint32_t nouts,
                                   bool has_custom_ops) {
  std::ostringstream e;
  if (ni > nv) {
    e << "num_inputs (" << ni << ") > tape length (" << nv << ")";
    return e.str();
  }
  for (uint32_t i = 0; i < nv; ++i) {
    if (op[i] > OP_CUSTOM) {
      e << "opcodes[" << i << "] (" << op[i] << ") is not a valid opcode";
      return e.str();
    }
    if ((op[i] == OP_INPUT) != (i < ni)) {
      if (i < ni) e << "opcodes[" << i << "] should be Input but is " << kOpNames[op[i]];
      else e << "opcodes[" << i << "] is Input, but only the first " << ni << " entries may be inputs";
      return e.str();
    }
    if (i < ni && (a0[i] != kUnused || a1[i] != kUnused)) {
      e << "arg_indices[" << i << "] must be [UNUSED, UNUSED] for an Input entry, found " << arg_pair(a0[i], a1[i]);
      return e.str();
    }
  }
  if (output_index >= nv) {
    e << "output_index (" << output_index << ") >= tape length (" << nv << ")";
    return e.str();
  }
  for (uint32_t j = 0; j < nouts; ++j) {
    if (outs[j] >= nv) {
      e << "output_indices[" << j << "] (" << outs[j] << ") >= tape length (" << nv << ")";
      return e.str();
    }
  }
  for (uint32_t i = ni; i < nv; ++i) {
    const uint32_t o = op[i];
    if (o == OP_CONST) {
      if (a0[i] != kUnused || a1[i] != kUnused) {
        e << "arg_indices[" << i << "] must be [UNUSED, UNUSED] for a Const entry, found " << arg_pair(a0[i], a1[i]);
        return e.str();
      }
      continue;
    }
    if (a0[i] >= i) {
      e << "arg_indices[" << i << "][0] (" << a0[i] << ") must reference an earlier slot";
      return e.str();
    }
    if (o == OP_POWI) continue;
    if (o == OP_CUSTOM) {
      if (!has_custom_ops) {
        e << "arg_indices[" << i << "][1] (" << a1[i] << ") is not a registered custom-op callback";
        return e.str();
      }
      continue;
    }
    if (is_binary(o)) {
      if (a1[i] >= i) {
        e << "arg_indices[" << i << "][1] (" << a1[i] << ") must reference an earlier slot";
        return e.str();
      }
    } else if (a1[i] != kUnused) {
      e << "arg_indices[" << i << "][1] (" << a1[i] << ") should be UNUSED for unary op " << kOpNames[o];
      return e.str();
    }
  }
  return std::string();
}

// src/gpu/mod.rs:397-564
std::string validate_gpu_tape_data(const uint32_t* op, const uint32_t* a0, const uint32_t* a1, uint32_t n_op,
                                   uint32_t n_a0, uint32_t n_a1, uint32_t n_const, uint32_t num_ops,
                                   uint32_t num_inputs, uint32_t num_variables, uint32_t output_index,
                                   const uint32_t* outs, uint32_t nouts) {
  std::ostringstream e;
  const uint32_t n = num_ops;
  if (n_op != n) { e << "opcodes.len() (" << n_op << ") != num_ops (" << n << ")"; return e.str(); }
  if (n_a0 != n) { e << "arg0.len() (" << n_a0 << ") != num_ops (" << n << ")"; return e.str(); }
  if (n_a1 != n) { e << "arg1.len() (" << n_a1 << ") != num_ops (" << n << ")"; return e.str(); }
  if (num_ops != num_variables) {
    e << "num_ops (" << num_ops << ") != num_variables (" << num_variables << ")";
    return e.str();
  }
  if (n_const != num_variables) {
    e << "constants.len() (" << n_const << ") != num_variables (" << num_variables << ")";
    return e.str();
  }
  if (num_inputs > num_variables) {
    e << "num_inputs (" << num_inputs << ") > num_variables (" << num_variables << ")";
    return e.str();
  }
  const uint32_t ni = num_inputs;
  for (uint32_t i = 0; i < n; ++i) {
    if (op[i] > OP_FRACT) { e << "opcodes[" << i << "] (" << op[i] << ") is not a GPU-executable opcode"; return e.str(); }
    if ((op[i] == OP_INPUT) != (i < ni)) {
      if (i < ni) e << "opcodes[" << i << "] (" << op[i] << ") should be Input";
      else e << "opcodes[" << i << "] is Input, but only the first " << ni << " entries may be inputs";
      return e.str();
    }
  }
  for (uint32_t i = ni; i < n; ++i) {
    const uint32_t o = op[i];
    if (o == OP_CONST) continue;
    if (a0[i] >= i) { e << "arg0[" << i << "] (" << a0[i] << ") must reference an earlier slot"; return e.str(); }
    if (o == OP_POWI) continue;
    if (is_binary(o)) {
      if (a1[i] >= i) { e << "arg1[" << i << "] (" << a1[i] << ") must reference an earlier slot"; return e.str(); }
    } else if (a1[i] != kUnused) {
      e << "arg1[" << i << "] (" << a1[i] << ") should be the UNUSED sentinel for unary opcode " << o;
      return e.str();
    }
  }
  if (output_index >= num_variables) {
    e << "output_index (" << output_index << ") >= num_variables (" << num_variables << ")";
    return e.str();
  }
  for (uint32_t j = 0; j < nouts; ++j) {
    if (outs[j] >= num_variables) {
      e << "output_indices[" << j << "] (" << outs[j] << ") >= num_variables (" << num_variables << ")";
      return e.str();
    }
  }
  return std::string();
}

namespace {

// Arithmetic/special op counts per tape opcode (forward); used for the
// roofline's algorithmic-flops figure.  Specials are libm-class calls.
void op_cost(uint32_t o, uint64_t& flops, uint64_t& specials) {
  switch (o) {
    case OP_ADD: case OP_SUB: case OP_MUL: case OP_DIV: case OP_NEG: flops += 1; break;
    case OP_MAX: case OP_MIN: case OP_ABS: case OP_FRACT: flops += 1; break;
    case OP_RECIP: case OP_SQRT: flops += 1; break;
    case OP_POWI: flops += 2; break;
    case OP_SIGNUM: case OP_FLOOR: case OP_CEIL: case OP_ROUND: case OP_TRUNC: break;
    default: specials += 1; break;  // transcendental / libm
  }
}

struct Loc {
  uint8_t mode = M_NONE;
  uint32_t idx = kNone;
};

// Linear-scan register assignment over intervals [start, end] (inclusive
// instruction positions).  A register whose interval ends at position p may be
// reused by an interval starting at p (instructions read before they write).
struct LinearScan {
  struct Iv {
    int64_t start, end;
    uint32_t id;
  };
  std::vector<Iv> ivs;
  std::vector<Loc> loc;  // by id
  uint32_t smem_used = 0, glob_used = 0;
  uint64_t max_live = 0;

  void run(uint32_t nids, uint32_t cap) {
    loc.assign(nids, Loc{});
    std::sort(ivs.begin(), ivs.end(), [](const Iv& x, const Iv& y) {
      return x.start != y.start ? x.start < y.start : x.id < y.id;
    });
    // Pass 1: decide shared vs global (furthest-end spill).
    std::vector<uint8_t> in_smem(nids, 0);
    std::set<std::pair<int64_t, uint32_t>> active;  // (end, id) of smem-resident intervals
    {
      std::set<std::pair<int64_t, uint32_t>> all_active;
      for (const Iv& iv : ivs) {
        // An interval ending at iv.start is read by the instruction that writes
        // iv (reads precede the write), so its register is free for iv.
        while (!active.empty() && active.begin()->first <= iv.start) active.erase(active.begin());
        while (!all_active.empty() && all_active.begin()->first < iv.start) all_active.erase(all_active.begin());
        all_active.insert({iv.end, iv.id});
        max_live = std::max<uint64_t>(max_live, all_active.size());
        if (active.size() < cap) {
          active.insert({iv.end, iv.id});
          in_smem[iv.id] = 1;
        } else if (cap > 0) {
          auto last = std::prev(active.end());
          if (last->first > iv.end) {
            in_smem[last->second] = 0;
            active.erase(last);
            active.insert({iv.end, iv.id});
            in_smem[iv.id] = 1;
          }
        }
      }
    }
    // Pass 2: concrete indices, separately for each class.
    for (int cls = 0; cls < 2; ++cls) {
      std::set<std::pair<int64_t, uint32_t>> busy;  // (end, reg)
      std::vector<uint32_t> free_regs;
      uint32_t next = 0;
      for (const Iv& iv : ivs) {
        if ((in_smem[iv.id] != 0) != (cls == 0)) continue;
        while (!busy.empty() && busy.begin()->first <= iv.start) {
          free_regs.push_back(busy.begin()->second);
          busy.erase(busy.begin());
        }
        uint32_t r;
        if (!free_regs.empty()) {
          r = free_regs.back();
          free_regs.pop_back();
        } else {
          r = next++;
        }
        busy.insert({iv.end, r});
        loc[iv.id] = Loc{cls == 0 ? (uint8_t)M_SMEM : (uint8_t)M_GLOB, r};
      }
      if (cls == 0) smem_used = next;
      else glob_used = next;
    }
  }
};

}  // namespace

Plan build_plan(const HostTape& t, Kind kind, uint32_t smem_cap, uint32_t dense_max) {
  const uint32_t nv = t.nv, ni = t.ni;
  const bool reverse = (kind == Kind::Gradient || kind == Kind::Hvp);
  const bool emit_outputs = (kind != Kind::Hvp);
  const uint32_t seed = t.outs.empty() ? t.out_index : t.outs[0];
  Plan pl;
  pl.dense_max = dense_max < 1 ? 1 : dense_max;

  auto is_const = [&](uint32_t s) { return t.op[s] == OP_CONST; };
  auto has_b = [&](uint32_t i) { return is_binary(t.op[i]); };

  // ---------------- liveness of the forward program ----------------
  std::vector<uint8_t> live(nv, 0);
  if (emit_outputs)
    for (uint32_t o : t.outs) live[o] = 1;
  if (reverse) live[seed] = 1;
  for (int64_t i = (int64_t)nv - 1; i >= (int64_t)ni; --i) {
    if (!live[i] || is_const((uint32_t)i)) continue;
    live[t.a0[i]] = 1;
    if (has_b((uint32_t)i)) live[t.a1[i]] = 1;
  }

  // ---------------- reverse reachability and value needs ----------------
  std::vector<uint8_t> reach(nv, 0);
  std::vector<uint8_t> saved(nv, 0);
  if (reverse) {
    reach[seed] = 1;
    for (int64_t i = seed; i >= (int64_t)ni; --i) {
      if (!reach[i] || is_const((uint32_t)i)) continue;
      reach[t.a0[i]] = 1;
      if (has_b((uint32_t)i)) reach[t.a1[i]] = 1;
    }
  }
  // which values each reverse op reads: bit0=a, bit1=b, bit2=r
  auto rev_needs = [&](uint32_t i, bool needA, bool needB) -> uint32_t {
    const uint32_t o = t.op[i];
    switch (o) {
      case OP_ADD: case OP_SUB: case OP_NEG: case OP_FRACT:
      case OP_SIGNUM: case OP_FLOOR: case OP_CEIL: case OP_ROUND: case OP_TRUNC:
        return 0;
      case OP_MUL: return (needA ? 2u : 0u) | (needB ? 1u : 0u);
      case OP_DIV: return (needA ? 2u : 0u) | (needB ? 6u : 0u);
      case OP_REM: return needB ? 3u : 0u;
      case OP_POWF: return 7u;
      case OP_ATAN2: case OP_MAX: case OP_MIN: return 3u;
      case OP_HYPOT: return (needA ? 5u : 0u) | (needB ? 6u : 0u);
      case OP_POWI: return (t.a1[i] == 0x80000000u) ? 5u : 1u;
      case OP_SQRT: case OP_CBRT: case OP_EXP: case OP_EXP2: case OP_EXPM1: return 4u;
      default: return 1u;  // unary partial reads its argument
    }
  };
  std::vector<uint32_t> needs(nv, 0);
  if (reverse) {
    for (uint32_t i = ni; i < nv; ++i) {
      if (!reach[i] || is_const(i)) continue;
      const bool needA = !is_const(t.a0[i]);
      const bool needB = has_b(i) && !is_const(t.a1[i]);
      if (!needA && !needB) continue;
      needs[i] = rev_needs(i, needA, needB);
      if ((needs[i] & 1u) && !is_const(t.a0[i])) saved[t.a0[i]] = 1;
      if ((needs[i] & 2u) && !is_const(t.a1[i])) saved[t.a1[i]] = 1;
      if (needs[i] & 4u) saved[i] = 1;
    }
  }
  std::vector<uint32_t> traj(nv, kNone);
  uint32_t ntraj = 0;
  for (uint32_t s = 0; s < nv; ++s)
    if (saved[s]) traj[s] = ntraj++;
  pl.traj_slots = ntraj;
  pl.stats.traj_values = ntraj;

  // ---------------- fused linear chains ----------------
  // A chain is a run of consecutive live ops (no other live op in between)
  //   s_1 = acc0 (+|-) term_1, s_t = s_{t-1} (+|-) term_t, ...
  // where every s_t (t < K) and every absorbed Mul term has exactly one use.
  // Consecutive ops keep the reverse accumulation order identical to the
  // per-op sweep, and no operand outlives the run, so register pressure is
  // unchanged.
  std::vector<uint32_t> uses(nv, 0);
  for (uint32_t i = ni; i < nv; ++i) {
    if (!live[i] || is_const(i)) continue;
    uses[t.a0[i]]++;
    if (has_b(i)) uses[t.a1[i]]++;
  }
  if (emit_outputs)
    for (uint32_t o : t.outs) uses[o]++;
  if (reverse) uses[seed]++;
  struct Chain {
    uint32_t first, last;        // tape index range of the absorbed ops
    int64_t acc0;                // slot, or -1 for a constant
    double acc0_val;
    uint32_t tb, tn;             // term range in pl.terms
  };
  std::vector<Chain> chains;
  std::vector<int32_t> chain_end(nv, -1);  // at s_K: chain id
  std::vector<uint8_t> absorbed(nv, 0);
  {
    std::vector<uint32_t> L;
    for (uint32_t i = ni; i < nv; ++i)
      if (live[i] && !is_const(i)) L.push_back(i);
    auto is_addsub = [&](uint32_t i) { return t.op[i] == OP_ADD || t.op[i] == OP_SUB; };
    size_t k = 0;
    while (k < L.size()) {
      size_t j = k;
      int64_t prev = -1;
      std::vector<PTerm> tl;
      int64_t acc0 = -1;
      double acc0_val = 0.0;
      uint32_t nops = 0;
      while (j < L.size()) {
        int64_t mul = -1;
        uint32_t as;
        if (j + 1 < L.size() && t.op[L[j]] == OP_MUL && is_addsub(L[j + 1]) && uses[L[j]] == 1 &&
            (t.a0[L[j + 1]] == L[j]) != (t.a1[L[j + 1]] == L[j]) &&
            !(is_const(t.a0[L[j]]) && is_const(t.a1[L[j]]))) {
          mul = L[j];
          as = L[j + 1];
        } else if (is_addsub(L[j])) {
          as = L[j];
        } else {
          break;
        }
        const uint32_t o0 = t.a0[as], o1 = t.a1[as];
        bool chain_is_a;
        if (prev < 0) {
          if (mul >= 0) chain_is_a = (o1 == (uint32_t)mul);
          else chain_is_a = true;
        } else {
          const bool pa = (o0 == (uint32_t)prev), pb = (o1 == (uint32_t)prev);
          if (pa == pb || uses[prev] != 1) break;  // must consume prev exactly once
          chain_is_a = pa;
          if (mul >= 0 && (chain_is_a ? o1 : o0) != (uint32_t)mul) break;
        }
        const uint32_t term_slot = chain_is_a ? o1 : o0;
        const uint32_t acc_slot = chain_is_a ? o0 : o1;
        PTerm pt{};
        pt.xs = pt.ys = kNone;
        pt.vx = pt.vy = kNone;
        const bool sub = t.op[as] == OP_SUB;
        pt.op = (uint8_t)((sub ? 2 : 0) + (chain_is_a ? 0 : 1));
        if (mul >= 0) {
          const uint32_t ma = t.a0[mul], mb = t.a1[mul];
          if (is_const(ma)) { pt.kind = CK_CX; pt.c = t.vals[ma]; pt.xs = mb; }
          else if (is_const(mb)) { pt.kind = CK_XC; pt.c = t.vals[mb]; pt.xs = ma; }
          else { pt.kind = CK_XY; pt.xs = ma; pt.ys = mb; }
        } else if (is_const(term_slot)) {
          pt.kind = CK_C;
          pt.c = t.vals[term_slot];
        } else {
          pt.kind = CK_X;
          pt.xs = term_slot;
        }
        if (prev < 0) {
          if (is_const(acc_slot)) { acc0 = -1; acc0_val = t.vals[acc_slot]; }
          else acc0 = acc_slot;
        }
        tl.push_back(pt);
        nops += (mul >= 0) ? 2u : 1u;
        prev = as;
        j += (mul >= 0) ? 2 : 1;
        if (uses[as] != 1) break;
      }
      if (nops >= 2 && !tl.empty()) {
        Chain ch;
        ch.first = L[k];
        ch.last = (uint32_t)prev;
        ch.acc0 = acc0;
        ch.acc0_val = acc0_val;
        ch.tb = (uint32_t)pl.terms.size();
        ch.tn = (uint32_t)tl.size();
        for (size_t q = k; q < j; ++q) absorbed[L[q]] = 1;
        chain_end[ch.last] = (int32_t)chains.size();
        chains.push_back(ch);
        pl.terms.insert(pl.terms.end(), tl.begin(), tl.end());
        pl.stats.chains++;
        pl.stats.chain_ops += nops;
        k = j;
      } else {
        k += 1;
      }
    }
  }

  // ---------------- direct input terms (TaylorDirect) ----------------
  // In a linear-combination chain (every term c*x or x*c added) a term whose x
  // is an input and whose constant is finite reads the input jet at its source;
  // an input whose every use is such a term is never loaded into a slot.
  std::vector<uint8_t> term_direct(pl.terms.size(), 0);
  std::vector<uint32_t> direct_uses(kind == Kind::TaylorDirect ? ni : 0, 0);
  if (kind == Kind::TaylorDirect) {
    for (const Chain& ch : chains) {
      bool lc = ch.tn > 0;
      for (uint32_t q = ch.tb; q < ch.tb + ch.tn && lc; ++q) {
        const PTerm& pt = pl.terms[q];
        lc = (pt.kind == CK_CX || pt.kind == CK_XC) && pt.op == 0;
      }
      if (!lc) continue;
      for (uint32_t q = ch.tb; q < ch.tb + ch.tn; ++q) {
        const PTerm& pt = pl.terms[q];
        if (pt.xs < ni && t.op[pt.xs] == OP_INPUT && std::isfinite(pt.c)) {
          term_direct[q] = 1;
          direct_uses[pt.xs]++;
        }
      }
    }
  }

  // ---------------- dense groups ----------------
  // Consecutive linear-combination chains that read the same operands in the
  // same order (a dense layer: z_j = b_j + sum_i W_ji x_i) run as one forward
  // instruction that loads each operand once for the whole group.  Each
  // chain's additions keep their order, so results are those of the chains;
  // the reverse program still sees the chains one by one.  The group runs
  // where its first chain would, so every later chain's acc0 must be a
  // constant or a value defined before the first chain's ops.
  struct DenseGroup {
    uint32_t c0, m;
  };
  std::vector<DenseGroup> groups;
  std::vector<int32_t> group_of(chains.size(), -1);
  if (dense_max > 1) {
    auto lc_chain = [&](const Chain& ch) {
      if (ch.tn == 0) return false;
      for (uint32_t q = ch.tb; q < ch.tb + ch.tn; ++q) {
        const PTerm& pt = pl.terms[q];
        if ((pt.kind != CK_CX && pt.kind != CK_XC) || pt.op != 0) return false;
      }
      return true;
    };
    auto same_operands = [&](const Chain& a, const Chain& b) {
      if (a.tn != b.tn) return false;
      for (uint32_t q = 0; q < a.tn; ++q) {
        if (pl.terms[a.tb + q].xs != pl.terms[b.tb + q].xs) return false;
        if (term_direct[a.tb + q] != term_direct[b.tb + q]) return false;
      }
      return true;
    };
    uint32_t c = 0;
    while (c < chains.size()) {
      if (!lc_chain(chains[c])) { ++c; continue; }
      const Chain& lead = chains[c];
      uint32_t m = 1;
      while (c + m < chains.size() && m < dense_max) {
        const Chain& ch = chains[c + m];
        if (!lc_chain(ch) || !same_operands(lead, ch)) break;
        if (ch.acc0 >= 0 && (uint64_t)ch.acc0 >= lead.first) break;
        ++m;
      }
      // only full groups: the kernels' dense executor is specialised for
      // exactly dense_max outputs; shorter runs stay chains
      if (m == dense_max) {
        for (uint32_t k = 0; k < m; ++k) group_of[c + k] = (int32_t)groups.size();
        groups.push_back({c, m});
      }
      c += m;
    }
  }

  // ---------------- forward program (symbolic) ----------------
  struct FSym {
    uint8_t opc;
    int32_t aux;
    int64_t d;       // vreg (slot) or -1
    int64_t a, b;    // vreg or -1
    bool a_imm, b_imm;
    double a_val, b_val;
    uint32_t save;
    int32_t chain;   // chain id for XI_CHAIN
  };
  std::vector<FSym> fs;
  fs.reserve(nv + t.outs.size());
  std::vector<int64_t> def_pos(nv, -1), last_pos(nv, -1);
  auto use = [&](uint32_t s, int64_t pos) { last_pos[s] = std::max(last_pos[s], pos); };
  std::vector<std::pair<uint32_t, uint32_t>> out_pairs;  // (slot, j)
  if (emit_outputs)
    for (uint32_t j = 0; j < (uint32_t)t.outs.size(); ++j) out_pairs.push_back({t.outs[j], j});
  std::sort(out_pairs.begin(), out_pairs.end());
  size_t op_cursor = 0;
  auto emit_outputs_for = [&](uint32_t s) {
    while (op_cursor < out_pairs.size() && out_pairs[op_cursor].first < s) ++op_cursor;
    size_t k = op_cursor;
    while (k < out_pairs.size() && out_pairs[k].first == s) {
      FSym f{};
      f.opc = XI_STOUT;
      f.aux = (int32_t)out_pairs[k].second;
      f.d = -1;
      f.b = -1;
      f.save = kNone;
      f.chain = -1;
      if (is_const(s)) {
        f.a = -1; f.a_imm = true; f.a_val = t.vals[s];
      } else {
        f.a = s; f.a_imm = false;
        use(s, (int64_t)fs.size());
      }
      fs.push_back(f);
      ++k;
    }
  };
  // constant outputs first
  for (auto& pr : out_pairs) {
    if (!is_const(pr.first)) continue;
    FSym f{};
    f.opc = XI_STOUT; f.aux = (int32_t)pr.second; f.d = -1; f.a = -1; f.b = -1;
    f.a_imm = true; f.a_val = t.vals[pr.first]; f.save = kNone; f.chain = -1;
    fs.push_back(f);
  }
  int64_t tmp_vreg = nv;  // extra vregs for materialised constants
  std::vector<std::pair<int64_t, int64_t>> tmp_iv;  // (def, use) of temps
  for (uint32_t i = 0; i < nv; ++i) {
    if (!live[i] || is_const(i)) continue;
    const uint32_t o = t.op[i];
    FSym f{};
    f.d = i;
    f.save = traj[i];
    f.b = -1;
    f.chain = -1;
    if (absorbed[i] && chain_end[i] < 0) continue;  // inside a fused chain
    if (chain_end[i] >= 0 && group_of[chain_end[i]] >= 0) {
      const DenseGroup& g = groups[group_of[chain_end[i]]];
      if ((uint32_t)chain_end[i] != g.c0) {  // computed with its group's first chain
        emit_outputs_for(i);
        continue;
      }
      const int64_t pos = (int64_t)fs.size();
      f.opc = XI_DENSE;
      f.chain = group_of[chain_end[i]];
      f.aux = (int32_t)g.m;
      f.a = -1;
      f.save = kNone;
      const Chain& lead = chains[g.c0];
      for (uint32_t q = 0; q < lead.tn; ++q)
        if (!term_direct[lead.tb + q]) use(pl.terms[lead.tb + q].xs, pos);
      for (uint32_t k = 0; k < g.m; ++k) {
        const Chain& ch = chains[g.c0 + k];
        if (ch.acc0 >= 0) use((uint32_t)ch.acc0, pos);
        if (k > 0) def_pos[ch.last] = pos;
        for (uint32_t q = ch.first; q <= ch.last; ++q) {
          if (!absorbed[q]) continue;
          op_cost(t.op[q], pl.stats.flops_fwd, pl.stats.specials_fwd);
          pl.stats.fwd_ops++;
        }
      }
    } else if (chain_end[i] >= 0) {
      const Chain& ch = chains[chain_end[i]];
      const int64_t pos = (int64_t)fs.size();
      f.opc = XI_CHAIN;
      f.chain = chain_end[i];
      f.aux = (int32_t)ch.tn;
      if (ch.acc0 >= 0) { f.a = ch.acc0; f.a_imm = false; use((uint32_t)ch.acc0, pos); }
      else { f.a = -1; f.a_imm = true; f.a_val = ch.acc0_val; }
      for (uint32_t q = 0; q < ch.tn; ++q) {
        const PTerm& pt = pl.terms[ch.tb + q];
        if (term_direct[ch.tb + q]) continue;  // read at the source, not from a slot
        if (pt.xs != kNone) use(pt.xs, pos);
        if (pt.ys != kNone) use(pt.ys, pos);
      }
      for (uint32_t q = ch.first; q <= ch.last; ++q) {
        if (!absorbed[q]) continue;
        op_cost(t.op[q], pl.stats.flops_fwd, pl.stats.specials_fwd);
        pl.stats.fwd_ops++;
      }
    } else if (o == OP_INPUT) {
      if (!direct_uses.empty() && direct_uses[i] == uses[i]) continue;  // every use reads the source
      f.opc = XI_LDIN; f.aux = (int32_t)i; f.a = -1;
    } else {
      f.opc = (uint8_t)o;
      f.aux = (o == OP_POWI) ? (int32_t)t.a1[i] : 0;
      const uint32_t sa = t.a0[i];
      const bool bin = has_b(i);
      const uint32_t sb = bin ? t.a1[i] : kUnused;
      const bool ca = is_const(sa), cb = bin && is_const(sb);
      if (ca && cb) {
        // both operands constant (hand-built tapes): materialise a into a temp
        FSym m{};
        m.opc = XI_MOV; m.d = tmp_vreg; m.a = -1; m.b = -1; m.a_imm = true; m.a_val = t.vals[sa]; m.save = kNone;
        m.chain = -1;
        const int64_t p = (int64_t)fs.size();
        fs.push_back(m);
        tmp_iv.push_back({p, p + 1});
        f.a = tmp_vreg++;
        f.a_imm = false;
      } else if (ca) {
        f.a = -1; f.a_imm = true; f.a_val = t.vals[sa];
      } else {
        f.a = sa; f.a_imm = false; use(sa, (int64_t)fs.size());
      }
      if (bin) {
        if (cb) { f.b = -1; f.b_imm = true; f.b_val = t.vals[sb]; }
        else { f.b = sb; f.b_imm = false; use(sb, (int64_t)fs.size()); }
      }
      op_cost(o, pl.stats.flops_fwd, pl.stats.specials_fwd);
      pl.stats.fwd_ops++;
    }
    def_pos[i] = (int64_t)fs.size();
    fs.push_back(f);
    emit_outputs_for(i);
  }
  // forward intervals
  LinearScan lsf;
  for (uint32_t s = 0; s < nv; ++s) {
    if (def_pos[s] < 0) continue;
    int64_t e = std::max(last_pos[s], def_pos[s]);
    lsf.ivs.push_back({def_pos[s], e, s});
  }
  for (size_t k = 0; k < tmp_iv.size(); ++k) lsf.ivs.push_back({tmp_iv[k].first, tmp_iv[k].second, (uint32_t)(nv + k)});
  lsf.run((uint32_t)(nv + tmp_iv.size()), smem_cap);
  pl.stats.max_live_fwd = lsf.max_live;
  pl.fwd.reserve(fs.size());
  for (const FSym& f : fs) {
    Ins in{};
    in.opc = f.opc;
    in.aux = f.aux;
    in.save = f.save;
    in.imm = 0.0;
    if (f.d >= 0) { in.md = lsf.loc[f.d].mode; in.d = lsf.loc[f.d].idx; }
    else { in.md = M_NONE; in.d = kNone; }
    if (f.a >= 0) { in.ma = lsf.loc[f.a].mode; in.a = lsf.loc[f.a].idx; }
    else if (f.a_imm) { in.ma = M_IMM; in.a = 0; in.imm = f.a_val; }
    else { in.ma = M_NONE; in.a = kNone; }
    if (f.opc == XI_DENSE) {
      const DenseGroup& g = groups[f.chain];
      in.a = (uint32_t)pl.dense.size();
      in.ma = M_NONE;
      in.mb = M_NONE;
      in.md = M_NONE;
      in.d = kNone;
      in.save = kNone;
      for (uint32_t k = 0; k < g.m; ++k) {
        const Chain& ch = chains[g.c0 + k];
        PDenseOut o{};
        o.tb = ch.tb;
        o.tn = ch.tn;
        if (ch.acc0 >= 0) { o.am = lsf.loc[ch.acc0].mode; o.ai = lsf.loc[ch.acc0].idx; o.a_val = 0.0; }
        else { o.am = M_IMM; o.ai = 0; o.a_val = ch.acc0_val; }
        o.dm = lsf.loc[ch.last].mode;
        o.di = lsf.loc[ch.last].idx;
        o.save = traj[ch.last];
        pl.dense.push_back(o);
      }
    } else if (f.opc == XI_CHAIN) {
      in.mb = M_NONE;
      in.b = chains[f.chain].tb;  // first term
    } else if (f.b >= 0) { in.mb = lsf.loc[f.b].mode; in.b = lsf.loc[f.b].idx; }
    else if (f.b_imm) { in.mb = M_IMM; in.b = 0; in.imm = f.b_val; }
    else { in.mb = M_NONE; in.b = kNone; }
    pl.fwd.push_back(in);
  }
  for (size_t q = 0; q < pl.terms.size(); ++q) {
    PTerm& pt = pl.terms[q];
    pt.fxm = pt.fym = M_NONE;
    pt.fxi = pt.fyi = kNone;
    if (term_direct[q]) { pt.fxm = M_INPUT; pt.fxi = pt.xs; }
    else if (pt.xs != kNone) { pt.fxm = lsf.loc[pt.xs].mode; pt.fxi = lsf.loc[pt.xs].idx; }
    if (pt.ys != kNone) { pt.fym = lsf.loc[pt.ys].mode; pt.fyi = lsf.loc[pt.ys].idx; }
    pt.rxm = pt.rym = M_NONE;
    pt.rxi = pt.ryi = kNone;
    if (pt.kind == CK_XY) { pt.vx = traj[pt.xs]; pt.vy = traj[pt.ys]; }
  }
  uint32_t smem_used = lsf.smem_used, glob_used = lsf.glob_used;

  // ---------------- reverse program ----------------
  if (reverse) {
    struct RSym {
      uint8_t opc;
      int32_t aux;
      uint16_t flags;
      int64_t r, a, b;   // adjoint vregs (slot ids), -1 none
      uint32_t va, vb, vr;
      int32_t chain;
    };
    std::vector<RSym> rs;
    std::vector<int64_t> birth(nv, -1), death(nv, -1);
    // minimum reachable consumer of every input (its gradient is final after it)
    std::vector<int64_t> min_cons(ni, -1);
    for (uint32_t i = ni; i < nv; ++i) {
      if (!reach[i] || is_const(i)) continue;
      const uint32_t sa = t.a0[i];
      if (sa < ni && min_cons[sa] < 0) min_cons[sa] = i;
      if (has_b(i)) {
        const uint32_t sb = t.a1[i];
        if (sb < ni && min_cons[sb] < 0) min_cons[sb] = i;
      }
    }
    auto mk = [](uint8_t opc) {
      RSym r{};
      r.opc = opc;
      r.r = r.a = r.b = -1;
      r.va = r.vb = r.vr = kNone;
      r.chain = -1;
      return r;
    };
    const bool seed_const = is_const(seed);
    for (uint32_t k = 0; k < ni; ++k) {
      const bool seeded = (!seed_const && k == seed);
      if (min_cons[k] < 0 && !seeded) {
        RSym g = mk(XI_STGRAD);
        g.aux = (int32_t)k;
        rs.push_back(g);
      }
    }
    if (!seed_const) {
      RSym sd = mk(XI_SEED);
      sd.r = seed;
      birth[seed] = (int64_t)rs.size();
      rs.push_back(sd);
      if (seed < ni && min_cons[seed] < 0) {
        RSym g = mk(XI_STGRAD);
        g.aux = (int32_t)seed;
        g.r = seed;
        death[seed] = (int64_t)rs.size();
        rs.push_back(g);
      }
    }
    auto value_of = [&](uint32_t s, uint32_t& v, bool& imm) {
      if (is_const(s)) {
        v = (uint32_t)pl.pool.size();
        pl.pool.push_back(t.vals[s]);
        imm = true;
      } else {
        v = traj[s];
        imm = false;
      }
    };
    // inputs whose gradient completes once tape ops [lo, hi] have been processed
    auto emit_grads = [&](uint32_t lo, uint32_t hi) {
      for (uint32_t q = hi + 1; q-- > lo;) {
        if (!reach[q] || is_const(q)) continue;
        const uint32_t ops2[2] = {t.a0[q], has_b(q) ? t.a1[q] : kUnused};
        for (int w = 0; w < 2; ++w) {
          const uint32_t s2 = ops2[w];
          if (s2 == kUnused || s2 >= ni) continue;
          if (w == 1 && s2 == ops2[0]) continue;
          if (min_cons[s2] == (int64_t)q && death[s2] < 0) {
            RSym g = mk(XI_STGRAD);
            g.aux = (int32_t)s2;
            g.r = s2;
            death[s2] = (int64_t)rs.size();
            rs.push_back(g);
          }
        }
      }
    };
    for (int64_t ii = (int64_t)nv - 1; ii >= (int64_t)ni && !seed_const; --ii) {
      const uint32_t i = (uint32_t)ii;
      if (!reach[i] || is_const(i)) continue;
      if (chain_end[i] >= 0) {
        const Chain& ch = chains[chain_end[i]];
        const int64_t pos = (int64_t)rs.size();
        if (birth[i] >= 0) death[i] = pos;
        RSym r = mk(XI_CHAIN);
        r.chain = chain_end[i];
        r.r = i;
        r.aux = (int32_t)ch.tn;
        r.va = ch.tb;
        uint16_t fl = 0;
        // contributions in the per-op reverse order: for t = K..1 the Add/Sub
        // (operand a, then b), then the absorbed Mul (a, then b)
        auto touch = [&](uint32_t s2) -> bool {  // returns "first contribution"
          if (birth[s2] < 0) { birth[s2] = pos; return true; }
          return false;
        };
        for (uint32_t q = ch.tn; q-- > 0;) {
          PTerm& pt = pl.terms[ch.tb + q];
          const bool chain_a = (pt.op & 1) == 0;
          auto acc_side = [&]() {
            if (q == 0 && ch.acc0 >= 0) {
              fl |= RF_HAS_A;
              if (touch((uint32_t)ch.acc0)) fl |= RF_A_INIT;
            }
          };
          auto term_side = [&]() {
            if (pt.kind == CK_X) {
              pt.flags |= CF_X_ADJ;
              if (touch(pt.xs)) pt.flags |= CF_X_INIT;
            }
          };
          if (chain_a) { acc_side(); term_side(); } else { term_side(); acc_side(); }
          if (pt.kind == CK_CX || pt.kind == CK_XC) {
            pt.flags |= CF_X_ADJ;
            if (touch(pt.xs)) pt.flags |= CF_X_INIT;
          } else if (pt.kind == CK_XY) {
            pt.flags |= CF_X_ADJ | CF_Y_ADJ;
            if (touch(pt.xs)) pt.flags |= CF_X_INIT;
            if (touch(pt.ys)) pt.flags |= CF_Y_INIT;
          }
        }
        if (fl & RF_HAS_A) r.a = ch.acc0;
        r.flags = fl;
        rs.push_back(r);
        for (uint32_t q = ch.first; q <= ch.last; ++q) {
          if (!absorbed[q]) continue;
          op_cost(t.op[q], pl.stats.flops_rev, pl.stats.specials_rev);
          pl.stats.flops_rev += (t.op[q] == OP_MUL) ? 2 : 2;
          pl.stats.rev_ops++;
        }
        emit_grads(ch.first, ch.last);
        ii = (int64_t)ch.first;  // loop decrement continues below the chain
        continue;
      }
      const uint32_t o = t.op[i];
      const uint32_t sa = t.a0[i];
      const bool bin = has_b(i);
      const uint32_t sb = bin ? t.a1[i] : kUnused;
      const bool needA = !is_const(sa);
      const bool needB = bin && !is_const(sb);
      const int64_t pos = (int64_t)rs.size();
      if (birth[i] >= 0) death[i] = pos;  // adj(i) read here
      if (!needA && !needB) continue;
      RSym r = mk((uint8_t)o);
      r.aux = (o == OP_POWI) ? (int32_t)t.a1[i] : 0;
      r.r = i;
      r.a = needA ? (int64_t)sa : -1;
      r.b = needB ? (int64_t)sb : -1;
      uint16_t fl = 0;
      if (needA) fl |= RF_HAS_A;
      if (needB) fl |= RF_HAS_B;
      if (needA && birth[sa] < 0) { birth[sa] = pos; fl |= RF_A_INIT; }
      if (needB && birth[sb] < 0) { birth[sb] = pos; fl |= RF_B_INIT; }
      const uint32_t nd = needs[i];
      bool imm;
      if (nd & 1u) { value_of(sa, r.va, imm); if (imm) fl |= RF_VA_IMM; }
      if (nd & 2u) { value_of(sb, r.vb, imm); if (imm) fl |= RF_VB_IMM; }
      if (nd & 4u) { r.vr = traj[i]; }
      r.flags = fl;
      rs.push_back(r);
      op_cost(o, pl.stats.flops_rev, pl.stats.specials_rev);
      pl.stats.flops_rev += 2 * ((needA ? 1 : 0) + (needB ? 1 : 0));
      pl.stats.rev_ops++;
      emit_grads(i, i);
    }
    // ── reverse gather of linear-combination chains ──
    // A run of linear-combination chain reverses (constant acc0, every term
    // c*x or x*c added) is rewritten when the reverse ops between them touch
    // none of the run's adjoint targets and no chain's result is a target of
    // the run: each chain becomes XI_NORM at its own position (its adjoint
    // passed through the unit Add once, in place: the value every term of the
    // chain multiplies), and one XI_GATHER after the run's last chain
    // accumulates each target over the run's contributions, in the original
    // order, and stores it once.  Every adjoint receives the same additions in
    // the same order, so results are unchanged; the per-term read-modify-write
    // of a target becomes a read of a chain adjoint.
    bool grouped = false;
    {
      auto lc_chain = [&](const RSym& r) -> bool {
        if (r.opc != XI_CHAIN || (r.flags & RF_HAS_A) || r.chain < 0) return false;
        const Chain& ch = chains[r.chain];
        if (ch.tn == 0) return false;
        for (uint32_t q = ch.tb; q < ch.tb + ch.tn; ++q) {
          const PTerm& pt = pl.terms[q];
          if ((pt.kind != CK_CX && pt.kind != CK_XC) || pt.op != 0) return false;
        }
        return true;
      };
      // adjoint slots an entry reads or writes
      auto touched = [&](const RSym& r, std::vector<int64_t>& out) {
        out.clear();
        if (r.r >= 0) out.push_back(r.r);
        if (r.a >= 0) out.push_back(r.a);
        if (r.b >= 0) out.push_back(r.b);
        if (r.opc == XI_CHAIN && r.chain >= 0) {
          const Chain& ch = chains[r.chain];
          for (uint32_t q = ch.tb; q < ch.tb + ch.tn; ++q) {
            const PTerm& pt = pl.terms[q];
            if (pt.flags & CF_X_ADJ) out.push_back(pt.xs);
            if (pt.flags & CF_Y_ADJ) out.push_back(pt.ys);
          }
        }
      };
      std::vector<RSym> out;
      out.reserve(rs.size());
      std::vector<int64_t> tv;
      size_t k = 0;
      while (k < rs.size()) {
        if (!lc_chain(rs[k])) {
          out.push_back(rs[k++]);
          continue;
        }
        std::vector<size_t> members;
        std::set<int64_t> targets, results;
        size_t last = k;
        for (size_t j = k; j < rs.size(); ++j) {
          const RSym& e = rs[j];
          if (lc_chain(e) && !targets.count(e.r)) {
            const Chain& ch = chains[e.chain];
            bool ok = true;
            for (uint32_t q = ch.tb; q < ch.tb + ch.tn && ok; ++q) ok = !results.count(pl.terms[q].xs);
            if (ok) {
              members.push_back(j);
              for (uint32_t q = ch.tb; q < ch.tb + ch.tn; ++q) targets.insert(pl.terms[q].xs);
              results.insert(e.r);
              last = j;
              continue;
            }
          }
          // runs before the gather: it must not touch the members' targets or results
          touched(e, tv);
          bool conflict = false;
          for (int64_t x : tv) conflict = conflict || targets.count(x) || results.count(x);
          if (conflict) break;
        }
        if (members.size() < 2) {
          out.push_back(rs[k++]);
          continue;
        }
        // targets in order of first contribution
        std::vector<int64_t> order;
        std::set<int64_t> seen;
        for (size_t m : members) {
          const Chain& ch = chains[rs[m].chain];
          for (uint32_t q = ch.tn; q-- > 0;) {
            const int64_t x = pl.terms[ch.tb + q].xs;
            if (seen.insert(x).second) order.push_back(x);
          }
        }
        RSym g = mk(XI_GATHER);
        g.va = (uint32_t)pl.gathers.size();
        g.aux = (int32_t)order.size();
        for (int64_t x : order) {
          GRec h{};
          h.s = (uint32_t)x;
          const size_t hpos = pl.gathers.size();
          pl.gathers.push_back(h);
          uint32_t nc = 0;
          uint16_t hf = 0;
          for (size_t m : members) {
            const Chain& ch = chains[rs[m].chain];
            for (uint32_t q = ch.tn; q-- > 0;) {
              const PTerm& pt = pl.terms[ch.tb + q];
              if (pt.xs != (uint32_t)x) continue;
              if (pt.flags & CF_X_INIT) hf |= CF_X_INIT;
              GRec c{};
              c.s = (uint32_t)rs[m].r;
              c.c = pt.c;
              pl.gathers.push_back(c);
              ++nc;
            }
          }
          pl.gathers[hpos].n = nc;
          pl.gathers[hpos].flags = hf;
        }
        size_t mi = 0;
        for (size_t j = k; j <= last; ++j) {
          if (mi < members.size() && members[mi] == j) {
            RSym nr = mk(XI_NORM);
            nr.r = rs[j].r;
            out.push_back(nr);
            ++mi;
          } else {
            out.push_back(rs[j]);
          }
        }
        out.push_back(g);
        grouped = true;
        k = last + 1;
      }
      if (grouped) {
        rs.swap(out);
        // live ranges from the rewritten order: first to last access
        std::fill(birth.begin(), birth.end(), -1);
        std::fill(death.begin(), death.end(), -1);
        auto at = [&](int64_t s2, int64_t pos) {
          if (s2 < 0) return;
          if (birth[s2] < 0) birth[s2] = pos;
          death[s2] = pos;
        };
        for (size_t pos = 0; pos < rs.size(); ++pos) {
          const RSym& e = rs[pos];
          if (e.opc == XI_GATHER) {
            // the gather reads its sources while it writes targets, so a target
            // must not take a source's register: sources stay live one past it
            for (uint32_t q = e.va, h = 0; h < (uint32_t)e.aux; ++h) {
              const GRec& hd = pl.gathers[q];
              for (uint32_t c = 1; c <= hd.n; ++c) at(pl.gathers[q + c].s, (int64_t)pos + 1);
              at(hd.s, (int64_t)pos);
              q += 1 + hd.n;
            }
            continue;
          }
          touched(e, tv);
          for (int64_t x : tv) at(x, (int64_t)pos);
        }
      }
    }
    // Every reachable op other than the seed has a reachable consumer, so its
    // adjoint is born (first contribution, RF_*_INIT) before it is read.
    LinearScan lsr;
    for (uint32_t s = 0; s < nv; ++s) {
      if (birth[s] < 0) continue;
      int64_t e = std::max(death[s], birth[s]);
      lsr.ivs.push_back({birth[s], e, s});
    }
    lsr.run(nv, smem_cap);
    pl.stats.max_live_rev = lsr.max_live;
    pl.rev.reserve(rs.size());
    for (const RSym& r : rs) {
      RIns in{};
      in.opc = r.opc;
      in.aux = r.aux;
      uint16_t fl = r.flags;
      if (r.r >= 0) {
        in.r = lsr.loc[r.r].idx;
        if (lsr.loc[r.r].mode == M_GLOB) fl |= RF_R_GLOB;
      } else {
        in.r = kNone;
      }
      if (r.a >= 0) {
        in.a = lsr.loc[r.a].idx;
        if (lsr.loc[r.a].mode == M_GLOB) fl |= RF_A_GLOB;
      } else {
        in.a = kNone;
      }
      if (r.b >= 0) {
        in.b = lsr.loc[r.b].idx;
        if (lsr.loc[r.b].mode == M_GLOB) fl |= RF_B_GLOB;
      } else {
        in.b = kNone;
      }
      in.va = r.va;
      in.vb = r.vb;
      in.vr = r.vr;
      in.flags = fl;
      pl.rev.push_back(in);
    }
    for (GRec& gr : pl.gathers) {
      gr.mode = lsr.loc[gr.s].mode;
      gr.idx = lsr.loc[gr.s].idx;
    }
    for (const Chain& ch : chains) {
      for (uint32_t q = 0; q < ch.tn; ++q) {
        PTerm& pt = pl.terms[ch.tb + q];
        if (pt.flags & CF_X_ADJ) {
          pt.rxm = lsr.loc[pt.xs].mode;
          pt.rxi = lsr.loc[pt.xs].idx;
        }
        if (pt.flags & CF_Y_ADJ) {
          pt.rym = lsr.loc[pt.ys].mode;
          pt.ryi = lsr.loc[pt.ys].idx;
        }
      }
    }
    smem_used = std::max(smem_used, lsr.smem_used);
    glob_used = std::max(glob_used, lsr.glob_used);
  }
  pl.smem_regs = smem_used;
  pl.far_slots = glob_used;
  if (pl.pool.empty()) pl.pool.push_back(0.0);
  return pl;
}

// A chain whose every term is c*x or x*c added to the running value runs the
// specialised linear-combination loop (D_CHAIN_LC).
static bool linear_combination(const Plan& p, uint32_t first, uint32_t n) {
  if (n == 0) return false;
  for (uint32_t q = first; q < first + n; ++q) {
    const PTerm& t = p.terms[q];
    if ((t.kind != CK_CX && t.kind != CK_XC) || t.op != 0) return false;
  }
  return true;
}

// A term record reinterpreted as an instruction-sized record of the stream.
template <class R, class T>
static R as_record(const T& t) {
  static_assert(sizeof(R) == sizeof(T), "records of one stream have one size");
  R r;
  std::memcpy(&r, &t, sizeof r);
  return r;
}

bool encode_plan(const Plan& p, uint32_t tile, uint32_t vbytes, bool f32, DevProgram& out, std::string& err) {
  const uint64_t row = (uint64_t)tile * vbytes;
  bool ok = true;
  auto off = [&](uint32_t idx) -> uint32_t {
    if (idx == kNone) return kNone;
    const uint64_t o = (uint64_t)idx * row;
    if (o >= 0xFFFFFFFFull) {
      ok = false;
      return 0;
    }
    return (uint32_t)o;
  };
  // linear-combination term constants: f32 programs carry the f32 rounding
  // (round to nearest, as the device's conversion) in the field's low word
  auto lc_c = [&](double c) {
    if (!f32) return c;
    const float f = (float)c;
    uint32_t u;
    std::memcpy(&u, &f, sizeof u);
    const uint64_t w = u;
    double r;
    std::memcpy(&r, &w, sizeof r);
    return r;
  };
  auto fterm = [&](const PTerm& pt) {
    DFTerm f{};
    f.kind = pt.kind;
    f.op = pt.op;
    f.xm = pt.fxm;
    f.ym = pt.fym;
    f.x = (pt.fxm == M_SMEM || pt.fxm == M_GLOB) ? off(pt.fxi) : kNone;
    f.y = (pt.fym == M_SMEM || pt.fym == M_GLOB) ? off(pt.fyi) : kNone;
    f.c = pt.c;
    return f;
  };
  auto rterm = [&](const PTerm& pt) {
    DRTerm r{};
    r.kind = pt.kind;
    r.op = pt.op;
    uint16_t fl = pt.flags & (CF_X_INIT | CF_Y_INIT | CF_X_ADJ | CF_Y_ADJ);
    if (pt.rxm == M_GLOB) fl |= CF_X_GLOB;
    if (pt.rym == M_GLOB) fl |= CF_Y_GLOB;
    r.flags = fl;
    r.ax = (pt.flags & CF_X_ADJ) ? off(pt.rxi) : kNone;
    r.ay = (pt.flags & CF_Y_ADJ) ? off(pt.ryi) : kNone;
    r.vx = off(pt.vx);
    r.vy = off(pt.vy);
    r.c = pt.c;
    return r;
  };
  out.fwd.clear();
  out.rev.clear();
  out.fwd.reserve(p.fwd.size());
  for (const Ins& in : p.fwd) {
    DIns d{};
    d.ma = in.ma;
    d.mb = in.mb;
    d.md = in.md;
    d.a = (in.ma == M_SMEM || in.ma == M_GLOB) ? off(in.a) : 0u;
    d.b = (in.mb == M_SMEM || in.mb == M_GLOB) ? off(in.b) : 0u;
    d.d = (in.md == M_SMEM || in.md == M_GLOB) ? off(in.d) : 0u;
    d.save = off(in.save);
    d.aux = in.aux;
    d.imm = in.imm;
    uint8_t opc = in.opc;
    const bool dsm = in.md == M_SMEM;
    if (opc == XI_DENSE) {
      const uint32_t first = in.a, m = (uint32_t)in.aux;
      const PDenseOut& lead = p.dense[first];
      const uint32_t n = lead.tn;
      DIns h{};
      h.opc = D_DENSE;
      h.aux = (int32_t)m;
      h.a = n;
      h.ma = h.mb = h.md = M_NONE;
      h.save = kNone;
      out.fwd.push_back(h);
      for (uint32_t k = 0; k < m; k += 2) {
        DDenseInit r{};
        for (uint32_t j = 0; j < 2 && k + j < m; ++j) {
          const PDenseOut& o = p.dense[first + k + j];
          r.mode[j] = o.am;
          r.off[j] = o.am == M_IMM ? 0u : off(o.ai);
          r.imm[j] = o.a_val;
        }
        out.fwd.push_back(as_record<DIns>(r));
      }
      const uint32_t per_rec = f32 ? 8u : 4u;
      for (uint32_t q0 = 0; q0 < n; q0 += 4) {
        DDenseOps ops{};
        for (uint32_t j = 0; j < 4 && q0 + j < n; ++j) {
          const PTerm& pt = p.terms[lead.tb + q0 + j];
          ops.m[j] = pt.fxm;
          ops.x[j] = pt.fxm == M_INPUT ? pt.fxi : off(pt.fxi);
        }
        out.fwd.push_back(as_record<DIns>(ops));
        for (uint32_t q = q0; q < q0 + 4 && q < n; ++q) {
          for (uint32_t k = 0; k < m; k += per_rec) {
            unsigned char rec[32] = {};
            for (uint32_t j = 0; j < per_rec && k + j < m; ++j) {
              const double c = p.terms[p.dense[first + k + j].tb + q].c;
              if (f32) {
                const float fc = (float)c;
                std::memcpy(rec + 4 * j, &fc, 4);
              } else {
                std::memcpy(rec + 8 * j, &c, 8);
              }
            }
            DIns r;
            std::memcpy(&r, rec, sizeof r);
            out.fwd.push_back(r);
          }
        }
      }
      for (uint32_t k = 0; k < m; k += 2) {
        DDenseFin r{};
        for (uint32_t j = 0; j < 2; ++j) {
          r.save[j] = kNone;
          if (k + j >= m) continue;
          const PDenseOut& o = p.dense[first + k + j];
          r.md[j] = o.dm;
          r.d[j] = off(o.di);
          r.save[j] = off(o.save);
        }
        out.fwd.push_back(as_record<DIns>(r));
      }
      continue;
    }
    if (opc == XI_CHAIN) {
      // the terms follow the instruction in the stream
      const uint32_t first = in.b, n = (uint32_t)in.aux;
      const bool lc = linear_combination(p, first, n);
      d.b = 0;
      d.mb = M_NONE;
      d.opc = lc ? D_CHAIN_LC : D_CHAIN;
      out.fwd.push_back(d);
      if (lc) {
        for (uint32_t k = 0; k < n; k += 2) {
          DFPair pr{};
          for (uint32_t j = 0; j < 2 && k + j < n; ++j) {
            const PTerm& pt = p.terms[first + k + j];
            pr.c[j] = lc_c(pt.c);
            pr.x[j] = pt.fxm == M_INPUT ? pt.fxi : off(pt.fxi);
            pr.m[j] = pt.fxm;
            pr.cx[j] = pt.kind == CK_CX ? 1 : 0;
          }
          out.fwd.push_back(as_record<DIns>(pr));
        }
      } else {
        for (uint32_t q = first; q < first + n; ++q) out.fwd.push_back(as_record<DIns>(fterm(p.terms[q])));
      }
      continue;
    }
    if (dsm && (opc == OP_ADD || opc == OP_SUB || opc == OP_MUL || opc == OP_DIV)) {
      const int base = opc == OP_ADD ? D_ADD_RR : opc == OP_SUB ? D_SUB_RR : opc == OP_MUL ? D_MUL_RR : D_DIV_RR;
      if (in.ma == M_SMEM && in.mb == M_SMEM) opc = (uint8_t)base;
      else if (in.ma == M_IMM && in.mb == M_SMEM) opc = (uint8_t)(base + 1);
      else if (in.ma == M_SMEM && in.mb == M_IMM) opc = (uint8_t)(base + 2);
    } else if (dsm && opc >= OP_NEG && opc <= OP_FRACT && in.ma == M_SMEM) {
      opc = (uint8_t)(D_FU_BASE + (opc - OP_NEG));
    }
    d.opc = opc;
    out.fwd.push_back(d);
  }
  out.rev.reserve(p.rev.size());
  for (const RIns& in : p.rev) {
    DRIns d{};
    d.flags = in.flags;
    d.aux = in.aux;
    if (in.opc == XI_NORM) {
      d.opc = D_NORM;
      d.r = off(in.r);
      d.a = d.b = d.va = d.vb = d.vr = kNone;
      out.rev.push_back(d);
      continue;
    }
    if (in.opc == XI_GATHER) {
      // per target: a header (target offset, flags, contribution count), then
      // its contributions two per record (chain adjoint offset, constant)
      d.opc = D_GATHER;
      d.r = d.a = d.b = d.va = d.vb = d.vr = kNone;
      out.rev.push_back(d);
      // gather tiles: consecutive targets whose contributions read the same
      // chain adjoints in the same order, every constant nonzero in the value
      // type (then no contribution is left out, and the targets share each
      // source's load, zero test and zero product)
      const uint32_t tmax = gather_tile_max(p.dense_max, !f32);
      std::vector<uint32_t> hpos;  // header index of each target
      for (uint32_t h = 0, q = in.va; h < (uint32_t)in.aux; ++h) {
        hpos.push_back(q);
        q += 1 + p.gathers[q].n;
      }
      auto zero_const = [&](double c) {
        const double cv = lc_c(c);
        if (!f32) return cv == 0.0;
        float f;
        std::memcpy(&f, &cv, sizeof f);
        return f == 0.0f;
      };
      auto tileable = [&](uint32_t q) {
        const GRec& hd = p.gathers[q];
        if (hd.n == 0 || off(hd.idx) > GT_OFF) return false;
        for (uint32_t c = 1; c <= hd.n; ++c)
          if (zero_const(p.gathers[q + c].c) || off(p.gathers[q + c].idx) > GT_OFF) return false;
        return true;
      };
      auto same_sources = [&](uint32_t qa, uint32_t qb) {
        const GRec& a = p.gathers[qa];
        const GRec& b = p.gathers[qb];
        if (a.n != b.n) return false;
        for (uint32_t c = 1; c <= a.n; ++c) {
          const GRec& ga = p.gathers[qa + c];
          const GRec& gb = p.gathers[qb + c];
          if (ga.idx != gb.idx || ga.mode != gb.mode) return false;
        }
        return true;
      };
      for (uint32_t h = 0; h < (uint32_t)in.aux;) {
        uint32_t T = 1;
        if (tmax >= 2 && tileable(hpos[h]))
          while (h + T < (uint32_t)in.aux && T < tmax && tileable(hpos[h + T]) && same_sources(hpos[h], hpos[h + T]))
            ++T;
        // only full tiles (the kernel's tile executor has no per-target bounds)
        if (T >= 2 && T == tmax) {
          const uint32_t ns = p.gathers[hpos[h]].n;
          DRTerm head{};
          head.kind = 1;
          head.op = (uint8_t)T;
          head.ay = ns;
          out.rev.push_back(as_record<DRIns>(head));
          DGatherTargets tg{};
          for (uint32_t k = 0; k < T; ++k) {
            const GRec& hd = p.gathers[hpos[h + k]];
            tg.tx[k] = off(hd.idx) | ((hd.flags & CF_X_INIT) ? GT_INIT : 0u) | (hd.mode == M_GLOB ? GT_GLOB : 0u);
          }
          out.rev.push_back(as_record<DRIns>(tg));
          for (uint32_t s0 = 0; s0 < ns; s0 += 12) {
            DGatherSrc sr{};
            for (uint32_t j = 0; j < 12 && s0 + j < ns; ++j) {
              const GRec& g = p.gathers[hpos[h] + 1 + s0 + j];
              sr.ax[j] = off(g.idx) | (g.mode == M_GLOB ? GT_GLOB : 0u);
            }
            out.rev.push_back(as_record<DRIns>(sr));
            for (uint32_t j = s0; j < s0 + 12 && j < ns; ++j) {
              unsigned char rec[sizeof(DRIns)] = {};
              for (uint32_t k = 0; k < T; ++k) {
                const double c = p.gathers[hpos[h + k] + 1 + j].c;
                if (f32) {
                  const float fc = (float)c;
                  std::memcpy(rec + 4 * k, &fc, 4);
                } else {
                  std::memcpy(rec + 8 * k, &c, 8);
                }
              }
              DRIns r;
              std::memcpy(&r, rec, sizeof r);
              out.rev.push_back(r);
            }
          }
          out.gather_tiles += 1;
          h += T;
          continue;
        }
        const uint32_t q = hpos[h];
        const GRec& hd = p.gathers[q];
        // a contribution whose constant is zero (after rounding to the value
        // type) never changes the target: it is left out, so the kernel skips
        // the zero-multiplier test
        std::vector<const GRec*> kept;
        for (uint32_t c = 0; c < hd.n; ++c) {
          const GRec& g = p.gathers[q + 1 + c];
          const double cv = lc_c(g.c);
          const bool zero = f32 ? ([&] { float f; std::memcpy(&f, &cv, sizeof f); return f == 0.0f; })()
                                : cv == 0.0;
          if (!zero) kept.push_back(&g);
        }
        DRTerm head{};
        head.flags = (uint16_t)(hd.flags | (hd.mode == M_GLOB ? CF_X_GLOB : 0));
        head.ax = off(hd.idx);
        head.ay = (uint32_t)kept.size();
        out.rev.push_back(as_record<DRIns>(head));
        for (size_t c = 0; c < kept.size(); c += 2) {
          DRPair pr{};
          for (size_t j = 0; j < 2 && c + j < kept.size(); ++j) {
            const GRec& g = *kept[c + j];
            pr.c[j] = lc_c(g.c);
            pr.ax[j] = off(g.idx);
            pr.flags[j] = g.mode == M_GLOB ? (uint16_t)CF_X_GLOB : (uint16_t)0;
          }
          out.rev.push_back(as_record<DRIns>(pr));
        }
        ++h;
      }
      continue;
    }
    if (in.opc == XI_CHAIN) {
      // the terms follow the instruction, last term first
      const uint32_t first = in.va, n = (uint32_t)in.aux;
      const bool lc = linear_combination(p, first, n);
      d.opc = lc ? D_CHAIN_LC : D_CHAIN;
      if (lc) {
        // pairwise distinct adjoint targets let the kernel batch the terms' updates
        std::set<std::pair<uint8_t, uint32_t>> targets;
        for (uint32_t q = first; q < first + n; ++q) targets.insert({p.terms[q].rxm, p.terms[q].rxi});
        if (targets.size() == n) d.flags |= RF_LC_DISTINCT;
      }
      d.r = off(in.r);
      d.a = off(in.a);
      d.b = kNone;
      d.va = kNone;
      d.vb = kNone;
      d.vr = kNone;
      out.rev.push_back(d);
      if (lc) {
        for (uint32_t k = 0; k < n; k += 2) {
          DRPair pr{};
          for (uint32_t j = 0; j < 2 && k + j < n; ++j) {
            const PTerm& pt = p.terms[first + n - 1 - k - j];
            const DRTerm r = rterm(pt);
            pr.c[j] = lc_c(pt.c);
            pr.ax[j] = r.ax;
            pr.flags[j] = r.flags;
          }
          out.rev.push_back(as_record<DRIns>(pr));
        }
      } else {
        for (uint32_t k = 0; k < n; ++k) out.rev.push_back(as_record<DRIns>(rterm(p.terms[first + n - 1 - k])));
      }
      continue;
    }
    d.r = off(in.r);
    d.a = off(in.a);
    d.b = off(in.b);
    d.vr = off(in.vr);
    d.imm = 0.0;
    if (in.flags & RF_VA_IMM) {
      d.imm = p.pool[in.va];
      d.va = kNone;
    } else {
      d.va = off(in.va);
    }
    if (in.flags & RF_VB_IMM) {
      if (in.flags & RF_VA_IMM) {
        err = "reverse op with two constant operands";
        return false;
      }
      d.imm = p.pool[in.vb];
      d.vb = kNone;
    } else {
      d.vb = off(in.vb);
    }
    uint8_t opc = in.opc;
    if (opc != XI_SEED && opc != XI_STGRAD && !(in.flags & (RF_R_GLOB | RF_A_GLOB | RF_B_GLOB)))
      opc = (uint8_t)(D_RF_BASE + opc);
    d.opc = opc;
    out.rev.push_back(d);
  }
  if (!ok) err = "slot region exceeds the 32-bit offset encoding; use a smaller tile";
  return ok;
}

}  // namespace ech
