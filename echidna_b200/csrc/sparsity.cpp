// Host-side structural sparsity and graph coloring for the sparse Jacobian /
// Hessian drop-ins.  Patterns and colors must equal the reference's exactly
// (the GPU sweeps are seeded by them), so the algorithms follow:
//   detect_sparsity_impl           src/bytecode_tape/sparse.rs:463-593
//   classify_op / is_binary_op     src/bytecode_tape/sparse.rs:603-668
//   detect_jacobian_sparsity_impl  src/bytecode_tape/sparse.rs:716-776
//   greedy_coloring                src/sparse.rs:57-98   (distance-2 via G^2)
//   column_coloring / row_coloring src/sparse.rs:292-316 (intersection graph)
//   greedy_distance1_coloring      src/sparse.rs:358-413 (largest degree first, stable)
// Dependency sets are bitsets of 64-bit words, one per tape slot.
#include <stdint.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/echidna_b200.h"
#include "ech_types.h"

namespace {

using namespace ech;

enum class OpClass { Linear, UnaryNonlinear, BinaryNonlinear, ZeroDerivative };

OpClass classify(uint32_t op) {
  switch (op) {
    case OP_ADD: case OP_SUB: case OP_NEG: case OP_FRACT:
      return OpClass::Linear;
    case OP_MUL: case OP_DIV: case OP_POWF: case OP_ATAN2: case OP_HYPOT: case OP_CUSTOM:
      return OpClass::BinaryNonlinear;
    case OP_ABS: case OP_SIGNUM: case OP_FLOOR: case OP_CEIL: case OP_ROUND: case OP_TRUNC:
    case OP_MAX: case OP_MIN: case OP_REM:
      return OpClass::ZeroDerivative;
    default:  // Recip .. Atanh, Powi
      return OpClass::UnaryNonlinear;
  }
}

bool binary_op(uint32_t op) {
  switch (op) {
    case OP_ADD: case OP_SUB: case OP_MUL: case OP_DIV: case OP_REM: case OP_POWF: case OP_ATAN2:
    case OP_HYPOT: case OP_MAX: case OP_MIN: case OP_CUSTOM:
      return true;
    default:
      return false;
  }
}

struct Deps {
  size_t words;
  std::vector<uint64_t> bits;  // [slot][word]
  Deps(size_t nv, size_t ni) : words((ni + 63) / 64), bits(nv * ((ni + 63) / 64), 0) {}
  uint64_t* row(size_t i) { return bits.data() + i * words; }
  void unite(size_t dst, size_t src) {
    if (dst == src) return;
    uint64_t* a = row(dst);
    const uint64_t* b = row(src);
    for (size_t w = 0; w < words; ++w) a[w] |= b[w];
  }
  // positions of set bits below max_bits, ascending
  std::vector<uint32_t> extract(size_t i, size_t max_bits) {
    std::vector<uint32_t> r;
    const uint64_t* a = row(i);
    for (size_t w = 0; w < words; ++w) {
      uint64_t x = a[w];
      while (x) {
        const uint32_t pos = (uint32_t)(w * 64 + __builtin_ctzll(x));
        if (pos < max_bits) r.push_back(pos);
        x &= x - 1;
      }
    }
    return r;
  }
};

using Pair = std::pair<uint32_t, uint32_t>;

void upper_pairs(std::vector<Pair>& out, const std::vector<uint32_t>& b) {
  for (size_t i = 0; i < b.size(); ++i)
    for (size_t j = 0; j <= i; ++j) out.push_back(b[i] >= b[j] ? Pair(b[i], b[j]) : Pair(b[j], b[i]));
}
void cross_pairs(std::vector<Pair>& out, const std::vector<uint32_t>& a, const std::vector<uint32_t>& b) {
  for (uint32_t va : a)
    for (uint32_t vb : b) out.push_back(va >= vb ? Pair(va, vb) : Pair(vb, va));
}

void seed_input(Deps& d, size_t i, uint32_t input_idx) { d.row(i)[input_idx / 64] |= 1ull << (input_idx % 64); }

// Largest degree first; ties keep vertex order (a stable sort, like Rust's sort_by).
std::pair<std::vector<uint32_t>, uint32_t> distance1(const std::vector<std::vector<uint32_t>>& adj, size_t n) {
  std::vector<size_t> order(n);
  for (size_t i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return adj[b].size() < adj[a].size(); });
  std::vector<uint32_t> colors(n, kUnused);
  uint32_t num = 0;
  std::vector<uint32_t> used;
  for (size_t v : order) {
    uint64_t bits = 0;
    bool fallback = false;
    for (uint32_t u : adj[v]) {
      const uint32_t c = colors[u];
      if (c == kUnused) continue;
      if (c < 64) bits |= 1ull << c;
      else fallback = true;
    }
    uint32_t color;
    if (!fallback) {
      const uint64_t free_bits = ~bits;
      color = free_bits ? (uint32_t)__builtin_ctzll(free_bits) : 64u;
    } else {
      used.clear();
      for (uint32_t u : adj[v])
        if (colors[u] != kUnused) used.push_back(colors[u]);
      std::sort(used.begin(), used.end());
      used.erase(std::unique(used.begin(), used.end()), used.end());
      color = 0;
      for (uint32_t u : used) {
        if (u != color) break;
        ++color;
      }
    }
    colors[v] = color;
    num = std::max(num, color + 1);
  }
  return {colors, num};
}

std::pair<std::vector<uint32_t>, uint32_t> intersection(const uint32_t* group_keys, const uint32_t* color_keys,
                                                        size_t nnz, size_t group_dim, size_t color_dim) {
  if (color_dim == 0) return {{}, 0};
  std::vector<std::vector<uint32_t>> groups(group_dim);
  for (size_t k = 0; k < nnz; ++k) groups[group_keys[k]].push_back(color_keys[k]);
  std::vector<std::vector<uint32_t>> adj(color_dim);
  for (const auto& m : groups)
    for (size_t i = 0; i < m.size(); ++i)
      for (size_t j = i + 1; j < m.size(); ++j) {
        adj[m[i]].push_back(m[j]);
        adj[m[j]].push_back(m[i]);
      }
  for (auto& l : adj) {
    std::sort(l.begin(), l.end());
    l.erase(std::unique(l.begin(), l.end()), l.end());
  }
  return distance1(adj, color_dim);
}

ech_status copy_out(const std::vector<uint32_t>& v, uint32_t* out, size_t cap) {
  if (cap < v.size()) return ECH_ERR_INVALID_ARG;
  if (!v.empty()) std::memcpy(out, v.data(), v.size() * sizeof(uint32_t));
  return ECH_OK;
}

}  // namespace

extern "C" {

ECH_API ech_status ech_detect_hessian_sparsity(const uint32_t* op, const uint32_t* a0, const uint32_t* a1,
                                               uint32_t nv, uint32_t ni, uint32_t* rows, uint32_t* cols,
                                               size_t cap, size_t* nnz) {
  if ((nv && (!op || !a0 || !a1)) || !nnz) return ECH_ERR_INVALID_ARG;
  Deps d(nv, ni);
  std::vector<Pair> inter;
  uint32_t input_idx = 0;
  for (uint32_t i = 0; i < nv; ++i) {
    const uint32_t o = op[i];
    if (o == OP_INPUT) { seed_input(d, i, input_idx++); continue; }
    if (o == OP_CONST) continue;
    const uint32_t a = a0[i], b = a1[i];
    switch (classify(o)) {
      case OpClass::Linear:
      case OpClass::ZeroDerivative:
        d.unite(i, a);
        if (binary_op(o) && b != kUnused) d.unite(i, b);
        break;
      case OpClass::UnaryNonlinear:
        d.unite(i, a);
        upper_pairs(inter, d.extract(i, ni));
        break;
      case OpClass::BinaryNonlinear:
        if (o == OP_CUSTOM) {  // no second operand on device tapes: unary custom op
          d.unite(i, a);
          upper_pairs(inter, d.extract(i, ni));
        } else {
          const std::vector<uint32_t> ba = d.extract(a, ni), bb = d.extract(b, ni);
          d.unite(i, a);
          d.unite(i, b);
          cross_pairs(inter, ba, bb);
          if (o != OP_MUL) {
            upper_pairs(inter, ba);
            upper_pairs(inter, bb);
          }
        }
        break;
    }
  }
  std::sort(inter.begin(), inter.end());
  inter.erase(std::unique(inter.begin(), inter.end()), inter.end());
  *nnz = inter.size();
  if (!rows || !cols) return cap == 0 ? ECH_OK : ECH_ERR_INVALID_ARG;
  if (cap < inter.size()) return ECH_ERR_INVALID_ARG;
  for (size_t k = 0; k < inter.size(); ++k) {
    rows[k] = inter[k].first;
    cols[k] = inter[k].second;
  }
  return ECH_OK;
}

ECH_API ech_status ech_detect_jacobian_sparsity(const uint32_t* op, const uint32_t* a0, const uint32_t* a1,
                                                uint32_t nv, uint32_t ni, const uint32_t* outs, uint32_t nouts,
                                                uint32_t* rows, uint32_t* cols, size_t cap, size_t* nnz) {
  if ((nv && (!op || !a0 || !a1)) || (nouts && !outs) || !nnz) return ECH_ERR_INVALID_ARG;
  Deps d(nv, ni);
  uint32_t input_idx = 0;
  for (uint32_t i = 0; i < nv; ++i) {
    const uint32_t o = op[i];
    if (o == OP_INPUT) { seed_input(d, i, input_idx++); continue; }
    if (o == OP_CONST) continue;
    d.unite(i, a0[i]);
    if (o != OP_CUSTOM && binary_op(o) && a1[i] != kUnused) d.unite(i, a1[i]);
  }
  std::vector<uint32_t> r, c;
  for (uint32_t j = 0; j < nouts; ++j) {
    if (outs[j] >= nv) return ECH_ERR_INVALID_ARG;
    for (uint32_t col : d.extract(outs[j], ni)) {
      r.push_back(j);
      c.push_back(col);
    }
  }
  *nnz = r.size();
  if (!rows || !cols) return cap == 0 ? ECH_OK : ECH_ERR_INVALID_ARG;
  if (copy_out(r, rows, cap) != ECH_OK) return ECH_ERR_INVALID_ARG;
  return copy_out(c, cols, cap);
}

ECH_API ech_status ech_greedy_coloring(uint32_t dim, const uint32_t* rows, const uint32_t* cols, size_t nnz,
                                       uint32_t* colors, uint32_t* num_colors) {
  if ((nnz && (!rows || !cols)) || (dim && !colors) || !num_colors) return ECH_ERR_INVALID_ARG;
  if (dim == 0) { *num_colors = 0; return ECH_OK; }
  std::vector<std::vector<uint32_t>> adj(dim), adj2(dim);
  for (size_t k = 0; k < nnz; ++k) {
    if (rows[k] >= dim || cols[k] >= dim) return ECH_ERR_INVALID_ARG;
    if (rows[k] != cols[k]) {
      adj[rows[k]].push_back(cols[k]);
      adj[cols[k]].push_back(rows[k]);
    }
  }
  for (uint32_t v = 0; v < dim; ++v) {
    auto& l = adj2[v];
    for (uint32_t u : adj[v]) l.push_back(u);
    for (uint32_t u : adj[v])
      for (uint32_t w : adj[u])
        if (w != v) l.push_back(w);
    std::sort(l.begin(), l.end());
    l.erase(std::unique(l.begin(), l.end()), l.end());
  }
  auto res = distance1(adj2, dim);
  std::memcpy(colors, res.first.data(), dim * sizeof(uint32_t));
  *num_colors = res.second;
  return ECH_OK;
}

ECH_API ech_status ech_column_coloring(uint32_t num_outputs, uint32_t num_inputs, const uint32_t* rows,
                                       const uint32_t* cols, size_t nnz, uint32_t* colors, uint32_t* num_colors) {
  if ((nnz && (!rows || !cols)) || (num_inputs && !colors) || !num_colors) return ECH_ERR_INVALID_ARG;
  for (size_t k = 0; k < nnz; ++k)
    if (rows[k] >= num_outputs || cols[k] >= num_inputs) return ECH_ERR_INVALID_ARG;
  auto res = intersection(rows, cols, nnz, num_outputs, num_inputs);
  if (!res.first.empty()) std::memcpy(colors, res.first.data(), res.first.size() * sizeof(uint32_t));
  *num_colors = res.second;
  return ECH_OK;
}

ECH_API ech_status ech_row_coloring(uint32_t num_outputs, uint32_t num_inputs, const uint32_t* rows,
                                    const uint32_t* cols, size_t nnz, uint32_t* colors, uint32_t* num_colors) {
  if ((nnz && (!rows || !cols)) || (num_outputs && !colors) || !num_colors) return ECH_ERR_INVALID_ARG;
  for (size_t k = 0; k < nnz; ++k)
    if (rows[k] >= num_outputs || cols[k] >= num_inputs) return ECH_ERR_INVALID_ARG;
  auto res = intersection(cols, rows, nnz, num_inputs, num_outputs);
  if (!res.first.empty()) std::memcpy(colors, res.first.data(), res.first.size() * sizeof(uint32_t));
  *num_colors = res.second;
  return ECH_OK;
}

}  // extern "C"
