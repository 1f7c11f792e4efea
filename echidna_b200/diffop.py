"""Differential operators and their sparse STDE sampling distributions (host side).

A restatement of the reference's operator algebra in ``src/diffop.rs``:

* ``MultiIndex`` (``diffop.rs:84-170``): per-variable differentiation orders.
* ``DiffOp`` (``diffop.rs:719-870``): ``L = sum_a C_a d^a`` with the named
  constructors ``laplacian``, ``biharmonic``, ``diagonal``, ``from_orders``.
* ``DiffOp.sparse_distribution`` (``diffop.rs:896-945``): per term, a
  collision-free assignment of jet slots (``plan_group``, ``diffop.rs:375-438``:
  primes from ``PRIMES``, highest-order variable on the smallest prime, the
  window shifted on a collision found by ``try_slots``, ``diffop.rs:310-372``),
  the output coefficient ``k = sum slot * order`` and the extraction prefactor
  ``prod q! (slot!)^q`` (``diffop.rs:222-255``).
* ``SparseSamplingDistribution`` (``diffop.rs:947-1045``): inverse-CDF
  ``sample_index`` over ``|C_a|``, normalisation ``Z = sum |C_a|``.

Arithmetic runs in the distribution's float type (``np.float64`` or
``np.float32``), in the reference's order, so the tables equal the reference's.
``stde_sparse`` / ``stde_sparse_batch`` run the estimator on the GPU through
``ech_stde_sparse_batch_*``.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass
from typing import List, Sequence, Tuple

import numpy as np

from . import _lib

PRIMES = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61, 67, 71)


class MultiIndex:
    """Per-variable differentiation orders (``src/diffop.rs:84-170``)."""

    def __init__(self, orders: Sequence[int]):
        if len(orders) == 0:
            raise ValueError("multi-index must have at least one variable")
        self._orders = tuple(int(o) for o in orders)

    @classmethod
    def diagonal(cls, num_vars: int, var: int, order: int) -> "MultiIndex":
        if var >= num_vars:
            raise ValueError(f"var ({var}) >= num_vars ({num_vars})")
        if order <= 0:
            raise ValueError("order must be > 0")
        o = [0] * num_vars
        o[var] = order
        return cls(o)

    @classmethod
    def partial(cls, num_vars: int, var: int) -> "MultiIndex":
        return cls.diagonal(num_vars, var, 1)

    def total_order(self) -> int:
        return sum(self._orders)

    def active_vars(self) -> List[Tuple[int, int]]:
        return [(i, o) for i, o in enumerate(self._orders) if o > 0]

    def active_var_set(self) -> List[int]:
        return [i for i, o in enumerate(self._orders) if o > 0]

    def num_vars(self) -> int:
        return len(self._orders)

    def orders(self) -> Tuple[int, ...]:
        return self._orders

    def __eq__(self, other):
        return isinstance(other, MultiIndex) and self._orders == other._orders

    def __repr__(self):
        return f"MultiIndex({list(self._orders)})"


def _factorial(n: int, ft):
    f = ft(1)
    for i in range(2, n + 1):
        f = ft(f * ft(i))
    return f


def partitions_with_support(k: int, slots: Sequence[int]) -> List[List[Tuple[int, int]]]:
    """Partitions of ``k`` into parts from ``slots`` as (slot, multiplicity)
    lists, in the reference's enumeration order (``diffop.rs:176-211``)."""
    results: List[List[Tuple[int, int]]] = []
    current: List[Tuple[int, int]] = []

    def rec(remaining, start):
        if remaining == 0:
            results.append(list(current))
            return
        for idx in range(start, len(slots)):
            s = slots[idx]
            if s > remaining:
                continue
            for mult in range(1, remaining // s + 1):
                current.append((s, mult))
                rec(remaining - s * mult, idx + 1)
                current.pop()

    rec(k, 0)
    return results


def extraction_prefactor(slot_orders: Sequence[Tuple[int, int]], ft) -> float:
    """``prod_t q_t! * (slot_t!)^q_t`` with the reference's log-domain fallback
    on overflow (``diffop.rs:222-255``)."""
    pref = ft(1)
    with np.errstate(over="ignore"):
        for slot, order in slot_orders:
            q_fact = _factorial(order, ft)
            j_fact = _factorial(slot, ft)
            j_pow = ft(1)
            for _ in range(order):
                j_pow = ft(j_pow * j_fact)
            pref = ft(ft(pref * q_fact) * j_pow)
        if np.isfinite(pref):
            return pref
        log_pref = ft(0)
        for slot, order in slot_orders:
            for i in range(2, order + 1):
                log_pref = ft(log_pref + ft(np.log(ft(i))))
            log_j = ft(0)
            for i in range(2, slot + 1):
                log_j = ft(log_j + ft(np.log(ft(i))))
            log_pref = ft(log_pref + ft(ft(order) * log_j))
        return ft(np.exp(log_pref))


def _try_slots(var_slot, members, ft):
    group_slots = [s for _, s in var_slot]
    extractions = []
    max_k = 0
    for result_index, mi in members:
        active = mi.active_vars()
        if not active:
            extractions.append((result_index, 0, ft(1)))
            continue
        slot_orders = [(dict(var_slot)[var], order) for var, order in active]
        k = sum(s * q for s, q in slot_orders)
        target = sorted(slot_orders)
        for p in partitions_with_support(k, group_slots):
            if sorted(p) != target:
                return None
        extractions.append((result_index, k, extraction_prefactor(slot_orders, ft)))
        max_k = max(max_k, k)
    return extractions, max_k


def plan_group(active_var_set: Sequence[int], members, ft):
    """Collision-free slot assignment for multi-indices sharing one active set
    (``diffop.rs:375-438``); returns (input_coeffs, extractions, jet_order)."""
    t = len(active_var_set)
    if t > len(PRIMES):
        raise ValueError(f"too many active variables ({t}) — max supported is {len(PRIMES)}")
    var_max = []
    for var in active_var_set:
        mo = max((mi.orders()[var] for _, mi in members), default=0)
        var_max.append((var, mo))
    var_max.sort(key=lambda vm: (-vm[1], vm[0]))
    for offset in range(len(PRIMES) - t + 1):
        var_slot = [(var, PRIMES[offset + i]) for i, (var, _) in enumerate(var_max)]
        got = _try_slots(var_slot, members, ft)
        if got is not None:
            extractions, max_k = got
            input_coeffs = [(var, slot, ft(ft(1) / _factorial(slot, ft))) for var, slot in var_slot]
            return input_coeffs, extractions, max_k + 1
    raise ValueError(f"failed to find collision-free slot assignment for active vars {list(active_var_set)}")


def _signum(c, ft):
    if np.isnan(c):
        return ft(np.nan)
    return ft(math.copysign(1.0, float(c)))


@dataclass
class SparseJetEntry:
    cumulative_weight: float
    input_coeffs: List[Tuple[int, int, float]]  # (var, slot, 1/slot!)
    output_coeff_index: int
    extraction_prefactor: float
    sign: float


class SparseSamplingDistribution:
    """Discrete distribution over sparse jets (``src/diffop.rs:947-1045``)."""

    def __init__(self, entries: List[SparseJetEntry], total_weight, ft):
        self.entries = entries
        self.total_weight = total_weight
        self.dtype = ft
        self._jet_order = max((e.output_coeff_index for e in entries), default=1)

    def sample_index(self, uniform_01) -> int:
        target = self.dtype(self.dtype(uniform_01) * self.total_weight)
        lo, hi = 0, len(self.entries)
        while lo < hi:  # first entry whose cumulative weight exceeds the target
            mid = (lo + hi) // 2
            if self.entries[mid].cumulative_weight <= target:
                lo = mid + 1
            else:
                hi = mid
        return min(lo, len(self.entries) - 1)

    def normalization(self):
        return self.total_weight

    def __len__(self):
        return len(self.entries)

    def is_empty(self) -> bool:
        return not self.entries

    def jet_order(self) -> int:
        return self._jet_order

    def entry(self, index: int) -> SparseJetEntry:
        return self.entries[index]

    def flatten(self):
        """The C ABI's tables: offsets, vars, slots, input coefficients,
        output coefficient indices, prefactors, signs (float arrays in the
        distribution's type)."""
        ft = self.dtype
        off = [0]
        vars_, slots, coeffs = [], [], []
        for e in self.entries:
            for var, slot, c in e.input_coeffs:
                vars_.append(var)
                slots.append(slot)
                coeffs.append(c)
            off.append(len(vars_))
        return (np.asarray(off, np.uint32), np.asarray(vars_, np.uint32), np.asarray(slots, np.uint32),
                np.asarray(coeffs, ft), np.asarray([e.output_coeff_index for e in self.entries], np.uint32),
                np.asarray([e.extraction_prefactor for e in self.entries], ft),
                np.asarray([e.sign for e in self.entries], ft))


class DiffOp:
    """``L = sum_a C_a d^a`` (``src/diffop.rs:719-870``)."""

    def __init__(self, num_vars: int, terms: Sequence[Tuple[float, MultiIndex]], dtype=np.float64):
        if len(terms) == 0:
            raise ValueError("DiffOp must have at least one term")
        for _, mi in terms:
            if mi.num_vars() != num_vars:
                raise ValueError(f"multi-index num_vars ({mi.num_vars()}) != expected ({num_vars})")
        self.dtype = dtype
        self._terms = [(dtype(c), mi) for c, mi in terms]
        self._num_vars = num_vars

    @classmethod
    def from_orders(cls, num_vars: int, terms: Sequence[Tuple[float, Sequence[int]]], dtype=np.float64):
        return cls(num_vars, [(c, MultiIndex(o)) for c, o in terms], dtype)

    @classmethod
    def laplacian(cls, n: int, dtype=np.float64):
        if n < 1:
            raise ValueError("laplacian requires at least one variable (n >= 1)")
        return cls(n, [(1.0, MultiIndex.diagonal(n, j, 2)) for j in range(n)], dtype)

    @classmethod
    def biharmonic(cls, n: int, dtype=np.float64):
        if n < 1:
            raise ValueError("biharmonic requires at least one variable (n >= 1)")
        two = dtype(dtype(1) + dtype(1))
        terms = [(1.0, MultiIndex.diagonal(n, j, 4)) for j in range(n)]
        for j in range(n):
            for k in range(j + 1, n):
                o = [0] * n
                o[j] = 2
                o[k] = 2
                terms.append((two, MultiIndex(o)))
        return cls(n, terms, dtype)

    @classmethod
    def diagonal(cls, n: int, k: int, dtype=np.float64):
        if n < 1:
            raise ValueError("diagonal requires at least one variable (n >= 1)")
        if k < 1:
            raise ValueError("diagonal order must be >= 1")
        return cls(n, [(1.0, MultiIndex.diagonal(n, j, k)) for j in range(n)], dtype)

    def terms(self):
        return list(self._terms)

    def num_vars(self) -> int:
        return self._num_vars

    def order(self) -> int:
        return max((mi.total_order() for _, mi in self._terms), default=0)

    def is_diagonal(self) -> bool:
        return all(len(mi.active_vars()) <= 1 for _, mi in self._terms)

    def split_by_order(self) -> List["DiffOp"]:
        groups: List[Tuple[int, list]] = []
        for c, mi in self._terms:
            o = mi.total_order()
            for g in groups:
                if g[0] == o:
                    g[1].append((c, mi))
                    break
            else:
                groups.append((o, [(c, mi)]))
        groups.sort(key=lambda g: g[0])
        return [DiffOp(self._num_vars, ts, self.dtype) for _, ts in groups]

    def sparse_distribution(self) -> SparseSamplingDistribution:
        """``DiffOp::sparse_distribution`` (``src/diffop.rs:896-945``); the
        operator must be homogeneous."""
        ft = self.dtype
        k = self._terms[0][1].total_order()
        for _, mi in self._terms:
            if mi.total_order() != k:
                raise ValueError(f"sparse_distribution requires homogeneous operator: found order {k} and order "
                                 f"{mi.total_order()}")
        entries = []
        cumulative = ft(0)
        for c, mi in self._terms:
            cumulative = ft(cumulative + ft(abs(c)))
            input_coeffs, extractions, _ = plan_group(mi.active_var_set(), [(0, mi)], ft)
            _, kout, pref = extractions[0]
            entries.append(SparseJetEntry(cumulative, input_coeffs, kout, pref, _signum(c, ft)))
        return SparseSamplingDistribution(entries, cumulative, ft)


# ── the estimator on the GPU ──

def stde_sparse_batch(backend, tape, xs, dist: SparseSamplingDistribution, sampled_indices):
    """``stde::stde_sparse`` (``src/stde/sparse.rs:37-78``) for every row of
    ``xs`` [B, n] with its own sampled entries ``sampled_indices`` [B, S], on
    the GPU (``ech_stde_sparse_batch_*``).  Returns a list of EstimatorResult."""
    from .gpu import _check
    from .stde_gpu import _result
    lib = _lib.load()
    f64 = bool(tape.f64)
    dt = np.float64 if f64 else np.float32
    xs = np.ascontiguousarray(xs, dtype=dt)
    if xs.ndim == 1:
        xs = xs[None, :]
    B = xs.shape[0]
    idx = np.ascontiguousarray(sampled_indices, dtype=np.uint64).reshape(B, -1)
    off, vars_, slots, coeffs, kout, pref, sign = dist.flatten()
    coeffs, pref, sign = (np.ascontiguousarray(a, dtype=dt) for a in (coeffs, pref, sign))
    res = (_lib.EstimatorResultC * B)()
    fn = lib.ech_stde_sparse_batch_f64 if f64 else lib.ech_stde_sparse_batch_f32
    z = ctypes.c_double(float(dist.normalization())) if f64 else ctypes.c_float(float(dist.normalization()))
    _check(fn(backend._h, tape._h, _lib.ptr(xs), xs.size, B, len(dist), _lib.ptr(off), _lib.ptr(vars_),
              _lib.ptr(slots), _lib.ptr(coeffs), _lib.ptr(kout), _lib.ptr(pref), _lib.ptr(sign), z, _lib.ptr(idx),
              idx.shape[1], res))
    return [_result(res[b], float) for b in range(B)]


def stde_sparse(backend, tape, x, dist: SparseSamplingDistribution, sampled_indices):
    """The reference call: one point, its sampled entry indices."""
    return stde_sparse_batch(backend, tape, np.asarray(x)[None, :], dist, np.asarray(sampled_indices)[None, :])[0]
