"""Differential operators and sparse STDE sampling distributions, on the CPU.

The distribution tables (``echidna_b200.diffop``) are checked against the known
answers of the reference's tests (tests/diffop.rs: weights, normalisation and
inverse-CDF sampling; tests/stde_dense.rs: sparse STDE on polynomial and
exp + sin tapes), the slot plans against the construction in src/diffop.rs,
and the oracle's ``stde_sparse`` restatement against exact operator values.
"""
import math

import numpy as np
import pytest

from echidna_b200 import record
from echidna_b200.diffop import DiffOp, MultiIndex, extraction_prefactor, partitions_with_support
from oracle.oracle import OracleTape


def _sum_of_squares(v):
    return v[0] * v[0] + v[1] * v[1]


def _cubic_mix(v):  # x^2 y + y^3 (third input unused)
    return v[0] * v[0] * v[1] + v[1] * v[1] * v[1]


def _quartic(v):
    return v[0] * v[0] * v[0] * v[0] + v[1] * v[1] * v[1] * v[1]


def _exp_plus_sin(v):
    return v[0].exp() + v[1].sin()


def test_laplacian_weights_and_normalisation():
    dist = DiffOp.laplacian(3).sparse_distribution()
    assert len(dist) == 3
    assert dist.normalization() == 3.0


def test_inverse_cdf_sampling():
    dist = DiffOp.laplacian(3).sparse_distribution()
    assert dist.sample_index(0.0) == 0
    assert dist.sample_index(0.99) == 2
    assert dist.sample_index(0.5) == 1
    assert dist.sample_index(1.0) == 2  # clamped into range
    d4 = DiffOp.laplacian(4).sparse_distribution()
    assert d4.normalization() == 4.0
    assert [d4.sample_index(u) for u in (0.1, 0.3, 0.6, 0.9)] == [0, 1, 2, 3]


def test_nonuniform_weights():
    dist = DiffOp.from_orders(2, [(3.0, [2, 0]), (1.0, [0, 2])]).sparse_distribution()
    assert len(dist) == 2 and dist.normalization() == 4.0
    assert [dist.sample_index(u) for u in (0.0, 0.7, 0.8, 0.99)] == [0, 0, 1, 1]


def test_slot_plans():
    # a pure second derivative: slot 2, coefficient 1/2!, c_4 * 2! (2!)^2 = d^2
    e = DiffOp.laplacian(2).sparse_distribution().entry(1)
    assert e.input_coeffs == [(1, 2, 0.5)] and e.output_coeff_index == 4 and e.extraction_prefactor == 8.0
    # a mixed partial d^2/dx dy: slots 2 and 3, k = 5, prefactor 2! * 3! = 12
    e = DiffOp.from_orders(2, [(1.0, [1, 1])]).sparse_distribution().entry(0)
    assert [(v, s) for v, s, _ in e.input_coeffs] == [(0, 2), (1, 3)]
    assert e.output_coeff_index == 5 and e.extraction_prefactor == 12.0
    # d^4/dx^2 dy^2: slots (2, 3) collide (10 = 2*5), the next window (3, 5) does not: k = 16
    e = DiffOp.from_orders(2, [(2.0, [2, 2])]).sparse_distribution().entry(0)
    assert [(v, s) for v, s, _ in e.input_coeffs] == [(0, 3), (1, 5)]
    assert e.output_coeff_index == 16
    assert e.extraction_prefactor == 2.0 * 6.0 ** 2 * 2.0 * 120.0 ** 2
    # a negative coefficient carries its sign; Z sums magnitudes
    d = DiffOp.from_orders(2, [(-2.0, [2, 0]), (1.0, [0, 2])]).sparse_distribution()
    assert d.entry(0).sign == -1.0 and d.entry(1).sign == 1.0 and d.normalization() == 3.0


def test_partitions_and_prefactor_helpers():
    assert partitions_with_support(5, [2, 3]) == [[(2, 1), (3, 1)]]
    assert sorted(map(sorted, partitions_with_support(10, [2, 3]))) == [[(2, 2), (3, 2)], [(2, 5)]]
    assert extraction_prefactor([(2, 2)], np.float64) == 8.0
    assert extraction_prefactor([(5, 3)], np.float32) == np.float32(6.0 * 120.0 ** 3)


def test_operator_constructors():
    b = DiffOp.biharmonic(3)
    assert len(b.terms()) == 3 + 3 and b.order() == 4 and not b.is_diagonal()
    assert DiffOp.diagonal(4, 3).is_diagonal()
    mixed = DiffOp.from_orders(2, [(1.0, [2, 0]), (1.0, [1, 0])])
    parts = mixed.split_by_order()
    assert [p.order() for p in parts] == [1, 2]
    with pytest.raises(ValueError, match="homogeneous"):
        mixed.sparse_distribution()
    with pytest.raises(ValueError):
        MultiIndex([])


def test_oracle_full_sample_matches_exact():
    tape, _ = record(_sum_of_squares, [1.0, 2.0])
    dist = DiffOp.laplacian(2).sparse_distribution()
    v, est, var, se, n = OracleTape(tape).stde_sparse([1.0, 2.0], dist, range(len(dist)))
    assert n == 2 and abs(est - 4.0) < 1e-12 and v == 5.0


def test_oracle_laplacian_convergence():
    tape, _ = record(_cubic_mix, [1.0, 2.0, 3.0])
    dist = DiffOp.laplacian(3).sparse_distribution()
    idx = [dist.sample_index(((i * 2654435761) % 1000) / 1000.0) for i in range(1000)]
    _, est, _, se, _ = OracleTape(tape).stde_sparse([1.0, 2.0, 3.0], dist, idx)
    assert abs(est - 16.0) < max(3 * se, 1.0)


def test_oracle_diagonal_fourth_order():
    tape, _ = record(_quartic, [2.0, 3.0])
    dist = DiffOp.diagonal(2, 4).sparse_distribution()
    assert dist.jet_order() == 8
    _, est, _, _, _ = OracleTape(tape).stde_sparse([2.0, 3.0], dist, range(len(dist)))
    assert abs(est - 48.0) < 1e-4


def test_oracle_mixed_second_order_needs_importance_sampling():
    x = [0.5, 1.0]
    tape, _ = record(_exp_plus_sin, x)
    expected = math.exp(0.5) - 2.0 * math.sin(1.0)
    dist = DiffOp.from_orders(2, [(1.0, [2, 0]), (2.0, [0, 2])]).sparse_distribution()
    o = OracleTape(tape)
    _, uniform, _, _, _ = o.stde_sparse(x, dist, range(len(dist)))
    assert abs(uniform - expected) > 1.0  # enumeration is biased for unequal |C_a|
    idx = [dist.sample_index((((i * 2654435761) & 0xFFFFFFFFFFFFFFFF) % 100_000) / 100_000.0) for i in range(50_000)]
    _, est, _, se, _ = o.stde_sparse(x, dist, idx)
    assert abs(est - expected) < 3 * se
