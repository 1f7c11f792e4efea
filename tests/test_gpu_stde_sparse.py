"""Sparse STDE over differential operators on the GPU (``ech_stde_sparse_batch_*``)
against the oracle's restatement of ``stde::stde_sparse`` (src/stde/sparse.rs:37-78).

Operators cover every jet width the GPU path runs: first order (jets of order 3),
the Laplacian (5), mixed second partials (6), third-order diagonals (7) and
fourth-order diagonals (9).  Polynomial tapes must match the oracle bit for bit
(the jet arithmetic rounds like the CPU); tapes with transcendentals to a
relative 1e-12 (f64), since CUDA's and libm's functions may differ in the last
bits.
"""
import math

import numpy as np
import pytest

from echidna_b200 import configs, record
from echidna_b200.diffop import DiffOp, stde_sparse, stde_sparse_batch
from echidna_b200.gpu import GpuTapeData
from oracle.oracle import OracleTape

pytestmark = pytest.mark.gpu


def _poly(v):  # x^2 y + y^3 z + x z^4 - 2 x y z
    return v[0] * v[0] * v[1] + v[1] * v[1] * v[1] * v[2] + v[0] * v[2] * v[2] * v[2] * v[2] - v[0] * v[1] * v[2] * 2.0


def _quartic(v):
    return v[0] * v[0] * v[0] * v[0] + v[1] * v[1] * v[1] * v[1]


def _exp_plus_sin(v):
    return v[0].exp() + v[1].sin()


OPERATORS = {
    "first_order": lambda: DiffOp.from_orders(3, [(1.0, [1, 0, 0]), (-2.0, [0, 1, 0]), (0.5, [0, 0, 1])]),
    "laplacian": lambda: DiffOp.laplacian(3),
    "weighted_laplacian": lambda: DiffOp.from_orders(3, [(3.0, [2, 0, 0]), (1.0, [0, 2, 0]), (-0.5, [0, 0, 2])]),
    "mixed_second": lambda: DiffOp.from_orders(3, [(1.0, [1, 1, 0]), (2.0, [0, 1, 1]), (-1.0, [2, 0, 0])]),
    "third_diagonal": lambda: DiffOp.diagonal(3, 3),
    "fourth_diagonal": lambda: DiffOp.diagonal(3, 4),
}


def _bits_equal(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return bool(((a.view(np.uint64) == b.view(np.uint64)) | (np.isnan(a) & np.isnan(b))).all())


@pytest.mark.parametrize("name", list(OPERATORS))
def test_full_sample_matches_oracle_bit_for_bit(ctx, name):
    dist = OPERATORS[name]().sparse_distribution()
    tape, _ = record(_poly, [0.3, -0.7, 1.1])
    gt = ctx.upload_tape_f64(tape)
    o = OracleTape(tape)
    x = [0.3, -0.7, 1.1]
    idx = list(range(len(dist))) * 3
    r = stde_sparse(ctx, gt, x, dist, idx)
    want = o.stde_sparse(x, dist, idx)
    got = (r.value, r.estimate, r.sample_variance, r.standard_error)
    assert _bits_equal(got, want[:4]), (name, got, want)
    assert r.num_samples == want[4]


def test_fourth_order_diagonal_known_answer(ctx):
    # sum_j d^4/dx_j^4 (x^4 + y^4) = 48 (jets of order 9)
    tape, _ = record(_quartic, [2.0, 3.0])
    dist = DiffOp.diagonal(2, 4).sparse_distribution()
    r = stde_sparse(ctx, ctx.upload_tape_f64(tape), [2.0, 3.0], dist, range(len(dist)))
    assert abs(r.estimate - 48.0) < 1e-9 and r.num_samples == 2


def test_importance_sampled_mixed_operator(ctx):
    # L = d2/dx2 + 2 d2/dy2 on exp(x) + sin(y): samples drawn proportional to |C_a|
    x = [0.5, 1.0]
    tape, _ = record(_exp_plus_sin, x)
    dist = DiffOp.from_orders(2, [(1.0, [2, 0]), (2.0, [0, 2])]).sparse_distribution()
    idx = [dist.sample_index((((i * 2654435761) & 0xFFFFFFFFFFFFFFFF) % 100_000) / 100_000.0) for i in range(50_000)]
    r = stde_sparse(ctx, ctx.upload_tape_f64(tape), x, dist, idx)
    want = OracleTape(tape).stde_sparse(x, dist, idx)
    np.testing.assert_allclose([r.value, r.estimate, r.sample_variance, r.standard_error], want[:4], rtol=1e-12)
    expected = math.exp(0.5) - 2.0 * math.sin(1.0)
    assert abs(r.estimate - expected) < 3 * r.standard_error


@pytest.mark.parametrize("f64", [True, False])
def test_batch_of_points_each_with_its_samples(ctx, f64):
    tape = configs.random_dag(6, 400, seed=21)
    n = tape.num_inputs
    terms = [(1.0 + j, [2 if i == j else 0 for i in range(n)]) for j in range(n)]
    terms += [(-0.5, [1 if i in (0, n - 1) else 0 for i in range(n)])]
    dist = DiffOp.from_orders(n, terms, dtype=np.float64 if f64 else np.float32).sparse_distribution()
    rng = np.random.default_rng(8)
    B, S = 96, 37
    X = rng.uniform(-0.8, 0.8, size=(B, n))
    idx = np.array([[dist.sample_index(u) for u in rng.uniform(size=S)] for _ in range(B)], dtype=np.uint64)
    if f64:
        gt = ctx.upload_tape_f64(tape)
        o = OracleTape(tape)
    else:
        gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
        o = OracleTape(tape, dtype=np.float32)
        X = X.astype(np.float32)
    res = stde_sparse_batch(ctx, gt, X, dist, idx)
    rtol = 1e-11 if f64 else 2e-4
    for b in (0, 1, 17, B - 1):
        want = o.stde_sparse(X[b], dist, idx[b])
        got = [res[b].value, res[b].estimate, res[b].sample_variance, res[b].standard_error]
        scale = max(1.0, abs(want[1]), abs(want[2]))
        assert np.allclose(got, want[:4], rtol=rtol, atol=rtol * scale), (b, got, want)
        assert res[b].num_samples == want[4]


def test_errors(ctx):
    tape, _ = record(_quartic, [2.0, 3.0])
    gt = ctx.upload_tape_f64(tape)
    dist = DiffOp.laplacian(2).sparse_distribution()
    with pytest.raises(Exception, match="sampled_indices must not be empty"):
        stde_sparse_batch(ctx, gt, np.zeros((1, 2)), dist, np.zeros((1, 0), np.uint64))
    with pytest.raises(Exception, match="out of bounds"):
        stde_sparse(ctx, gt, [1.0, 2.0], dist, [0, 5])
    # d^4/dx^2 dy^2 needs output coefficient 16: beyond the GPU jets
    with pytest.raises(Exception, match="exceeds the GPU jets"):
        stde_sparse(ctx, gt, [1.0, 2.0], DiffOp.from_orders(2, [(1.0, [2, 2])]).sparse_distribution(), [0])
