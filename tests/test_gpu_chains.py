"""Fused linear-combination chains on the GPU, bit for bit against the oracle.

A dot product ``s = b + c_1 x_{i_1} + ... + c_n x_{i_n}`` becomes one fused
chain instruction.  The forward sweep reads its terms in groups (several operand
loads in flight); the reverse sweep batches the terms' adjoint updates when the
chain's operands are pairwise distinct and falls back to one term at a time when
an operand repeats.  Lengths around the group sizes (1..33 terms), distinct and
repeated operands, and operands that also feed other ops cover both paths.  The
functions are polynomials, so with -fmad=false every result must equal the
oracle's exactly.
"""
import numpy as np
import pytest

from echidna_b200 import constant, record
from echidna_b200.gpu import GpuTapeData
from oracle.oracle import OracleTape

pytestmark = pytest.mark.gpu

LENGTHS = [1, 2, 3, 4, 5, 7, 8, 9, 12, 16, 17, 33]


def _chain_tape(n_inputs, idx, coef, extra):
    def f(v):
        s = constant(0.25)
        for i, c in zip(idx, coef):
            s = s + constant(float(c)) * v[i]
        r = s * s * constant(0.5)
        if extra:  # the inputs' adjoints also get contributions outside the chain
            r = r + v[0] * v[n_inputs - 1] + s * v[1 % n_inputs]
        return r
    return record(f, [0.1] * n_inputs)[0]


def _cases():
    rng = np.random.default_rng(5)
    for n in LENGTHS:
        coef = rng.normal(size=n)
        yield f"distinct{n}", n, list(range(n)), coef, False
        yield f"distinct{n}x", n, list(rng.permutation(n)), coef, True
        m = max(1, n // 3)
        yield f"repeat{n}", m, [k % m for k in range(n)], coef, True


CASES = list(_cases())


def _bits_equal(a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b).astype(a.dtype)
    u = np.uint32 if a.dtype == np.float32 else np.uint64
    both_nan = np.isnan(a) & np.isnan(b)
    return bool(((a.view(u) == b.view(u)) | both_nan).all())


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_linear_combination_chain_bit_exact(ctx, case):
    name, ni, idx, coef, extra = case
    tape = _chain_tape(ni, idx, coef, extra)
    o = OracleTape(tape)
    rng = np.random.default_rng(len(idx))
    B = 517
    X = rng.uniform(-2.0, 2.0, size=(B, ni))
    V = rng.choice([-1.0, 1.0], size=(B, ni))
    ov, og = o.gradient(X)
    ohg, ohh = o.hvp(X, V)
    gt = ctx.upload_tape_f64(tape)
    v, g = ctx.gradient_batch_f64(gt, X, B)
    assert _bits_equal(v, ov[:, 0]), name
    assert _bits_equal(g.reshape(B, ni), og), name
    hg, hh = ctx.hvp_batch_points_f64(gt, X, V, B)
    assert _bits_equal(hg.reshape(B, ni), ohg), name
    assert _bits_equal(hh.reshape(B, ni), ohh), name
    # f32: the engine against itself in f64-rounded-to-f32 is not exact, so
    # compare the f32 sweep with the oracle's f32 restatement
    o32 = OracleTape(tape, dtype=np.float32)
    X32 = X.astype(np.float32)
    V32 = V.astype(np.float32)
    g32t = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    v32, g32 = ctx.gradient_batch(g32t, X32, B)
    ov32, og32 = o32.gradient(X32)
    assert _bits_equal(v32, ov32[:, 0]), name
    assert _bits_equal(g32.reshape(B, ni), og32), name
    hg32, hh32 = ctx.hvp_batch_points(g32t, X32, V32, B)
    ohg32, ohh32 = o32.hvp(X32, V32)
    assert _bits_equal(hg32.reshape(B, ni), ohg32), name
    assert _bits_equal(hh32.reshape(B, ni), ohh32), name


@pytest.mark.parametrize("f64", [True, False])
def test_dense_layers_with_zero_weights_bit_exact(ctx, f64):
    # two dense layers whose reverses become gathers; a third of the weights
    # are zero (and some round to zero in f32), so contributions are left out
    rng = np.random.default_rng(13)
    n, w = 6, 5
    W1 = rng.normal(size=(w, n)) * (rng.random((w, n)) > 0.33)
    W1[0, 0] = 1e-60  # zero once rounded to f32
    W2 = rng.normal(size=(w, w)) * (rng.random((w, w)) > 0.33)

    def f(v):
        h = []
        for j in range(w):
            s = constant(0.1 * j)
            for i in range(n):
                s = s + constant(float(W1[j, i])) * v[i]
            h.append(s * s)
        out = constant(0.0)
        for j in range(w):
            s = constant(-0.2)
            for i in range(w):
                s = s + constant(float(W2[j, i])) * h[i]
            out = out + s * s
        return out
    tape = record(f, [0.1] * n)[0]
    X = rng.uniform(-1.0, 1.0, size=(300, n))
    V = rng.choice([-1.0, 1.0], size=(300, n))
    dt = np.float64 if f64 else np.float32
    o = OracleTape(tape, dtype=dt)
    gt = ctx.upload_tape_f64(tape) if f64 else ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    Xd, Vd = X.astype(dt), V.astype(dt)
    if f64:
        v, g = ctx.gradient_batch_f64(gt, Xd, 300)
        hg, hh = ctx.hvp_batch_points_f64(gt, Xd, Vd, 300)
    else:
        v, g = ctx.gradient_batch(gt, Xd, 300)
        hg, hh = ctx.hvp_batch_points(gt, Xd, Vd, 300)
    ov, og = o.gradient(Xd)
    ohg, ohh = o.hvp(Xd, Vd)
    assert _bits_equal(v, ov[:, 0])
    assert _bits_equal(g.reshape(300, n), og)
    assert _bits_equal(hg.reshape(300, n), ohg)
    assert _bits_equal(hh.reshape(300, n), ohh)
