"""Linear-combination chains in jet sweeps, bit for bit.

A dense layer ``z_j = b_j + sum_i W_ji x_i`` becomes one linear-combination
chain.  In a jet sweep each term is a constant times a jet, which the reference
evaluates as the truncated Cauchy product of the constant jet (c, 0, ..) with x;
the kernels scale instead and track non-finite lower coefficients, and when the
chain's operands are inputs of a point-direction launch (shared host
directions, device Rademacher signs, basis vectors) they read each input jet at
its source instead of from a slot.  Every result must equal the per-op product:

* Taylor jets of order 1..5 of polynomial tapes against the oracle (f64 and
  f32), with -0, inf and NaN among the inputs and directions;
* Laplacian estimates with shared directions and with device Rademacher
  directions against the same directions passed per unit (the slot path), the
  device stream reproduced on the host with Philox-4x32-10;
* Hessian diagonals (basis directions) against the oracle.
"""
import numpy as np
import pytest

from echidna_b200 import constant, record
from echidna_b200.gpu import GpuTapeData
from echidna_b200.stde_gpu import DIR_PER_POINT, DIR_RADEMACHER, DIR_SHARED, laplacian_batch
from oracle.oracle import OracleTape
from tests.helpers import philox_bits

pytestmark = pytest.mark.gpu


def _layer_tape(n, m, seed, mixed):
    """0.5 sum_j z_j^2 (+ sum_j z_j x_j x_{j+1} when mixed: inputs used outside
    the chains too) with z = W x + b; a polynomial, so every sweep is exact."""
    rng = np.random.default_rng(seed)
    W = rng.normal(size=(m, n))
    W[0, 0] = 0.0
    W[1 % m, n - 1] = -0.0
    b = rng.normal(size=m)

    def f(x):
        s = constant(0.0)
        for j in range(m):
            z = constant(float(b[j]))
            for i in range(n):
                z = z + float(W[j, i]) * x[i]
            s = s + z * z
            if mixed:
                s = s + z * x[j % n] * x[(j + 1) % n]
        return 0.5 * s
    return record(f, [0.1] * n)[0]


def _bits_equal(a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b).astype(a.dtype)
    u = np.uint32 if a.dtype == np.float32 else np.uint64
    both_nan = np.isnan(a) & np.isnan(b)
    return bool(((a.view(u) == b.view(u)) | both_nan).all())


def _special_rows(X, V):
    X[0, 0], V[0, 1] = -0.0, -0.0
    X[1, 2] = np.inf
    X[2, 1] = np.nan
    V[3, 0] = np.inf
    V[4, 3] = np.nan
    X[5, :] = 0.0
    V[5, :] = -0.0


@pytest.mark.parametrize("f64", [True, False])
@pytest.mark.parametrize("mixed", [False, True])
def test_taylor_jets_of_dense_layers_bit_exact(ctx, f64, mixed):
    n, m, B = 7, 5, 300
    tape = _layer_tape(n, m, 3, mixed)
    dt = np.float64 if f64 else np.float32
    rng = np.random.default_rng(4)
    X = rng.uniform(-2, 2, size=(B, n)).astype(dt)
    V = rng.normal(size=(B, n)).astype(dt)
    _special_rows(X, V)
    o = OracleTape(tape, dtype=dt)
    gt = ctx.upload_tape_f64(tape) if f64 else ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    fn = ctx.taylor_forward_kth_batch_f64 if f64 else ctx.taylor_forward_kth_batch
    for order in range(1, 6):
        r = fn(gt, X, V, B, order)
        oc = o.taylor(X, V, order)
        for k in range(order):
            assert _bits_equal(r.coefficients[k], oc[k]), (order, k)


def _stats(r):
    return np.stack([r["value"], r["estimate"], r["sample_variance"], r["standard_error"]], axis=1), r["num_samples"]


@pytest.mark.parametrize("f64", [True, False])
def test_laplacian_shared_directions_equal_per_unit(ctx, f64):
    n, m, B, S = 40, 24, 150, 16
    tape = _layer_tape(n, m, 5, True)
    dt = np.float64 if f64 else np.float32
    rng = np.random.default_rng(6)
    X = rng.normal(size=(B, n)).astype(dt)
    D = rng.normal(size=(S, n)).astype(dt)
    X[3, 4] = np.inf
    D[2, 7] = np.nan
    gt = ctx.upload_tape_f64(tape) if f64 else ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    shared = laplacian_batch(ctx, gt, X, S, D, DIR_SHARED)
    per_unit = laplacian_batch(ctx, gt, X, S, np.ascontiguousarray(np.broadcast_to(D, (B, S, n))), DIR_PER_POINT)
    a, na = _stats(shared)
    b, nb = _stats(per_unit)
    assert _bits_equal(a, b)
    assert np.array_equal(na, nb)


@pytest.mark.parametrize("f64", [True, False])
@pytest.mark.parametrize("n", [33, 64, 100])
def test_laplacian_device_rademacher_equals_host_replay(ctx, f64, n):
    # the device stream: sign of input i of direction s at point p is bit 0 of
    # philox_bits(seed, p, s, i) (1 -> +1, 0 -> -1)
    m, B, S, seed = 12, 70, 8, 0x5EED1234ABCD
    tape = _layer_tape(n, m, 7, True)
    dt = np.float64 if f64 else np.float32
    X = np.random.default_rng(8).normal(size=(B, n)).astype(dt)
    gt = ctx.upload_tape_f64(tape) if f64 else ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    dev = laplacian_batch(ctx, gt, X, S, None, DIR_RADEMACHER, seed=seed)
    p = np.arange(B, dtype=np.uint64)[:, None, None]
    s = np.arange(S, dtype=np.uint64)[None, :, None]
    i = np.arange(n, dtype=np.uint64)[None, None, :]
    bits = philox_bits(seed, p, s, i)
    D = np.where(bits & 1, 1.0, -1.0).astype(dt)
    host = laplacian_batch(ctx, gt, X, S, np.ascontiguousarray(D), DIR_PER_POINT)
    a, na = _stats(dev)
    b, nb = _stats(host)
    assert _bits_equal(a, b)
    assert np.array_equal(na, nb)


@pytest.mark.parametrize("f64", [True, False])
def test_hessian_diagonal_basis_directions_bit_exact(ctx, f64):
    torch = pytest.importorskip("torch")
    from echidna_b200.learned import hessian_diagonals
    n, m, B = 20, 9, 64
    tape = _layer_tape(n, m, 9, True)
    dt = np.float64 if f64 else np.float32
    X = np.random.default_rng(10).normal(size=(B, n)).astype(dt)
    gt = ctx.upload_tape_f64(tape) if f64 else ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    d = hessian_diagonals(ctx, gt, torch.tensor(X, device="cuda")).cpu().numpy()
    o = OracleTape(tape, dtype=dt)
    # diag_j = 2 * c2 of the jet along e_j (stde_gpu.rs:103-129)
    E = np.eye(n, dtype=dt)
    for b in range(B):
        c = o.taylor(np.tile(X[b], (n, 1)), E, 3)
        assert _bits_equal(d[b], (dt(2) * c[2]).astype(dt)), b


@pytest.mark.parametrize("f64", [True, False])
@pytest.mark.parametrize("mode", ["shared", "rademacher", "basis"])
@pytest.mark.parametrize("S", [16, 15])
def test_two_units_per_thread_equal_one(ctx, f64, mode, S):
    # point-direction launches at two units per thread (both directions of one
    # point when S is even, of two points across a thread when S is odd) equal
    # one unit per thread bit for bit, and the per-unit slot path
    torch = pytest.importorskip("torch")
    from echidna_b200.learned import hessian_diagonals
    n, m, B, seed = 40, 24, 150, 0x5EED
    tape = _layer_tape(n, m, 11, True)
    dt = np.float64 if f64 else np.float32
    rng = np.random.default_rng(12)
    X = rng.normal(size=(B, n)).astype(dt)
    X[3, 4] = np.inf
    X[7, 0] = np.nan
    D = rng.normal(size=(S, n)).astype(dt)
    gt = ctx.upload_tape_f64(tape) if f64 else ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))

    def run(ppt):
        ctx.set_launch(128, ppt, 0)
        try:
            if mode == "shared":
                return _stats(laplacian_batch(ctx, gt, X, S, D, DIR_SHARED))
            if mode == "rademacher":
                return _stats(laplacian_batch(ctx, gt, X, S, None, DIR_RADEMACHER, seed=seed))
            d = hessian_diagonals(ctx, gt, torch.tensor(X, device="cuda")).cpu().numpy()
            return d, None
        finally:
            ctx.set_launch(0, 0, 0)
            ctx.set_autotune(True)

    a, na = run(2)
    b, nb = run(1)
    assert _bits_equal(a, b), (mode, S)
    if na is not None:
        assert np.array_equal(na, nb)
    if mode == "shared":
        # and the per-unit slot path (no input-direct terms)
        c, nc = _stats(laplacian_batch(ctx, gt, X, S, np.ascontiguousarray(np.broadcast_to(D, (B, S, n))),
                                       DIR_PER_POINT))
        assert _bits_equal(a, c)


@pytest.mark.parametrize("f64", [True, False])
@pytest.mark.parametrize("mode", ["shared", "rademacher", "basis"])
def test_warps_of_one_point_share_coefficient_zero(ctx, f64, mode):
    # S a multiple of 32 at one unit per thread: every warp's units are directions
    # of one point, and the dense groups accumulate coefficient 0 one output per
    # lane, broadcast by shuffles.  Results equal the per-unit slot path (no
    # input-direct terms) or the oracle bit for bit, with inf and NaN inputs.
    torch = pytest.importorskip("torch")
    from echidna_b200.learned import hessian_diagonals
    n = 64 if mode == "basis" else 40
    m, B, S, seed = 40, 70, 64, 0x5EED77
    tape = _layer_tape(n, m, 13, True)
    dt = np.float64 if f64 else np.float32
    rng = np.random.default_rng(14)
    X = rng.normal(size=(B, n)).astype(dt)
    X[3, 4] = np.inf
    X[7, 0] = np.nan
    gt = ctx.upload_tape_f64(tape) if f64 else ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    ctx.set_launch(128, 1, 0)
    try:
        if mode == "basis":
            d = hessian_diagonals(ctx, gt, torch.tensor(X, device="cuda")).cpu().numpy()
            o = OracleTape(tape, dtype=dt)
            E = np.eye(n, dtype=dt)
            for b in (0, 3, 7, 40, 69):
                c = o.taylor(np.tile(X[b], (n, 1)), E, 3)
                assert _bits_equal(d[b], (dt(2) * c[2]).astype(dt)), b
            return
        if mode == "shared":
            D = rng.normal(size=(S, n)).astype(dt)
            a, na = _stats(laplacian_batch(ctx, gt, X, S, D, DIR_SHARED))
            per_unit = np.ascontiguousarray(np.broadcast_to(D, (B, S, n)))
        else:
            a, na = _stats(laplacian_batch(ctx, gt, X, S, None, DIR_RADEMACHER, seed=seed))
            p = np.arange(B, dtype=np.uint64)[:, None, None]
            s = np.arange(S, dtype=np.uint64)[None, :, None]
            i = np.arange(n, dtype=np.uint64)[None, None, :]
            per_unit = np.ascontiguousarray(np.where(philox_bits(seed, p, s, i) & 1, 1.0, -1.0).astype(dt))
        b, nb = _stats(laplacian_batch(ctx, gt, X, S, per_unit, DIR_PER_POINT))
        assert _bits_equal(a, b)
        assert np.array_equal(na, nb)
    finally:
        ctx.set_launch(0, 0, 0)
        ctx.set_autotune(True)
