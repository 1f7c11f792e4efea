"""Taylor jets and GPU STDE against the oracle and the reference's known answers
(tests/gpu_cuda_tests.rs:328-619, tests/stde_core.rs:61-112, tests/gpu_stde.rs)."""
import numpy as np
import pytest

from echidna_b200 import configs, record
from echidna_b200.gpu import GpuError, GpuTapeData
from echidna_b200 import stde_gpu
from oracle.oracle import OracleTape
from tests.helpers import rosenbrock_2

pytestmark = pytest.mark.gpu


def poly(v):
    return v[0] * v[0] + v[1] * v[1]


def test_taylor_kth_polynomial_all_orders(ctx):
    tape, _ = record(poly, [3.0, 4.0])
    gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    for order in range(1, 6):
        r = ctx.taylor_forward_kth_batch(gt, [3.0, 4.0], [1.0, 0.0], 1, order)
        assert r.order == order and len(r.coefficients) == order
        assert abs(r.coefficients[0][0] - 25.0) < 1e-3
        if order >= 2:
            assert abs(r.coefficients[1][0] - 6.0) < 1e-3
        if order >= 3:
            assert abs(r.coefficients[2][0] - 1.0) < 1e-3
        if order >= 4:
            assert abs(r.coefficients[3][0]) < 1e-3


def test_taylor_exp_higher_order(ctx):
    tape, _ = record(lambda v: v[0].exp(), [1.0])
    gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    r = ctx.taylor_forward_kth_batch(gt, [1.0], [1.0], 1, 5)
    e = np.e
    for k, want in enumerate([e, e, e / 2, e / 6, e / 24]):
        assert abs(r.coefficients[k][0] - want) < max(0.05 * want, 1e-2)


def test_taylor_unsupported_order(ctx):
    tape, _ = record(lambda v: v[0] * v[0], [1.0])
    gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    with pytest.raises(GpuError, match="unsupported Taylor order 6, must be 1..=5"):
        ctx.taylor_forward_kth_batch(gt, [1.0], [1.0], 1, 6)
    with pytest.raises(GpuError, match="unsupported Taylor order 0"):
        ctx.taylor_forward_kth_batch(gt, [1.0], [1.0], 1, 0)


def test_taylor_multi_batch(ctx):
    tape, _ = record(poly, [3.0, 4.0])
    gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    r = ctx.taylor_forward_kth_batch(gt, [3.0, 4.0, 3.0, 4.0], [1.0, 0.0, 0.0, 1.0], 2, 4)
    c = r.coefficients
    assert abs(c[0][0] - 25) < 1e-3 and abs(c[0][1] - 25) < 1e-3
    assert abs(c[1][0] - 6) < 1e-3 and abs(c[1][1] - 8) < 1e-3
    assert abs(c[2][0] - 1) < 1e-3 and abs(c[2][1] - 1) < 1e-3
    assert abs(c[3][0]) < 1e-3 and abs(c[3][1]) < 1e-3


def test_taylor_2nd_matches_kth(ctx):
    tape, _ = record(rosenbrock_2, [1.5, 2.5])
    gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    a = ctx.taylor_forward_2nd_batch(gt, [1.5, 2.5], [0.6, 0.8], 1)
    b = ctx.taylor_forward_kth_batch(gt, [1.5, 2.5], [0.6, 0.8], 1, 3)
    assert a.values[0] == b.coefficients[0][0] and a.c1s[0] == b.coefficients[1][0] and a.c2s[0] == b.coefficients[2][0]


@pytest.mark.parametrize("order", [1, 2, 3, 4, 5])
def test_taylor_f64_matches_oracle_on_dag(ctx, order):
    tape = configs.random_dag(6, 500, seed=order)
    o = OracleTape(tape)
    rng = np.random.default_rng(order)
    P = rng.uniform(-1, 1, size=(50, 6))
    S = rng.normal(size=(50, 6))
    ref = o.taylor(P, S, order)
    gt = ctx.upload_tape_f64(tape)
    r = ctx.taylor_forward_kth_batch_f64(gt, P, S, 50, order)
    got = np.stack(r.coefficients)
    np.testing.assert_allclose(got, ref, rtol=1e-11, atol=1e-12 * max(1.0, np.abs(ref).max()))


@pytest.mark.parametrize("fn", ["exp", "ln", "sqrt", "sin", "cos", "tan", "tanh", "atan", "asin", "acos",
                                "asinh", "acosh", "atanh", "sinh", "cosh", "cbrt", "exp2", "log2", "log10",
                                "ln_1p", "exp_m1", "abs", "recip"])
def test_taylor_k3_per_opcode_f32(ctx, fn):
    # tests/gpu_stde.rs:187-226: abs tol 1e-2, rel 1e-4 (c0, c1), 1e-3 (c2)
    x0 = {"acosh": 1.7, "asin": 0.3, "acos": 0.3, "atanh": 0.3, "ln": 1.3, "sqrt": 1.3, "log2": 1.3,
          "log10": 1.3}.get(fn, 0.7)
    tape, _ = record(lambda v: getattr(v[0], fn)(), [x0])
    o = OracleTape(tape)
    ref = o.taylor([[x0]], [[1.0]], 3)[:, 0]
    gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    r = ctx.taylor_forward_kth_batch(gt, [x0], [1.0], 1, 3)
    for k, rel in ((0, 1e-4), (1, 1e-4), (2, 1e-3)):
        got = float(r.coefficients[k][0])
        assert abs(got - ref[k]) <= max(1e-2 * 0 + rel * abs(ref[k]), 1e-5), (fn, k, got, ref[k])


def test_laplacian_gpu_known_answers(ctx):
    # tests/stde_core.rs:61-112 with the Rademacher enumeration
    sq, _ = record(lambda v: v[0] * v[0] + v[1] * v[1], [1.0, 2.0])
    gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(sq))
    r = stde_gpu.laplacian_gpu(ctx, gt, [1.0, 2.0], [[1.0, 1.0], [1.0, -1.0]])
    assert abs(r.value - 5.0) < 1e-5 and abs(r.estimate - 4.0) < 1e-5 and r.num_samples == 2
    cm, _ = record(lambda v: v[0] * v[0] * v[1] + v[1] * v[1] * v[1], [1.0, 2.0, 3.0])
    gt2 = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(cm))
    signs = [[a, b, c] for a in (1.0, -1.0) for b in (1.0, -1.0) for c in (1.0, -1.0)]
    r2 = stde_gpu.laplacian_gpu(ctx, gt2, [1.0, 2.0, 3.0], signs)
    assert abs(r2.value - 10.0) < 1e-4 and abs(r2.estimate - 16.0) < 1e-4
    v, d = stde_gpu.hessian_diagonal_gpu(ctx, gt, [1.0, 2.0])
    assert abs(v - 5.0) < 1e-5 and np.allclose(d, [2.0, 2.0])


def test_laplacian_gpu_matches_reference_welford_f32(ctx):
    # the drop-in reduces in f32 in direction order, like aggregate_laplacian
    tape = configs.random_dag(8, 400, seed=2, dtype=np.float32)
    gt = ctx.upload_tape(GpuTapeData.from_tape(tape))
    rng = np.random.default_rng(4)
    x = rng.uniform(-1, 1, 8).astype(np.float32)
    dirs = rng.choice([-1.0, 1.0], size=(33, 8)).astype(np.float32)
    r = stde_gpu.laplacian_gpu(ctx, gt, x, dirs)
    t2 = ctx.taylor_forward_2nd_batch(gt, np.tile(x, 33), dirs, 33)
    # host restatement of aggregate_laplacian in f32
    mean = np.float32(0); m2 = np.float32(0); n = 0
    for c2 in t2.c2s:
        s = np.float32(2.0) * c2
        if not np.isfinite(s):
            continue
        n += 1
        d = s - mean
        mean = np.float32(mean + d / np.float32(n))
        m2 = np.float32(m2 + d * (s - mean))
    assert r.num_samples == n and np.float32(r.estimate) == mean
    var = max(np.float32(m2 / np.float32(n - 1)), np.float32(0))
    assert np.float32(r.sample_variance) == var


def test_laplacian_with_control_gpu(ctx):
    tape, _ = record(lambda v: v[0] * v[0] * v[1] + v[1].sin() * v[2], [1.0, 2.0, 3.0])
    gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    o = OracleTape(tape)
    x = [0.3, -0.7, 1.1]
    _, diag = o.hessian_diagonal(x)
    rng = np.random.default_rng(8)
    dirs = rng.normal(size=(64, 3))
    ref = o.laplacian_with_control(x, dirs, diag)
    r = stde_gpu.laplacian_with_control_gpu(ctx, gt, x, dirs, diag)
    assert abs(r.estimate - ref[1]) < 1e-4 * max(1.0, abs(ref[1]))
    assert r.num_samples == 64


def test_laplacian_batch_host_directions_f64_exact(ctx):
    tape = configs.logsumexp_tanh(16, 32)
    o = OracleTape(tape)
    rng = np.random.default_rng(configs.SEEDS["logsumexp_tanh"])
    B, S = 20, 16
    X = rng.normal(size=(B, 16))
    D = rng.choice([-1.0, 1.0], size=(B, S, 16))
    ref = o.laplacian_stats_batch(X, D)
    gt = ctx.upload_tape_f64(tape)
    res = stde_gpu.laplacian_batch(ctx, gt, X, S, D, stde_gpu.DIR_PER_POINT)
    np.testing.assert_allclose(res["estimate"], ref[:, 1], rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(res["sample_variance"], ref[:, 2], rtol=1e-9, atol=1e-13)
    assert (res["num_samples"] == S).all()


def test_laplacian_batch_device_rng_statistics(ctx):
    # Rademacher directions from the device RNG: unbiased for tr(H); check against
    # the exact trace from the dense oracle Hessian with a z-test per point.
    tape = configs.logsumexp_tanh(16, 32)
    o = OracleTape(tape)
    rng = np.random.default_rng(5)
    X = rng.normal(size=(12, 16))
    gt = ctx.upload_tape_f64(tape)
    res = stde_gpu.laplacian_batch(ctx, gt, X, 4096, None, stde_gpu.DIR_RADEMACHER, seed=1234)
    for b in range(12):
        _, _, H = o.hessian(X[b])
        tr = np.trace(H)
        z = (res["estimate"][b] - tr) / max(res["standard_error"][b], 1e-300)
        assert abs(z) < 5.0, (b, res["estimate"][b], tr, res["standard_error"][b])


def test_taylor_2nd_chunked_matches_single_dispatch(ctx):
    # src/gpu/mod.rs:652-733: a buffer budget of 3 elements forces 4 chunks for 10 points
    tape, _ = record(rosenbrock_2, [1.0, 2.0])
    gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    rng = np.random.default_rng(11)
    P = rng.uniform(-1, 1, size=(10, 2)).astype(np.float32)
    S = rng.normal(size=(10, 2)).astype(np.float32)
    nv = len(tape.opcodes)
    whole = ctx.taylor_forward_2nd_batch(gt, P, S, 10)
    chunked = ctx.taylor_forward_2nd_batch_chunked(gt, P, S, 10, 2, nv, max_buffer_bytes=3 * nv * 12)
    for a, b in ((whole.values, chunked.values), (whole.c1s, chunked.c1s), (whole.c2s, chunked.c2s)):
        assert np.array_equal(a, b)
    with pytest.raises(GpuError, match="too small for a single element"):
        ctx.taylor_forward_2nd_batch_chunked(gt, P, S, 10, 2, nv, max_buffer_bytes=nv * 12 - 1)


@pytest.mark.parametrize("k", [2, 3, 4])
def test_diagonal_kth_order_stochastic_matches_oracle(ctx, k):
    # stde/higher_order.rs:173-227 on the GPU vs the oracle restatement, same sampled indices
    tape = configs.random_dag(8, 400, seed=20 + k)
    rng = np.random.default_rng(k)
    x = rng.uniform(-0.8, 0.8, size=8)
    idx = rng.integers(0, 8, size=12)
    gt = ctx.upload_tape_f64(tape)
    got = stde_gpu.diagonal_kth_order_stochastic_gpu(ctx, gt, x, k, idx)
    ref = OracleTape(tape).diagonal_kth_order_stochastic(x, k, idx)
    assert got.num_samples == int(ref[4])
    for j, key in enumerate(("value", "estimate", "sample_variance", "standard_error")):
        a, b = getattr(got, key), float(ref[j])
        assert abs(a - b) <= 1e-10 * max(1.0, abs(b)), (key, a, b)


def test_diagonal_kth_order_stochastic_errors(ctx):
    tape = configs.random_dag(4, 50, seed=1)
    gt = ctx.upload_tape_f64(tape)
    x = np.zeros(4)
    with pytest.raises(GpuError, match="sampled_indices must not be empty"):
        stde_gpu.diagonal_kth_order_stochastic_gpu(ctx, gt, x, 2, [])
    with pytest.raises(GpuError, match="k must be >= 2"):
        stde_gpu.diagonal_kth_order_stochastic_gpu(ctx, gt, x, 1, [0])
    with pytest.raises(GpuError, match="out of bounds"):
        stde_gpu.diagonal_kth_order_stochastic_gpu(ctx, gt, x, 2, [4])


@pytest.mark.parametrize("k", [2, 3, 5, 8])
def test_diagonal_kth_order_vector_matches_oracle(ctx, k):
    # stde/higher_order.rs:40-95 on the GPU (one launch over the n basis jets) vs
    # the oracle's single-index estimates n * k! * c_k
    tape = configs.random_dag(8, 400, seed=40 + k)
    x = np.random.default_rng(k).uniform(-0.8, 0.8, size=8)
    value, diag = stde_gpu.diagonal_kth_order_gpu(ctx, ctx.upload_tape_f64(tape), x, k)
    o = OracleTape(tape)
    for j in range(8):
        r = o.diagonal_kth_order_stochastic(x, k, [j])
        want = float(r[1]) / 8
        assert abs(diag[j] - want) <= 1e-10 * max(1.0, abs(want)), (j, diag[j], want)
        assert abs(value - float(r[0])) <= 1e-12 * max(1.0, abs(float(r[0])))
