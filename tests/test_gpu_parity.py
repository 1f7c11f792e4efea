"""GPU parity against the oracle (the reference's CPU f64 tape, restated).

Mirrors the reference's tests/gpu_cpu_parity.rs (per-case ULP budgets, both-NaN
match, +-Inf exact) and tests/gpu_cuda_tests.rs (Rosenbrock grids, f64 rel 1e-10).
"""
import numpy as np
import pytest

from echidna_b200 import configs, record
from echidna_b200.gpu import GpuTapeData
from oracle.oracle import OracleTape
from tests.helpers import PARITY_CASES, rosenbrock_2, ulp_diff

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", PARITY_CASES, ids=[c[0] for c in PARITY_CASES])
def test_cuda_f64_parity(ctx, case):
    name, build, points, _f32_ulp, f64_ulp = case
    tape, _ = build()
    o = OracleTape(tape)
    gt = ctx.upload_tape_f64(tape)
    X = np.asarray(points, dtype=np.float64)
    cpu_val, cpu_grad = o.gradient(X)
    # one point per call (as the reference test) and the whole table in one batch
    for b in range(len(points)):
        val, grad = ctx.gradient_batch_f64(gt, X[b], 1)
        assert ulp_diff(val[0], cpu_val[b, 0]).max() <= f64_ulp, (name, b, val, cpu_val[b])
        assert ulp_diff(grad, cpu_grad[b]).max() <= f64_ulp, (name, b, grad, cpu_grad[b])
    val, grad = ctx.gradient_batch_f64(gt, X, len(points))
    assert ulp_diff(val, cpu_val[:, 0]).max() <= f64_ulp
    assert ulp_diff(grad.reshape(X.shape), cpu_grad).max() <= f64_ulp
    fwd = ctx.forward_batch_f64(gt, X, len(points))
    assert ulp_diff(fwd, cpu_val[:, 0]).max() <= f64_ulp


@pytest.mark.parametrize("case", PARITY_CASES, ids=[c[0] for c in PARITY_CASES])
def test_cuda_f32_parity(ctx, case):
    name, build, points, f32_ulp, _ = case
    tape, _ = build()
    o = OracleTape(tape)
    gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    X = np.asarray(points, dtype=np.float64)
    cpu_val, cpu_grad = o.gradient(X)
    for b in range(len(points)):
        val, grad = ctx.gradient_batch(gt, X[b].astype(np.float32), 1)
        assert ulp_diff(val[0], np.float32(cpu_val[b, 0]), np.float32).max() <= f32_ulp, (name, b, val, cpu_val[b])
        assert ulp_diff(grad, cpu_grad[b].astype(np.float32), np.float32).max() <= f32_ulp, (name, b, grad, cpu_grad[b])


def _approx(gpu, cpu, rel, abs_):
    gpu = np.asarray(gpu, dtype=np.float64)
    cpu = np.asarray(cpu, dtype=np.float64)
    diff = np.abs(gpu - cpu)
    return np.where(np.abs(cpu) < abs_, diff < abs_, diff / np.maximum(np.abs(cpu), 1e-300) < rel).all()


def test_rosenbrock_grid_f32_and_f64(ctx):
    # tests/gpu_cuda_tests.rs:50-222
    tape, _ = record(rosenbrock_2, [1.0, 2.0])
    o = OracleTape(tape)
    t = np.arange(100) / 99.0
    pts = np.stack([-2.0 + 4.0 * t, -1.0 + 3.0 * t], axis=1)
    cpu_v, cpu_g = o.gradient(pts)
    g32 = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    v32 = ctx.forward_batch(g32, pts.astype(np.float32), 100)
    assert _approx(v32, cpu_v[:, 0], 1e-5, 1e-6)
    _, gr32 = ctx.gradient_batch(g32, pts[:50].astype(np.float32), 50)
    assert _approx(gr32.reshape(50, 2), cpu_g[:50], 1e-4, 1e-3)
    g64 = ctx.upload_tape_f64(tape)
    v64 = ctx.forward_batch_f64(g64, pts[:50], 50)
    assert _approx(v64, cpu_v[:50, 0], 1e-10, 1e-12)
    _, gr64 = ctx.gradient_batch_f64(g64, pts[:50], 50)
    assert _approx(gr64.reshape(50, 2), cpu_g[:50], 1e-10, 1e-12)


@pytest.mark.parametrize("B", [1, 31, 129, 1000])
def test_rosenbrock_n100_gradient_f64(ctx, B):
    # extended Rosenbrock n=100, f64; U[-2, 2]^100 from a fixed seed
    tape = configs.rosenbrock(100)
    o = OracleTape(tape)
    rng = np.random.default_rng(configs.SEEDS["rosenbrock"])
    X = rng.uniform(-2.0, 2.0, size=(B, 100))
    cpu_v, cpu_g = o.gradient(X)
    gt = ctx.upload_tape_f64(tape)
    v, g = ctx.gradient_batch_f64(gt, X, B)
    # +,-,* only: bit-exact under -fmad=false
    np.testing.assert_array_equal(v, cpu_v[:, 0])
    np.testing.assert_array_equal(g.reshape(B, 100), cpu_g)


def test_mlp_gradient_and_hvp_f64(ctx):
    # the n=64 two-layer MLP tape at a reduced batch: f64 parity run
    tape = configs.mlp(64, 64)
    o = OracleTape(tape)
    rng = np.random.default_rng(configs.SEEDS["mlp"])
    B = 300
    X = rng.normal(size=(B, 64))
    V = rng.choice([-1.0, 1.0], size=(B, 64))
    cpu_v, cpu_g = o.gradient(X)
    gt = ctx.upload_tape_f64(tape)
    v, g = ctx.gradient_batch_f64(gt, X, B)
    assert ulp_diff(v, cpu_v[:, 0]).max() <= 64
    assert np.max(np.abs(g.reshape(B, 64) - cpu_g)) <= 1e-13 * max(1.0, np.abs(cpu_g).max())
    og, oh = o.hvp(X, V)
    hg, hh = ctx.hvp_batch_points_f64(gt, X, V, B)
    assert np.max(np.abs(hg.reshape(B, 64) - og)) <= 1e-13 * max(1.0, np.abs(og).max())
    assert np.max(np.abs(hh.reshape(B, 64) - oh)) <= 1e-12 * max(1.0, np.abs(oh).max())


def test_hvp_batch_single_x_f64(ctx):
    # hvp_batch: one x, B directions (src/gpu/cuda_backend.rs:234-304)
    tape = configs.random_dag(5, 400, seed=5)
    o = OracleTape(tape)
    rng = np.random.default_rng(0)
    x = rng.uniform(-1, 1, size=5)
    V = rng.normal(size=(17, 5))
    og, oh = o.hvp(np.tile(x, (17, 1)), V)
    gt = ctx.upload_tape_f64(tape)
    g, h = ctx.hvp_batch_f64(gt, x, V, 17)
    np.testing.assert_allclose(g.reshape(17, 5), og, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(h.reshape(17, 5), oh, rtol=1e-11, atol=1e-13)


def test_hessian_via_hvp_rosenbrock_analytic(ctx):
    # tests/hessian.rs:247-285: H = [[2-400y+1200x^2, -400x], [-400x, 200]] at (1.5, 2)
    tape, _ = record(rosenbrock_2, [1.5, 2.0])
    gt = ctx.upload_tape_f64(tape)
    x, y = 1.5, 2.0
    _, h = ctx.hvp_batch_f64(gt, [x, y], np.eye(2), 2)
    H = h.reshape(2, 2)
    np.testing.assert_allclose(H, [[2 - 400 * y + 1200 * x * x, -400 * x], [-400 * x, 200]], atol=1e-10)


def test_tangent_forward_matches_oracle_jvp(ctx):
    tape = configs.random_dag(4, 200, seed=9)
    o = OracleTape(tape)
    rng = np.random.default_rng(1)
    X = rng.uniform(-1, 1, size=(40, 4))
    V = rng.normal(size=(40, 4))
    ov, ot = o.jvp(X, V)
    gt = ctx.upload_tape_f64(tape)
    v, t = ctx.tangent_forward_batch_f64(gt, X, V, 40)
    np.testing.assert_allclose(v, ov[:, 0], rtol=1e-13)
    np.testing.assert_allclose(t, ot[:, 0], rtol=1e-12, atol=1e-14)
