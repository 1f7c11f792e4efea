"""Operator estimators on GPU jets (src/stde/laplacian.rs:252-344, src/stde/pde.rs)
checked against closed forms from the oracle's dense Hessian / Jacobian."""
import numpy as np
import pytest

from echidna_b200 import configs, record_multi, stde_gpu
from echidna_b200.gpu import GpuError
from oracle.oracle import OracleTape

pytestmark = pytest.mark.gpu


def _setup(n=12, seed=0):
    tape = configs.random_dag(n, 400, seed=seed)
    rng = np.random.default_rng(seed)
    x = rng.uniform(-0.7, 0.7, size=n)
    H = OracleTape(tape).hessian(x)[2]
    return tape, x, H, rng


def test_hutchpp_full_sketch_is_exact(ctx):
    # tests/stde_core.rs-style closed form: a sketch of rank n spans R^n, so the
    # exact part is tr(H) and the projected residual directions vanish
    tape, x, H, rng = _setup()
    gt = ctx.upload_tape_f64(tape)
    n = len(x)
    S = rng.normal(size=(n, n))
    G = rng.choice([-1.0, 1.0], size=(8, n))
    r = stde_gpu.laplacian_hutchpp_gpu(ctx, gt, x, S, G)
    assert abs(r.estimate - np.trace(H)) <= 1e-9 * max(1.0, np.abs(H).sum())
    assert r.num_samples == 8


def test_hutchpp_partial_sketch_unbiased_residual(ctx):
    tape, x, H, rng = _setup(seed=1)
    gt = ctx.upload_tape_f64(tape)
    n = len(x)
    S = rng.normal(size=(3, n))
    G = rng.choice([-1.0, 1.0], size=(4000, n))
    r = stde_gpu.laplacian_hutchpp_gpu(ctx, gt, x, S, G)
    assert abs(r.estimate - np.trace(H)) <= 5 * r.standard_error + 1e-9


def test_parabolic_diffusion_matches_dense(ctx):
    tape, x, H, rng = _setup(seed=2)
    gt = ctx.upload_tape_f64(tape)
    sig = rng.normal(size=(5, len(x)))
    v, e = stde_gpu.parabolic_diffusion_gpu(ctx, gt, x, sig)
    ref = 0.5 * sum(s @ H @ s for s in sig)
    assert abs(e - ref) <= 1e-10 * max(1.0, abs(ref))
    r = stde_gpu.parabolic_diffusion_stochastic_gpu(ctx, gt, x, sig, [0, 1, 2, 3, 4])
    assert abs(r.estimate - ref) <= 1e-10 * max(1.0, abs(ref))
    with pytest.raises(GpuError, match="out of bounds"):
        stde_gpu.parabolic_diffusion_stochastic_gpu(ctx, gt, x, sig, [5])


def test_dense_stde_2nd_matches_dense(ctx):
    tape, x, H, rng = _setup(seed=3)
    gt = ctx.upload_tape_f64(tape)
    n = len(x)
    L = np.tril(rng.normal(size=(n, n)))
    Z = rng.normal(size=(16, n))
    r = stde_gpu.dense_stde_2nd_gpu(ctx, gt, x, L, Z)
    samples = np.array([(L @ z) @ H @ (L @ z) for z in Z])
    assert abs(r.estimate - samples.mean()) <= 1e-9 * max(1.0, np.abs(samples).max())
    assert abs(r.sample_variance - samples.var(ddof=1)) <= 1e-7 * max(1.0, samples.var())


def test_divergence_matches_jacobian_trace_samples(ctx):
    f = lambda v: [v[0] * v[1], v[1].sin() + v[2], v[0] * v[2].exp()]  # noqa: E731
    tape, _ = record_multi(f, [0.3, -0.2, 0.5])
    gt = ctx.upload_tape_f64(tape)
    x = np.array([0.3, -0.2, 0.5])
    V = np.random.default_rng(4).choice([-1.0, 1.0], size=(32, 3))
    vals, r = stde_gpu.divergence_gpu(ctx, gt, x, V)
    o = OracleTape(tape)
    J = np.stack([o.jvp(x[None], np.eye(3)[k][None])[1][0] for k in range(3)], axis=1)
    samples = np.array([v @ J @ v for v in V])
    assert abs(r.estimate - samples.mean()) <= 1e-12 * max(1.0, np.abs(samples).max())
    assert np.allclose(vals, o.forward(x[None])[0], rtol=1e-15)
