"""Known answers from the reference's own tests, checked on the oracle (CPU)
and on the engine (GPU-marked copies of the same cases).

Each case cites the reference test it transcribes.  The oracle cases pin the
CPU restatement; the GPU cases show the sweeps keep the same conventions.
"""
import math

import numpy as np
import pytest

from echidna_b200 import record
from echidna_b200.gpu import GpuTapeData
from oracle.oracle import OracleTape

INF = math.inf


def _rec(fn, x0):
    return record(fn, list(x0))[0]


# (name, recorder, record point, eval point, per-component check of the gradient)
#  check: float -> exact value; "inf" / "+inf" / "nan" / ("approx", v, tol)
GRAD_CASES = [
    # tests/zero_multiplier_convention.rs:16-41
    ("hypot_origin", lambda v: v[0].hypot(v[1]).sqrt(), (3.0, 4.0), (0.0, 0.0), [0.0, 0.0]),
    ("hypot_replay", lambda v: v[0].hypot(v[1]).sqrt(), (3.0, 4.0), (3.0, 4.0),
     [("approx", (3.0 / 5.0) * 0.5 / math.sqrt(5.0), 1e-12), ("approx", (4.0 / 5.0) * 0.5 / math.sqrt(5.0), 1e-12)]),
    # tests/zero_multiplier_convention.rs:43-49
    ("atan2_origin", lambda v: v[0].atan2(v[1]).sqrt(), (3.0, 4.0), (0.0, 0.0), [0.0, 0.0]),
    # tests/zero_multiplier_convention.rs:53-70
    ("max_loser", lambda v: (v[0].max(v[1]) - 4.0).sqrt(), (5.0, 1.0), (4.0, 1.0), ["inf", 0.0]),
    # tests/zero_multiplier_convention.rs:72-82
    ("mul_zero", lambda v: (v[0] * v[1]).sqrt(), (2.0, 3.0), (5.0, 0.0), [0.0, "inf"]),
    # tests/zero_multiplier_convention.rs:86-94
    ("nan_partial", lambda v: v[0].ln().sqrt(), (2.0,), (-1.0,), ["nan"]),
    # tests/abs_kink_convention.rs:60-64 and :87-121 (both zeros)
    ("abs_kink_pos", lambda v: abs(v[0]), (1.0,), (0.0,), [0.0]),
    ("abs_kink_neg", lambda v: abs(v[0]), (1.0,), (-0.0,), [0.0]),
    # tests/abs_kink_convention.rs:32-38
    ("abs_pos", lambda v: abs(v[0]), (1.0,), (2.0,), [1.0]),
    ("abs_neg", lambda v: abs(v[0]), (1.0,), (-2.0,), [-1.0]),
    # tests/abs_kink_convention.rs:123-131
    ("abs_nan", lambda v: abs(v[0]), (1.0,), (math.nan,), ["nan"]),
    # tests/domain_nan_convention.rs:55-60 (out of domain -> NaN)
    ("ln_ood", lambda v: v[0].ln(), (2.0,), (-2.0,), ["nan"]),
    ("log2_ood", lambda v: v[0].log2(), (2.0,), (-2.0,), ["nan"]),
    ("log10_ood", lambda v: v[0].log10(), (2.0,), (-2.0,), ["nan"]),
    ("ln_1p_ood", lambda v: v[0].ln_1p(), (2.0,), (-2.0,), ["nan"]),
    ("atanh_ood", lambda v: v[0].atanh(), (0.5,), (1.5,), ["nan"]),
    ("acosh_ood", lambda v: v[0].acosh(), (2.0,), (-2.0,), ["nan"]),
    # tests/domain_nan_convention.rs:66-80 (boundary keeps the one-sided limit)
    ("ln_at_pos_zero", lambda v: v[0].ln(), (2.0,), (0.0,), ["+inf"]),
    ("ln_in_domain", lambda v: v[0].ln(), (1.0,), (2.0,), [0.5]),
]


def _check(got, want, name):
    for k, (g, w) in enumerate(zip(np.asarray(got, dtype=np.float64).ravel(), want)):
        if w == "nan":
            assert math.isnan(g), (name, k, g)
        elif w == "inf":
            assert math.isinf(g), (name, k, g)
        elif w == "+inf":
            assert math.isinf(g) and g > 0, (name, k, g)
        elif isinstance(w, tuple):
            assert abs(g - w[1]) < w[2], (name, k, g, w)
        else:
            assert g == w, (name, k, g, w)


@pytest.mark.parametrize("case", GRAD_CASES, ids=[c[0] for c in GRAD_CASES])
def test_oracle_gradient_known_answers(case):
    name, fn, x0, x, want = case
    tape = _rec(fn, x0)
    _, g = OracleTape(tape).gradient(np.asarray([x]))
    _check(g[0], want, name)


@pytest.mark.gpu
@pytest.mark.parametrize("case", GRAD_CASES, ids=[c[0] for c in GRAD_CASES])
def test_gpu_gradient_known_answers(ctx, case):
    name, fn, x0, x, want = case
    tape = _rec(fn, x0)
    gt = ctx.upload_tape_f64(tape)
    _, g = ctx.gradient_batch_f64(gt, np.asarray(x), 1)
    _check(g, want, name)
    if name.startswith("abs_kink"):
        # abs_kink_convention.rs:93-112: f32 reverse 0, HVP gradient 0 and H*v finite
        g32t = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
        _, g32 = ctx.gradient_batch(g32t, np.asarray(x, dtype=np.float32), 1)
        assert g32[0] == 0.0
        g2, hv = ctx.hvp_batch(g32t, np.asarray(x, dtype=np.float32), np.ones(1, np.float32), 1)
        assert g2[0] == 0.0 and np.isfinite(hv[0])


def test_oracle_abs_kink_hvp():
    # tests/abs_kink_convention.rs:60-64
    tape = _rec(lambda v: abs(v[0]), (0.0,))
    g, h = OracleTape(tape).hvp(np.zeros((1, 1)), np.ones((1, 1)))
    assert g[0, 0] == 0.0 and h[0, 0] == 0.0


def _rosen2(v):
    x, y = v[0], v[1]
    return (1.0 - x) * (1.0 - x) + 100.0 * (y - x * x) * (y - x * x)


def test_oracle_rosenbrock_hessian_analytic():
    # tests/hessian.rs:246-285: H = [[2 - 400y + 1200x^2, -400x], [-400x, 200]] at (1.5, 2)
    x, y = 1.5, 2.0
    tape = _rec(_rosen2, (x, y))
    _, _, H = OracleTape(tape).hessian(np.array([x, y]))
    want = np.array([[2.0 - 400.0 * y + 1200.0 * x * x, -400.0 * x], [-400.0 * x, 200.0]])
    assert np.abs(H - want).max() < 1e-10


def _poly(v):
    return v[0] * v[0] + v[1] * v[1]


@pytest.mark.parametrize("order", [1, 2, 3, 4, 5])
def test_oracle_taylor_polynomial(order):
    # tests/gpu_cuda_tests.rs:328-372: x^2 + y^2 at (3, 4) along (1, 0): 25, 6, 1, 0, 0
    tape = _rec(_poly, (3.0, 4.0))
    c = OracleTape(tape).taylor(np.array([[3.0, 4.0]]), np.array([[1.0, 0.0]]), order)
    want = [25.0, 6.0, 1.0, 0.0, 0.0][:order]
    assert np.allclose(c[:, 0], want, atol=1e-12)


def test_oracle_taylor_multi_batch():
    # tests/gpu_cuda_tests.rs:481-513: directions (1,0) and (0,1): c1 = 6 and 8, c2 = 1
    tape = _rec(_poly, (3.0, 4.0))
    c = OracleTape(tape).taylor(np.array([[3.0, 4.0], [3.0, 4.0]]), np.array([[1.0, 0.0], [0.0, 1.0]]), 4)
    assert np.allclose(c[0], [25.0, 25.0]) and np.allclose(c[1], [6.0, 8.0]) and np.allclose(c[2], [1.0, 1.0])
    assert np.allclose(c[3], [0.0, 0.0])


def test_oracle_taylor_k1_primal_only():
    # tests/gpu_cuda_tests.rs:516-538: K=1 at (2, 3) gives 13
    tape = _rec(_poly, (2.0, 3.0))
    c = OracleTape(tape).taylor(np.array([[2.0, 3.0]]), np.array([[1.0, 0.0]]), 1)
    assert c.shape == (1, 1) and abs(c[0, 0] - 13.0) < 1e-12


def test_oracle_taylor_exp_coefficients():
    # tests/gpu_cuda_tests.rs:426-462: exp(x) at 1 along 1: c_k = e / k!
    tape = _rec(lambda v: v[0].exp(), (1.0,))
    c = OracleTape(tape).taylor(np.array([[1.0]]), np.array([[1.0]]), 5)
    want = [math.e / math.factorial(k) for k in range(5)]
    assert np.allclose(c[:, 0], want, rtol=1e-14)


def test_oracle_hvp_tape_reuse():
    # tests/hessian.rs: f = x^2 y + y^3; H = [[2y, 2x], [2x, 6y]]
    tape = _rec(lambda v: v[0] * v[0] * v[1] + v[1] * v[1] * v[1], (1.0, 1.0))
    o = OracleTape(tape)
    for x, y in [(1.0, 1.0), (2.0, 3.0), (-1.5, 0.5)]:
        H = np.array([[2 * y, 2 * x], [2 * x, 6 * y]])
        for v in (np.array([1.0, 0.0]), np.array([0.3, -0.7])):
            _, hv = o.hvp(np.array([[x, y]]), v[None, :])
            assert np.allclose(hv[0], H @ v, rtol=1e-14, atol=1e-14)
