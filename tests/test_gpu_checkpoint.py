"""Checkpointed gradients of iterated maps (src/checkpoint.rs): equal for every
checkpoint budget, and equal to the gradient of the unrolled composition."""
import numpy as np
import pytest

from echidna_b200 import record, record_multi
from echidna_b200.checkpoint import grad_checkpointed
from oracle.oracle import OracleTape

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

N = 4


def step_fn(x):
    # a smooth, dimension-preserving map (tests/checkpoint.rs style: mix + nonlinearity)
    return [(x[i] * 0.9 + (x[(i + 1) % N] * 0.3).sin() + 0.05 * x[(i + 2) % N] * x[i]) for i in range(N)]


def loss_fn(x):
    s = x[0] * x[0]
    for i in range(1, N):
        s = s + x[i] * x[i]
    return s


def unrolled(T):
    def f(x):
        for _ in range(T):
            x = step_fn(x)
        return loss_fn(x)
    return f


@pytest.mark.parametrize("T", [0, 1, 7, 20])
def test_matches_unrolled_gradient_for_every_budget(ctx, T):
    x0 = [0.3, -0.2, 0.5, 0.1]
    st, _ = record_multi(step_fn, x0)
    ls, _ = record(loss_fn, x0)
    gs, gl = ctx.upload_tape_f64(st), ctx.upload_tape_f64(ls)
    X0 = np.random.default_rng(T).uniform(-1, 1, size=(300, N))
    X = torch.tensor(X0, device="cuda")
    ut, _ = record(unrolled(T), x0)
    _, ref = OracleTape(ut).gradient(X0)
    results = []
    for c in (1, 3, max(T, 1) + 5):
        g = grad_checkpointed(ctx, gs, gl, X, T, c).cpu().numpy()
        assert np.allclose(g, ref, rtol=1e-12, atol=1e-12), (T, c)
        results.append(g)
    for g in results[1:]:  # the budget changes memory, not arithmetic
        assert np.array_equal(g, results[0])
