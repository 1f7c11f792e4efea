"""The two builds of each sweep kernel compute the same bits.

Every sweep kernel exists with and without the dense-group executor; programs
with dense groups need the first, and the autotuner picks either for the rest
(the build without it needs fewer registers).  `ech_ctx_set_dense_kernel` forces
the dense-group build on the fixed shape; these tests run the same calls both
ways (and with the autotuner's choice) and require identical results, on tapes
without dense groups (Rosenbrock, a random DAG, the softplus chain's jets) and
with them (the MLP).
"""
import numpy as np
import pytest

from echidna_b200 import _lib, configs
from echidna_b200.gpu import GpuTapeData, MultiTapeHvp

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture
def builds(ctx):
    """Runs fn() with the automatic choice (tuned), the fixed shape without the
    dense-group build, and the fixed shape with it; restores the defaults."""
    def run(fn):
        out = []
        try:
            for launch, dense in (("auto", False), ("fixed", False), ("fixed", True)):
                ctx.set_autotune(launch == "auto")
                ctx.set_dense_kernel(dense)
                out.append(fn())
        finally:
            ctx.set_dense_kernel(False)
            ctx.set_autotune(True)
        return out
    yield run


def _same(results):
    first = results[0]
    for r in results[1:]:
        for a, b in zip(first, r):
            np.testing.assert_array_equal(np.asarray(a), np.asarray(b))


def test_rosenbrock_gradient_and_hvp_f64(ctx, builds):
    tape = configs.rosenbrock(100)
    gt = ctx.upload_tape_f64(tape)
    rng = np.random.default_rng(11)
    B = 1024
    X = rng.uniform(-2, 2, size=(B, 100))
    V = rng.choice([-1.0, 1.0], size=(B, 100))
    assert ctx.plan_stats(gt, "gradient")["n_instructions"] > 0
    _same(builds(lambda: ctx.gradient_batch_f64(gt, X.reshape(-1), B)))
    _same(builds(lambda: ctx.hvp_batch_points_f64(gt, X.reshape(-1), V.reshape(-1), B)))


def test_random_dag_f32_gradient_hvp_and_jets(ctx, builds):
    tape = configs.random_dag(24, 3000, seed=5)
    gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    rng = np.random.default_rng(12)
    B = 4096
    X = rng.uniform(-1, 1, size=(B, 24)).astype(np.float32)
    V = rng.normal(size=(B, 24)).astype(np.float32)
    _same(builds(lambda: ctx.gradient_batch(gt, X.reshape(-1), B)))
    _same(builds(lambda: ctx.hvp_batch_points(gt, X.reshape(-1), V.reshape(-1), B)))
    for order in (2, 3, 5):
        _same(builds(lambda: ctx.taylor_forward_kth_batch(gt, X.reshape(-1), V.reshape(-1), B, order).coefficients))


def test_softplus_chain_jets_f32(ctx, builds):
    tape = configs.softplus_chain(256)
    gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    rng = np.random.default_rng(13)
    B = 2048
    X = rng.normal(size=(B, 256)).astype(np.float32)
    V = rng.choice([-1.0, 1.0], size=(B, 256)).astype(np.float32)
    _same(builds(lambda: ctx.taylor_forward_kth_batch(gt, X.reshape(-1), V.reshape(-1), B, 3).coefficients))


def test_mlp_with_dense_groups_f32(ctx, builds):
    tape = configs.mlp(64, 64)
    gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    rng = np.random.default_rng(14)
    B = 8192
    X = rng.normal(size=(B, 64)).astype(np.float32)
    V = rng.choice([-1.0, 1.0], size=(B, 64)).astype(np.float32)
    _same(builds(lambda: ctx.gradient_batch(gt, X.reshape(-1), B)))
    _same(builds(lambda: ctx.hvp_batch_points(gt, X.reshape(-1), V.reshape(-1), B)))


def test_many_tape_launch_on_both_builds(ctx):
    suite = configs.uneven_suite(count=8, seed=78, max_points=2000, max_len=2500, max_dim=40)
    rng = np.random.default_rng(15)
    jobs = []
    for _, tape, n in suite:
        gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
        ni = tape.num_inputs
        x = torch.tensor(rng.uniform(-1, 1, size=(n, ni)), dtype=torch.float32, device="cuda")
        v = torch.tensor(rng.choice([-1.0, 1.0], size=(n, ni)), dtype=torch.float32, device="cuda")
        jobs.append((gt, n, x, v))
    outs = []
    try:
        for dense in (False, True):
            ctx.set_dense_kernel(dense)
            res = []
            items = []
            for gt, n, x, v in jobs:
                g = torch.full((x.numel(),), float("nan"), device="cuda")
                h = torch.full((x.numel(),), float("nan"), device="cuda")
                res.append((g, h))
                items.append((gt, x.data_ptr(), v.data_ptr(), n, g.data_ptr(), h.data_ptr()))
            torch.cuda.synchronize()
            m = MultiTapeHvp(ctx, items, f64=False, autotune=True)
            assert m.info()["dense_kernel"] == int(dense)
            m.launch()
            assert _lib.load().ech_ctx_synchronize(ctx._h) == 0, _lib.last_error()
            m.close()
            outs.append(res)
    finally:
        ctx.set_dense_kernel(False)
    for (g0, h0), (g1, h1) in zip(*outs):
        assert torch.equal(g0, g1)
        assert torch.equal(h0, h1)
