"""Host-buffer sweeps of large batches run in chunks on several streams once
their launch shape is tuned (copies of one chunk overlap the sweeps of the
others).  The chunked calls must return exactly what the first, whole-batch
call returned, for ragged batch sizes (the largest stages chunks of several
MiB, which the host copies in parts on its copy threads), and the f64 gradients
must match the oracle."""
import numpy as np
import pytest

from echidna_b200 import configs
from echidna_b200.gpu import GpuTapeData
from oracle.oracle import OracleTape

pytestmark = pytest.mark.gpu


def _bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32 if a.dtype == np.float32 else np.uint64)


@pytest.mark.parametrize("B", [16384, 50001, 200003])
def test_chunked_gradient_and_hvp_equal_whole_batch(ctx, B):
    tape = configs.mlp(16, 16)
    rng = np.random.default_rng(B)
    X = rng.normal(size=(B, 16)).astype(np.float32)
    V = rng.choice([-1.0, 1.0], size=(B, 16)).astype(np.float32)
    gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    first = ctx.gradient_batch(gt, X, B)        # whole batch; tunes the shape
    again = ctx.gradient_batch(gt, X, B)        # chunked
    for a, b in zip(first, again):
        assert (_bits(a) == _bits(b)).all()
    h1 = ctx.hvp_batch_points(gt, X, V, B)
    h2 = ctx.hvp_batch_points(gt, X, V, B)
    for a, b in zip(h1, h2):
        assert (_bits(a) == _bits(b)).all()


def test_chunked_f64_gradient_matches_oracle(ctx):
    tape = configs.rosenbrock(12)
    B = 40000
    X = np.random.default_rng(3).uniform(-2, 2, size=(B, 12))
    gt = ctx.upload_tape_f64(tape)
    ctx.gradient_batch_f64(gt, X, B)
    v, g = ctx.gradient_batch_f64(gt, X, B)
    ov, og = OracleTape(tape).gradient(X)
    assert (_bits(v) == _bits(ov[:, 0])).all()
    assert (_bits(g.reshape(B, 12)) == _bits(og)).all()


def test_chunked_calls_from_two_threads(ctx):
    # two contexts on one device, each called from its own thread with pageable
    # arrays big enough that both stage their chunks through the shared pool of
    # copy threads at once: every call returns what a call on its own returns
    import threading

    from echidna_b200.gpu import CudaContext
    tape = configs.mlp(16, 16)
    B = 200003
    rng = np.random.default_rng(7)
    X = [rng.normal(size=(B, 16)).astype(np.float32) for _ in range(2)]
    ctxs = [ctx, CudaContext.new(0)]
    tapes = [c.upload_tape(GpuTapeData.from_tape_f64_lossy(tape)) for c in ctxs]
    want = []
    for c, t, x in zip(ctxs, tapes, X):
        c.gradient_batch(t, x, B)                  # tunes the shape (whole batch)
        want.append(c.gradient_batch(t, x, B))     # chunked, alone
    got = [None, None]
    errors = []

    def run(i):
        try:
            for _ in range(3):
                got[i] = ctxs[i].gradient_batch(tapes[i], X[i], B)
        except Exception as e:  # reported below
            errors.append(e)
    threads = [threading.Thread(target=run, args=(i,)) for i in range(2)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    assert not errors, errors
    for i in range(2):
        for a, b in zip(got[i], want[i]):
            assert (_bits(a) == _bits(b)).all()
    tapes.clear()
    ctxs[1].close()
