"""Reverse gather tiles on the GPU, bit for bit against the oracle.

The reverse of a dense layer is a gather: each input's adjoint sums c_kj times
the adjoint of every chain k that reads it, in one order.  Runs of consecutive
targets that read the same chain adjoints with nonzero constants run as full
tiles (12 f32 / 6 f64 targets, fewer at four points per thread; a shorter run
stays plain gathers): each chain adjoint is loaded and zero-tested once for the
tile.  These tapes put layer
widths around the tile limits (full and tail tiles), zero weights that keep
their targets out of tiles, adjoints that are zero for some points, and inputs
whose adjoints are infinite or NaN, at one, two and four points per thread.
"""
import numpy as np
import pytest

from echidna_b200 import constant, record
from echidna_b200.gpu import GpuTapeData
from oracle.oracle import OracleTape

pytestmark = pytest.mark.gpu


def _bits_equal(a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b).astype(a.dtype)
    u = np.uint32 if a.dtype == np.float32 else np.uint64
    both_nan = np.isnan(a) & np.isnan(b)
    return bool(((a.view(u) == b.view(u)) | both_nan).all())


def _layer_tape(n, w, W1, W2, act):
    """s = W1 x + b (w chains of n terms), h = act(s), out = sum_k (W2 h + c)_k^2."""
    def f(v):
        h = []
        for j in range(w):
            s = constant(0.1 * j - 0.3)
            for i in range(n):
                s = s + constant(float(W1[j, i])) * v[i]
            h.append(act(s))
        out = constant(0.0)
        for k in range(W2.shape[0]):
            s = constant(-0.2)
            for j in range(w):
                s = s + constant(float(W2[k, j])) * h[j]
            out = out + s * s
        return out
    return record(f, [0.1] * n)[0]


# correctly rounded operations only (products, sums, quotients, square roots),
# so the device and the oracle agree bit for bit
ACTS = {
    "square": lambda s: s * s,
    "rational": lambda s: s / (constant(1.0) + s * s),
    "sqrt": lambda s: (s * s).sqrt(),       # adjoint 0/0 = NaN where s = 0
    "recip": lambda s: constant(1.0) / s,   # infinite where s = 0
}


def _cases():
    rng = np.random.default_rng(41)
    for n, w, zeros, act in [(13, 7, 0.0, "square"), (25, 30, 0.0, "rational"), (12, 24, 0.0, "square"),
                             (40, 3, 0.0, "rational"), (17, 19, 0.15, "square"), (9, 14, 0.0, "sqrt"),
                             (11, 6, 0.0, "recip")]:
        W1 = rng.normal(size=(w, n)) * (rng.random((w, n)) >= zeros)
        W2 = rng.normal(size=(5, w)) * (rng.random((5, w)) >= zeros)
        yield f"n{n}_w{w}_z{zeros}_{act}", n, w, W1, W2, act


CASES = list(_cases())


@pytest.fixture
def launch(ctx):
    yield ctx
    ctx.set_launch(0, 0, 0)
    ctx.set_autotune(True)


def _inputs(n, B, act, dt):
    rng = np.random.default_rng(n * 7 + B)
    X = rng.uniform(-1.5, 1.5, size=(B, n))
    if act in ("sqrt", "recip"):
        X[::5] = 0.0          # s = b at these points
        X[1::7, 0] = np.inf   # infinite inputs
        X[2::11, 1] = np.nan
    V = rng.choice([-1.0, 1.0], size=(B, n))
    V[3::9] = 0.0             # zero directions: zero tangents in the reverse
    return X.astype(dt), V.astype(dt)


@pytest.mark.parametrize("ppt", [1, 2, 4])
@pytest.mark.parametrize("f64", [True, False])
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_gather_tiles_bit_exact(launch, case, f64, ppt):
    ctx = launch
    name, n, w, W1, W2, act = case
    tape = _layer_tape(n, w, W1, W2, ACTS[act])
    dt = np.float64 if f64 else np.float32
    o = OracleTape(tape, dtype=dt)
    B = 389
    X, V = _inputs(n, B, act, dt)
    ctx.set_launch(128, ppt, 0)
    gt = ctx.upload_tape_f64(tape) if f64 else ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    if f64:
        v, g = ctx.gradient_batch_f64(gt, X, B)
        hg, hh = ctx.hvp_batch_points_f64(gt, X, V, B)
    else:
        v, g = ctx.gradient_batch(gt, X, B)
        hg, hh = ctx.hvp_batch_points(gt, X, V, B)
    with np.errstate(all="ignore"):
        ov, og = o.gradient(X)
        ohg, ohh = o.hvp(X, V)
    assert _bits_equal(v, ov[:, 0]), name
    assert _bits_equal(g.reshape(B, n), og), name
    assert _bits_equal(hg.reshape(B, n), ohg), name
    assert _bits_equal(hh.reshape(B, n), ohh), name
    for kind in ("gradient", "hvp"):
        if not (W1 == 0).any() and n >= _tile_size(f64, ppt, kind):
            # the first layer's reverse runs as tiles of its inputs
            ps = ctx.program_stats(gt, kind, B)
            assert ps["gather_tiles"] > 0 and ps["dense_kernel"] == 1, (name, kind, ps)


def _tile_size(f64, ppt, kind):
    """Targets per gather tile: gather_tile_max(dense_group_max(value bytes, P))."""
    vbytes = (8 if f64 else 4) * (2 if kind == "hvp" else 1)
    dense = min(16, 256 // (vbytes * ppt)) & ~1
    return min(dense, 6 if f64 else 12)


def test_mlp_reverse_runs_as_tiles(ctx):
    from echidna_b200 import configs
    tape = configs.mlp(64, 64)
    gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    ctx.set_launch(128, 2, 0)
    try:
        for kind in ("gradient", "hvp"):
            ps = ctx.program_stats(gt, kind, 65536)
            # two 64-wide layers: 64 targets each, five full tiles of 12
            assert ps["gather_tiles"] >= 2 * 5 and ps["dense_groups"] >= 8, (kind, ps)
    finally:
        ctx.set_launch(0, 0, 0)
