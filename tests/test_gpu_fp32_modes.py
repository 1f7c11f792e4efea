"""FP32 options of the batch STDE calls (ech_ctx_set_fp32_mode) on the STDE
Laplacian tape logsumexp(tanh(Wx+b)), n=256, W 512x256.

* Reduction: the per-point mean of the same FP32 samples in FP32 Welford,
  in FP32 with compensated sums, and in FP64 Welford (the default).  Against the
  FP64 reduction, the compensated FP32 mean's error must be well below the
  uncompensated one's (median over points, many directions per point).
* Sweep: FP32 jets with and without compensated linear chains against the FP64
  sweep with the same device directions.  On this tape both errors are a few
  FP32 ulps (median ~2e-7 relative): the libm-class ops, not the sums, set
  the sweep's error, so compensation does not lower it; the test bounds both.
* The default mode is unchanged by the options: setting them back restores the
  default results bit for bit.
"""
import numpy as np
import pytest

from echidna_b200 import configs
from echidna_b200.gpu import GpuTapeData
from echidna_b200.stde_gpu import DIR_RADEMACHER, laplacian_batch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c3(ctx):
    tape = configs.logsumexp_tanh(256, 512)
    g32 = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    g64 = ctx.upload_tape_f64(tape)
    X = np.random.default_rng(21).normal(size=(16, 256))
    yield g32, g64, X
    ctx.set_fp32_mode(0)


def _est(ctx, gt, X, S, flags, seed=5):
    ctx.set_fp32_mode(flags)
    try:
        return laplacian_batch(ctx, gt, X, S, None, DIR_RADEMACHER, seed=seed)
    finally:
        ctx.set_fp32_mode(0)


def test_compensated_fp32_mean_beats_fp32_welford(ctx, c3):
    g32, _, X = c3
    S = 4096
    X32 = X.astype(np.float32)
    ref = _est(ctx, g32, X32, S, 0)                                  # FP64 Welford of the FP32 samples
    plain = _est(ctx, g32, X32, S, ctx.FP32_PLAIN_MEANS)
    comp = _est(ctx, g32, X32, S, ctx.FP32_COMPENSATED_MEANS)
    assert np.array_equal(plain["num_samples"], ref["num_samples"])
    assert np.array_equal(comp["num_samples"], ref["num_samples"])
    e_plain = np.abs(plain["estimate"] - ref["estimate"]) / np.abs(ref["estimate"])
    e_comp = np.abs(comp["estimate"] - ref["estimate"]) / np.abs(ref["estimate"])
    v_comp = np.abs(comp["sample_variance"] - ref["sample_variance"]) / ref["sample_variance"]
    print(f"mean rel err vs FP64 reduction: fp32 welford {np.median(e_plain):.3g}, compensated {np.median(e_comp):.3g}")
    # the compensated mean is the FP32 rounding of the exact mean of the samples
    assert np.all(e_comp <= 2 * np.finfo(np.float32).eps)
    assert np.median(e_comp) * 4 <= np.median(e_plain)
    assert np.all(v_comp <= 1e-5)


def test_compensated_fp32_jets_against_fp64_sweep(ctx, c3):
    g32, g64, X = c3
    S = 256
    ref = laplacian_batch(ctx, g64, X, S, None, DIR_RADEMACHER, seed=9)["estimate"]
    plain = _est(ctx, g32, X.astype(np.float32), S, ctx.FP32_COMPENSATED_MEANS, seed=9)["estimate"]
    comp = _est(ctx, g32, X.astype(np.float32), S, ctx.FP32_COMPENSATED_JETS | ctx.FP32_COMPENSATED_MEANS,
                seed=9)["estimate"]
    e_plain = np.abs(plain - ref) / np.abs(ref)
    e_comp = np.abs(comp - ref) / np.abs(ref)
    print(f"estimate rel err vs FP64 sweep: fp32 jets {np.median(e_plain):.3g}, compensated {np.median(e_comp):.3g}")
    assert np.max(e_plain) <= 1e-5
    assert np.max(e_comp) <= 1e-5


def test_options_leave_the_default_unchanged(ctx, c3):
    g32, _, X = c3
    a = _est(ctx, g32, X.astype(np.float32), 64, 0)
    _est(ctx, g32, X.astype(np.float32), 64, ctx.FP32_COMPENSATED_JETS | ctx.FP32_COMPENSATED_MEANS)
    b = _est(ctx, g32, X.astype(np.float32), 64, 0)
    for f in ("value", "estimate", "sample_variance", "standard_error", "num_samples"):
        assert np.array_equal(a[f], b[f])


def test_invalid_flags_rejected(ctx):
    with pytest.raises(AssertionError, match="exclude each other"):
        ctx.set_fp32_mode(ctx.FP32_COMPENSATED_MEANS | ctx.FP32_PLAIN_MEANS)
    with pytest.raises(AssertionError, match="unknown FP32 mode flag"):
        ctx.set_fp32_mode(64)
