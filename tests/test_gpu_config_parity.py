"""Parity at the benchmarked configurations, with the launch shapes the bench uses.

* MLP n=64, two tanh layers of width 64, 65,536 points, FP32: gradient and
  per-point HVP through the device-pointer calls with the autotuner on (the
  bench's kernels), and through the host-buffer calls (four chunked streams),
  against the FP32 oracle and the FP64 oracle.
* The uneven batch at its full size (64 tapes, up to ~17k ops and 512 inputs,
  670k points): one persistent many-tape launch, sampled rows of every tape
  against the oracle's per-point HVP.
* The STDE Laplacian of logsumexp(tanh(Wx+b)), n=256, W 512x256: FP32 estimates
  against the exact Hessian trace of the oracle's dense tape Hessian
  (src/bytecode_tape/tangent.rs:334-376) and, with the same host directions,
  against the oracle's stde::laplacian (src/stde/laplacian.rs:28-41).

Tolerances (FP32 sweeps through CUDA's tanhf/expf/logf against glibc's, f32
arithmetic otherwise rounded like the CPU):
* MLP: max |gpu - oracle_f32| <= 2e-5 * max |oracle_f64| per array, and the GPU's
  error against FP64 at most 2x the FP32 oracle's own (+1e-6 of the magnitude).
* Uneven batch: max |gpu - oracle_f32| <= 1e-4 * max(1, max |oracle_f64|) per tape.
* STDE: every point's |estimate - trace| / standard_error < 5 (Student t, 63
  degrees of freedom); host-direction estimates within 1e-4 of the sample
  spread of the FP64 oracle's estimate.
"""
import concurrent.futures as cf
import os

import numpy as np
import pytest

from echidna_b200 import _lib, configs
from echidna_b200.gpu import GpuTapeData, MultiTapeHvp
from echidna_b200.stde_gpu import DIR_PER_POINT, DIR_RADEMACHER, laplacian_batch
from oracle.oracle import OracleTape

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

NTH = os.cpu_count() or 1


def _err(a, ref, scale):
    return float(np.max(np.abs(np.asarray(a, np.float64) - np.asarray(ref, np.float64)))) / scale


@pytest.fixture(scope="module")
def mlp_case(ctx):
    ctx.set_launch(0, 0, 0)
    ctx.set_autotune(True)
    tape = configs.mlp(64, 64)
    B, n = 65536, 64
    rng = np.random.default_rng(configs.SEEDS["mlp"])
    X = rng.normal(size=(B, n)).astype(np.float32)
    V = rng.choice([-1.0, 1.0], size=(B, n)).astype(np.float32)
    gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    o32, o64 = OracleTape(tape, dtype=np.float32), OracleTape(tape)
    return tape, gt, X, V, o32, o64


def test_mlp_gradient_65536_tuned_shape(ctx, mlp_case):
    tape, gt, X, V, o32, o64 = mlp_case
    B, n = X.shape
    lib = _lib.load()
    dX = torch.from_numpy(X).cuda()
    out = torch.full((B,), float("nan"), device="cuda")
    g = torch.full((B * n,), float("nan"), device="cuda")
    for _ in range(2):  # the first call tunes the shape, the second runs the tuned shape
        st = lib.ech_gradient_batch_device(ctx._h, gt._h, 0, dX.data_ptr(), B, out.data_ptr(), g.data_ptr(), None)
        assert st == 0, _lib.last_error()
        assert lib.ech_ctx_synchronize(ctx._h) == 0, _lib.last_error()
    assert ctx.launch_shape(gt, "gradient", B)["tuned"] == 1
    v_gpu, g_gpu = out.cpu().numpy(), g.cpu().numpy().reshape(B, n)
    v32, g32 = o32.gradient(X, NTH)
    v64, g64 = o64.gradient(X.astype(np.float64), NTH)
    gs, vs = np.abs(g64).max(), np.abs(v64).max()
    assert _err(v_gpu, v32[:, 0], vs) <= 2e-5
    assert _err(g_gpu, g32, gs) <= 2e-5
    assert _err(g_gpu, g64, gs) <= 2 * _err(g32, g64, gs) + 1e-6
    assert _err(v_gpu, v64[:, 0], vs) <= 2 * _err(v32[:, 0], v64[:, 0], vs) + 1e-6
    # the host-buffer call (chunked over four streams once tuned) gives the same bits
    hv, hg = ctx.gradient_batch(gt, X, B)
    np.testing.assert_array_equal(hv, v_gpu)
    np.testing.assert_array_equal(hg.reshape(B, n), g_gpu)


def test_mlp_hvp_65536_tuned_shape(ctx, mlp_case):
    tape, gt, X, V, o32, o64 = mlp_case
    B, n = X.shape
    lib = _lib.load()
    dX, dV = torch.from_numpy(X).cuda(), torch.from_numpy(V).cuda()
    g = torch.full((B * n,), float("nan"), device="cuda")
    h = torch.full((B * n,), float("nan"), device="cuda")
    for _ in range(2):
        st = lib.ech_hvp_batch_device(ctx._h, gt._h, 0, dX.data_ptr(), 1, dV.data_ptr(), B, g.data_ptr(),
                                      h.data_ptr(), None)
        assert st == 0, _lib.last_error()
        assert lib.ech_ctx_synchronize(ctx._h) == 0, _lib.last_error()
    assert ctx.launch_shape(gt, "hvp", B)["tuned"] == 1
    g_gpu, h_gpu = g.cpu().numpy().reshape(B, n), h.cpu().numpy().reshape(B, n)
    g32, h32 = o32.hvp(X, V, NTH)
    g64, h64 = o64.hvp(X.astype(np.float64), V.astype(np.float64), NTH)
    gs, hs = np.abs(g64).max(), np.abs(h64).max()
    assert _err(g_gpu, g32, gs) <= 2e-5
    assert _err(h_gpu, h32, hs) <= 2e-5
    assert _err(h_gpu, h64, hs) <= 2 * _err(h32, h64, hs) + 1e-6
    hg, hh = ctx.hvp_batch_points(gt, X, V, B)
    np.testing.assert_array_equal(hg.reshape(B, n), g_gpu)
    np.testing.assert_array_equal(hh.reshape(B, n), h_gpu)


def test_uneven_batch_full_config_against_oracle(ctx):
    ctx.set_launch(0, 0, 0)
    suite = configs.uneven_suite(64, configs.SEEDS["uneven"])
    rng = np.random.default_rng([configs.SEEDS["uneven"], 0])
    jobs = []
    for name, tape, n in suite:
        ni = tape.num_inputs
        x = rng.uniform(-1.0, 1.0, size=(n, ni)).astype(np.float32)
        v = rng.choice([-1.0, 1.0], size=(n, ni)).astype(np.float32)
        gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
        dx, dv = torch.from_numpy(x).cuda(), torch.from_numpy(v).cuda()
        g = torch.full((n * ni,), float("nan"), device="cuda")
        h = torch.full((n * ni,), float("nan"), device="cuda")
        jobs.append((name, tape, gt, n, x, v, dx, dv, g, h))
    assert max(len(j[1].arrays()[0]) for j in jobs) > 10000 and max(j[1].num_inputs for j in jobs) > 256
    torch.cuda.synchronize()
    m = MultiTapeHvp(ctx, [(gt, dx.data_ptr(), dv.data_ptr(), n, g.data_ptr(), h.data_ptr())
                           for _, _, gt, n, _, _, dx, dv, g, h in jobs], f64=False, autotune=True)
    m.launch()
    assert _lib.load().ech_ctx_synchronize(ctx._h) == 0, _lib.last_error()

    def check(job):
        name, tape, _, n, x, v, _, _, g, h = job
        ni = tape.num_inputs
        rows = np.unique(np.r_[np.arange(min(n, 16)), np.arange(max(0, n - 16), n)])
        o32, o64 = OracleTape(tape, dtype=np.float32), OracleTape(tape)
        g32, h32 = o32.hvp(x[rows], v[rows])
        g64, h64 = o64.hvp(x[rows].astype(np.float64), v[rows].astype(np.float64))
        gg = g.view(n, ni)[rows].cpu().numpy()
        hh = h.view(n, ni)[rows].cpu().numpy()
        sg, sh = max(1.0, np.abs(g64).max()), max(1.0, np.abs(h64).max())
        return name, _err(gg, g32, sg), _err(hh, h32, sh), bool(np.isfinite(gg).all() and np.isfinite(hh).all())

    with cf.ThreadPoolExecutor(NTH) as ex:
        results = list(ex.map(check, jobs))
    for name, eg, eh, finite in results:
        assert finite, name
        assert eg <= 1e-4, (name, eg)
        assert eh <= 1e-4, (name, eh)
    m.close()


@pytest.fixture(scope="module")
def stde_case(ctx):
    tape = configs.logsumexp_tanh(256, 512)
    gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    rng = np.random.default_rng(configs.SEEDS["logsumexp_tanh"])
    X = rng.normal(size=(16, 256))
    o64 = OracleTape(tape)
    with cf.ThreadPoolExecutor(NTH) as ex:
        traces = np.array(list(ex.map(lambda x: np.trace(o64.hessian(x)[2]), X)))
    return tape, gt, X, o64, traces


def test_stde_laplacian_fp32_device_rng_against_exact_trace(ctx, stde_case):
    _, gt, X, _, traces = stde_case
    S = 64
    r = laplacian_batch(ctx, gt, X.astype(np.float32), S, None, DIR_RADEMACHER, seed=configs.SEEDS["logsumexp_tanh"])
    assert (r["num_samples"] == S).all()
    z = (r["estimate"] - traces) / r["standard_error"]
    assert np.all(np.abs(z) < 5.0), z


def test_stde_laplacian_fp32_host_directions_against_oracle(ctx, stde_case):
    _, gt, X, o64, _ = stde_case
    S, n = 64, 256
    rng = np.random.default_rng(3)
    D = rng.choice([-1.0, 1.0], size=(len(X), S, n))
    r = laplacian_batch(ctx, gt, X.astype(np.float32), S, D.astype(np.float32), DIR_PER_POINT)
    ref = o64.laplacian_stats_batch(X, D, NTH)   # value, estimate, variance, se, n
    spread = np.sqrt(ref[:, 2])
    assert np.all(np.abs(r["estimate"] - ref[:, 1]) <= 1e-4 * (np.abs(ref[:, 1]) + spread)), (r["estimate"], ref[:, 1])
    assert np.all(np.abs(r["value"] - ref[:, 0]) <= 1e-5 * np.abs(ref[:, 0]).max())
