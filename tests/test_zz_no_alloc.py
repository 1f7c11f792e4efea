"""ech_gradient_batch_device_noalloc against ech_gradient_batch_device.

Both calls run the same sweep kernel on the same program, so the tolerance is
exact equality (0 ulp).  The allocation-free call is made twice in a row to
show that nothing left in its fixed region from one call changes the next.
Collected last so it also runs after every other test in the session.
"""
import ctypes

import numpy as np
import pytest

from echidna_b200 import _lib, configs, record
from echidna_b200.gpu import GpuTapeData

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _run(ctx, gt, f64, X, no, ni, noalloc):
    lib = _lib.load()
    dt = torch.float64 if f64 else torch.float32
    B = X.shape[0]
    dX = torch.tensor(X, dtype=dt, device="cuda")
    out = torch.full((B * no,), float("nan"), dtype=dt, device="cuda")
    grads = torch.full((B * ni,), float("nan"), dtype=dt, device="cuda")
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    fn = lib.ech_gradient_batch_device_noalloc if noalloc else lib.ech_gradient_batch_device
    with torch.cuda.stream(s):
        st = fn(ctx._h, gt._h, int(f64), dX.data_ptr(), B, out.data_ptr(), grads.data_ptr(),
                ctypes.c_void_p(s.cuda_stream))
    assert st == _lib.OK, _lib.last_error()
    s.synchronize()
    assert lib.ech_ctx_synchronize(ctx._h) == _lib.OK, _lib.last_error()
    return out.cpu().numpy(), grads.cpu().numpy()


def _check_same(ctx, gt, f64, X, no, ni):
    ref_v, ref_g = _run(ctx, gt, f64, X, no, ni, noalloc=False)
    for _ in range(2):
        v, g = _run(ctx, gt, f64, X, no, ni, noalloc=True)
        np.testing.assert_array_equal(v, ref_v)
        np.testing.assert_array_equal(g, ref_g)


def test_region_size_is_stated(engine_lib):
    assert engine_lib.ech_noalloc_region_bytes() == 64 << 20


def test_noalloc_matches_gradient_mlp_f32(ctx):
    tape = configs.mlp(64, 64)
    gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    X = np.random.default_rng(7).normal(size=(4096, 64))
    _check_same(ctx, gt, False, X, 1, 64)


def test_noalloc_matches_gradient_rosenbrock_f64_shrunk_grid(ctx):
    # 396 trajectory slots * 128 points * 8 B per CTA: the 64 MiB region holds
    # fewer CTAs than the occupancy limit, so the grid shrinks
    tape = configs.rosenbrock(100)
    gt = ctx.upload_tape_f64(tape)
    X = np.random.default_rng(8).uniform(-2.0, 2.0, size=(100_000, 100))
    _check_same(ctx, gt, True, X, 1, 100)


def _sin_chain(n):
    def f(x):
        y = x[0]
        for _ in range(n):
            y = y.sin()
        return y
    return record(f, [0.5])[0]


def test_noalloc_one_cta_grid_f32(ctx):
    # 70,000 trajectory slots * 128 points * 4 B = 35.8 MB: one CTA fits
    tape = _sin_chain(70_000)
    gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    X = np.random.default_rng(9).uniform(-1.0, 1.0, size=(1000, 1))
    _check_same(ctx, gt, False, X, 1, 1)


def test_noalloc_rejects_oversized_scratch(ctx):
    # 70,000 trajectory slots * 128 points * 8 B = 71.7 MB > 64 MiB
    tape = _sin_chain(70_000)
    gt = ctx.upload_tape_f64(tape)
    lib = _lib.load()
    dX = torch.zeros(128, dtype=torch.float64, device="cuda")
    out = torch.zeros(128, dtype=torch.float64, device="cuda")
    g = torch.zeros(128, dtype=torch.float64, device="cuda")
    st = lib.ech_gradient_batch_device_noalloc(ctx._h, gt._h, 1, dX.data_ptr(), 128, out.data_ptr(), g.data_ptr(),
                                               None)
    assert st == _lib.OUT_OF_MEMORY
    assert "no-alloc region too small" in _lib.last_error()


def test_noalloc_rosenbrock_1024_points_bit_exact_against_oracle(ctx):
    # extended Rosenbrock n=100, 1,024 points, f64: +, -, * only, so the sweep must
    # equal the reference's CPU tape bit for bit; two calls in a row (the second
    # finds the program already in the region and skips the copy)
    from oracle.oracle import OracleTape
    tape = configs.rosenbrock(100)
    gt = ctx.upload_tape_f64(tape)
    X = np.random.default_rng(configs.SEEDS["rosenbrock"]).uniform(-2.0, 2.0, size=(1024, 100))
    ov, og = OracleTape(tape).gradient(X)
    for _ in range(2):
        v, g = _run(ctx, gt, True, X, 1, 100, noalloc=True)
        np.testing.assert_array_equal(v, ov[:, 0])
        np.testing.assert_array_equal(g.reshape(1024, 100), og)


def test_noalloc_alternating_tapes_recopy_programs(ctx):
    # two tapes alternating: each call must find its own program in the region
    a = configs.rosenbrock(20)
    b = configs.mlp(16, 16)
    ga, gb = ctx.upload_tape_f64(a), ctx.upload_tape_f64(b)
    rng = np.random.default_rng(12)
    Xa, Xb = rng.uniform(-2, 2, size=(700, 20)), rng.normal(size=(500, 16))
    ra = _run(ctx, ga, True, Xa, 1, 20, noalloc=False)
    rb = _run(ctx, gb, True, Xb, 1, 16, noalloc=False)
    for _ in range(2):
        for gt, X, ni, ref in ((ga, Xa, 20, ra), (gb, Xb, 16, rb)):
            v, g = _run(ctx, gt, True, X, 1, ni, noalloc=True)
            np.testing.assert_array_equal(v, ref[0])
            np.testing.assert_array_equal(g, ref[1])


def test_noalloc_calls_leave_device_memory_unchanged(ctx):
    # after the inputs and outputs exist, calls on a freshly uploaded tape (host
    # lowering only) change the device's free memory by nothing
    lib = _lib.load()
    tape = configs.rosenbrock(60)
    X = np.random.default_rng(13).uniform(-2.0, 2.0, size=(50_000, 60))
    dX = torch.tensor(X, device="cuda")
    out = torch.empty(50_000, dtype=torch.float64, device="cuda")
    g = torch.empty(50_000 * 60, dtype=torch.float64, device="cuda")
    # a warm-up call on another tape first: the first call in a process loads the
    # module that holds the region and the kernel (lazy loading)
    warm = ctx.upload_tape_f64(configs.rosenbrock(8))
    st = lib.ech_gradient_batch_device_noalloc(ctx._h, warm._h, 1, dX.data_ptr(), 1000, out.data_ptr(),
                                               g.data_ptr(), None)
    assert st == _lib.OK, _lib.last_error()
    assert lib.ech_ctx_synchronize(ctx._h) == _lib.OK, _lib.last_error()
    torch.cuda.synchronize()
    gt = ctx.upload_tape_f64(tape)
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        st = lib.ech_gradient_batch_device_noalloc(ctx._h, gt._h, 1, dX.data_ptr(), 50_000, out.data_ptr(),
                                                   g.data_ptr(), None)
        assert st == _lib.OK, _lib.last_error()
    assert lib.ech_ctx_synchronize(ctx._h) == _lib.OK, _lib.last_error()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
