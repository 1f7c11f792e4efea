"""GPU STDE estimators (``src/gpu/stde_gpu.rs``) over the engine's C ABI.

``laplacian_gpu``, ``hessian_diagonal_gpu`` and ``laplacian_with_control_gpu`` keep
the reference's signatures and errors.  ``laplacian_batch`` is this engine's
extension: many points, ``S`` directions each, one Taylor launch plus an on-device
per-point Welford reduction; directions come from the caller or from a
counter-based device RNG.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .gpu import CudaContext, CudaTapeBuffers, CudaTapeBuffersF64, EstimatorResult, _check

DIR_PER_POINT, DIR_SHARED, DIR_RADEMACHER = 0, 1, 2


def _result(r: _lib.EstimatorResultC, dt=float) -> EstimatorResult:
    return EstimatorResult(dt(r.value), dt(r.estimate), dt(r.sample_variance), dt(r.standard_error),
                           int(r.num_samples))


def laplacian_gpu(backend: CudaContext, tape: CudaTapeBuffers, x, directions) -> EstimatorResult:
    """Hutchinson Laplacian at one point (``src/gpu/stde_gpu.rs:51-81``)."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    dirs = [np.ascontiguousarray(d, dtype=np.float32) for d in directions]
    for d in dirs:
        assert d.size == x.size, "direction length must match x"
    flat = np.ascontiguousarray(np.stack(dirs) if dirs else np.zeros((0, x.size), np.float32), dtype=np.float32)
    out = _lib.EstimatorResultC()
    _check(_lib.load().ech_laplacian_gpu_f32(backend._h, tape._h, _lib.ptr(x), x.size, _lib.ptr(flat), len(dirs),
                                             ctypes.byref(out)))
    return _result(out, np.float32)


def hessian_diagonal_gpu(backend: CudaContext, tape: CudaTapeBuffers, x):
    """Exact Hessian diagonal via ``n`` basis pushforwards (``src/gpu/stde_gpu.rs:103-129``)."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    value = np.zeros(1, dtype=np.float32)
    diag = np.empty(x.size, dtype=np.float32)
    _check(_lib.load().ech_hessian_diagonal_gpu_f32(backend._h, tape._h, _lib.ptr(x), x.size, _lib.ptr(value),
                                                    _lib.ptr(diag)))
    return value[0], diag


def laplacian_with_control_gpu(backend: CudaContext, tape: CudaTapeBuffers, x, directions,
                               control_diagonal) -> EstimatorResult:
    """Control-variate Laplacian (``src/gpu/stde_gpu.rs:135-200``)."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    c = np.ascontiguousarray(control_diagonal, dtype=np.float32)
    assert c.size == x.size, "control diagonal length must match x"
    dirs = [np.ascontiguousarray(d, dtype=np.float32) for d in directions]
    for d in dirs:
        assert d.size == x.size, "direction length must match x"
    flat = np.ascontiguousarray(np.stack(dirs) if dirs else np.zeros((0, x.size), np.float32), dtype=np.float32)
    out = _lib.EstimatorResultC()
    _check(_lib.load().ech_laplacian_with_control_gpu_f32(backend._h, tape._h, _lib.ptr(x), x.size, _lib.ptr(flat),
                                                          len(dirs), _lib.ptr(c), ctypes.byref(out)))
    return _result(out, np.float32)


def laplacian_batch(backend: CudaContext, tape, xs, num_directions: int, directions=None,
                    mode: int = DIR_PER_POINT, seed: int = 0):
    """Per-point Hutchinson Laplacians for ``xs[B, n]`` with ``num_directions`` each.

    ``mode``: ``DIR_PER_POINT`` (``directions[B, S, n]``), ``DIR_SHARED``
    (``directions[S, n]``) or ``DIR_RADEMACHER`` (device RNG, ``directions=None``).
    Returns a structured array with fields value/estimate/sample_variance/
    standard_error/num_samples.
    """
    f64 = isinstance(tape, CudaTapeBuffersF64)
    dt = np.float64 if f64 else np.float32
    xs = np.ascontiguousarray(xs, dtype=dt)
    B = xs.shape[0] if xs.ndim > 1 else 1
    d = None if directions is None else np.ascontiguousarray(directions, dtype=dt)
    res = (_lib.EstimatorResultC * B)()
    fn = _lib.load().ech_laplacian_batch_f64 if f64 else _lib.load().ech_laplacian_batch_f32
    _check(fn(backend._h, tape._h, _lib.ptr(xs), xs.size, B, _lib.ptr(d), 0 if d is None else d.size,
              int(num_directions), int(mode), ctypes.c_uint64(seed & 0xFFFFFFFFFFFFFFFF), res))
    out = np.zeros(B, dtype=[("value", "f8"), ("estimate", "f8"), ("sample_variance", "f8"),
                             ("standard_error", "f8"), ("num_samples", "u8")])
    for i in range(B):
        out[i] = (res[i].value, res[i].estimate, res[i].sample_variance, res[i].standard_error, res[i].num_samples)
    return out


def diagonal_kth_order_stochastic_gpu(backend: CudaContext, tape, x, k: int, sampled_indices) -> EstimatorResult:
    """``stde::diagonal_kth_order_stochastic`` (``src/stde/higher_order.rs:173-227``) on the GPU:
    ``n * mean_j(k! * c_k)`` over jets along ``e_j`` for the sampled coordinates (k = 2..8)."""
    lib = _lib.load()
    f64 = bool(tape.f64)
    dt = np.float64 if f64 else np.float32
    xx = np.ascontiguousarray(x, dtype=dt).ravel()
    idx = np.ascontiguousarray(sampled_indices, dtype=np.uint32).ravel()
    r = _lib.EstimatorResultC()
    fn = lib.ech_diagonal_kth_order_stochastic_f64 if f64 else lib.ech_diagonal_kth_order_stochastic_f32
    _check(fn(backend._h, tape._h, _lib.ptr(xx), xx.size, int(k), _lib.ptr(idx), idx.size, ctypes.byref(r)))
    return _result(r, float)


def diagonal_kth_order_gpu(backend: CudaContext, tape, x, k: int):
    """``stde::diagonal_kth_order`` (``src/stde/higher_order.rs:40-95``) on the GPU:
    ``(f(x), [k! * c_k along e_j for every j])`` in one launch (k = 2..8)."""
    lib = _lib.load()
    f64 = bool(tape.f64)
    dt = np.float64 if f64 else np.float32
    xx = np.ascontiguousarray(x, dtype=dt).ravel()
    value = np.zeros(1, dtype=dt)
    diag = np.zeros(xx.size, dtype=dt)
    fn = lib.ech_diagonal_kth_order_f64 if f64 else lib.ech_diagonal_kth_order_f32
    _check(fn(backend._h, tape._h, _lib.ptr(xx), xx.size, int(k), _lib.ptr(value), _lib.ptr(diag)))
    return float(value[0]), diag


# ── operator estimators (src/stde/laplacian.rs:252-344, src/stde/pde.rs) ──

def _fn(tape, name):
    lib = _lib.load()
    return getattr(lib, f"ech_{name}_{'f64' if tape.f64 else 'f32'}"), (np.float64 if tape.f64 else np.float32)


def laplacian_hutchpp_gpu(backend: CudaContext, tape, x, sketch_directions, stochastic_directions) -> EstimatorResult:
    """``stde::laplacian_hutchpp``: exact trace on the span of H*S, Hutchinson on the rest."""
    fn, dt = _fn(tape, "laplacian_hutchpp")
    xx = np.ascontiguousarray(x, dtype=dt).ravel()
    S = np.ascontiguousarray(sketch_directions, dtype=dt).reshape(-1, xx.size)
    G = np.ascontiguousarray(stochastic_directions, dtype=dt).reshape(-1, xx.size)
    r = _lib.EstimatorResultC()
    _check(fn(backend._h, tape._h, _lib.ptr(xx), xx.size, _lib.ptr(S), S.shape[0], _lib.ptr(G), G.shape[0],
              ctypes.byref(r)))
    return _result(r)


def parabolic_diffusion_gpu(backend: CudaContext, tape, x, sigma_columns):
    """``stde::parabolic_diffusion``: (value, 1/2 sum_i (sigma e_i)^T H (sigma e_i))."""
    fn, dt = _fn(tape, "parabolic_diffusion")
    xx = np.ascontiguousarray(x, dtype=dt).ravel()
    sig = np.ascontiguousarray(sigma_columns, dtype=dt).reshape(-1, xx.size)
    v, e = np.zeros(1, dt), np.zeros(1, dt)
    _check(fn(backend._h, tape._h, _lib.ptr(xx), xx.size, _lib.ptr(sig), sig.shape[0], _lib.ptr(v), _lib.ptr(e)))
    return float(v[0]), float(e[0])


def parabolic_diffusion_stochastic_gpu(backend: CudaContext, tape, x, sigma_columns, sampled_indices):
    fn, dt = _fn(tape, "parabolic_diffusion_stochastic")
    xx = np.ascontiguousarray(x, dtype=dt).ravel()
    sig = np.ascontiguousarray(sigma_columns, dtype=dt).reshape(-1, xx.size)
    idx = np.ascontiguousarray(sampled_indices, dtype=np.uint32).ravel()
    r = _lib.EstimatorResultC()
    _check(fn(backend._h, tape._h, _lib.ptr(xx), xx.size, _lib.ptr(sig), sig.shape[0], _lib.ptr(idx), idx.size,
              ctypes.byref(r)))
    return _result(r)


LAPLACIAN, GRADIENT_SQUARED_NORM = 0, 1


def estimate_gpu(backend: CudaContext, tape, x, directions, estimator: int = LAPLACIAN,
                 weights=None) -> EstimatorResult:
    """``stde::estimate`` / ``stde::estimate_weighted`` (``src/stde/pipeline.rs:20-142``) with the
    ``Laplacian`` (2 c2) or ``GradientSquaredNorm`` (c1^2) estimator: jets on the GPU, the
    reference's Welford or West's weighted statistics on the host."""
    fn, dt = _fn(tape, "estimate")
    xx = np.ascontiguousarray(x, dtype=dt).ravel()
    V = np.ascontiguousarray(directions, dtype=dt).reshape(-1, xx.size)
    w = None if weights is None else np.ascontiguousarray(weights, dtype=dt).ravel()
    if w is not None and w.size != V.shape[0]:
        raise ValueError("weights.len() must match directions.len()")
    r = _lib.EstimatorResultC()
    _check(fn(backend._h, tape._h, _lib.ptr(xx), xx.size, int(estimator), _lib.ptr(V), V.shape[0], _lib.ptr(w),
              ctypes.byref(r)))
    return _result(r)


def dense_stde_2nd_gpu(backend: CudaContext, tape, x, cholesky, z_vectors) -> EstimatorResult:
    """``stde::dense_stde_2nd``: samples (L z)^T H (L z), L lower triangular [n, n]."""
    fn, dt = _fn(tape, "dense_stde_2nd")
    xx = np.ascontiguousarray(x, dtype=dt).ravel()
    L = np.ascontiguousarray(cholesky, dtype=dt).reshape(xx.size, xx.size)
    Z = np.ascontiguousarray(z_vectors, dtype=dt).reshape(-1, xx.size)
    r = _lib.EstimatorResultC()
    _check(fn(backend._h, tape._h, _lib.ptr(xx), xx.size, _lib.ptr(L), _lib.ptr(Z), Z.shape[0], ctypes.byref(r)))
    return _result(r)


def divergence_gpu(backend: CudaContext, tape, x, directions):
    """``stde::divergence``: (values, estimate of tr J from v^T J v samples)."""
    fn, dt = _fn(tape, "divergence")
    xx = np.ascontiguousarray(x, dtype=dt).ravel()
    V = np.ascontiguousarray(directions, dtype=dt).reshape(-1, xx.size)
    vals = np.zeros(xx.size, dt)
    r = _lib.EstimatorResultC()
    _check(fn(backend._h, tape._h, _lib.ptr(xx), xx.size, _lib.ptr(V), V.shape[0], _lib.ptr(vals), ctypes.byref(r)))
    return vals, _result(r)
