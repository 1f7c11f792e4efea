"""Shared test helpers: ULP distance with the reference's conventions and the
parity table of tests/gpu_cpu_parity.rs (echidna), as recorded tapes."""
from __future__ import annotations

import math

import numpy as np

from echidna_b200 import constant, record
from echidna_b200.rng import philox_bits  # noqa: F401  (re-exported for the tests)


def ulp_diff(a, b, dtype=np.float64):
    """ULP distance; both-NaN match, +-Inf must match exactly (gpu_cpu_parity.rs:646-695)."""
    a = np.asarray(a, dtype=dtype)
    b = np.asarray(b, dtype=dtype)
    ibits = np.int64 if dtype == np.float64 else np.int32
    ubits = np.uint64 if dtype == np.float64 else np.uint32
    big = np.iinfo(np.uint64).max if dtype == np.float64 else np.iinfo(np.uint32).max
    out = np.zeros(a.shape, dtype=np.float64)
    for idx in np.ndindex(a.shape):
        x, y = a[idx], b[idx]
        if not np.isfinite(x) or not np.isfinite(y):
            if np.isnan(x) and np.isnan(y):
                out[idx] = 0
            else:
                out[idx] = 0 if x.view(ubits) == y.view(ubits) else float(big)
            continue
        xb = int(x.view(ubits))
        yb = int(y.view(ubits))
        sign = 1 << (63 if dtype == np.float64 else 31)
        if (xb ^ yb) & sign == 0:
            out[idx] = abs(xb - yb)
        else:
            out[idx] = (xb & (sign - 1)) + (yb & (sign - 1))
    return out


def _r(f, x):
    return lambda: record(f, x)


NAN = float("nan")

# name, builder, points, f32_ulp, f64_ulp — tests/gpu_cpu_parity.rs:208-644
PARITY_CASES = [
    ("add", _r(lambda v: v[0] + v[1], [1.0, 1.0]), [[1.0, 1.0], [-3.5, 2.25], [1e10, 1e-10], [0.0, 0.0]], 2, 2),
    ("sub", _r(lambda v: v[0] - v[1], [1.0, 1.0]), [[1.0, 1.0], [-3.5, 2.25], [2.0, -1.5]], 4, 4),
    ("mul", _r(lambda v: v[0] * v[1], [1.0, 1.0]), [[1.0, 1.0], [-2.5, 4.0], [1e10, 1e-10], [0.0, 5.0]], 2, 2),
    ("div", _r(lambda v: v[0] / v[1], [1.0, 1.0]), [[1.0, 2.0], [-6.0, 3.0], [1.0, 1e-3]], 4, 4),
    ("sqrt", _r(lambda v: v[0].sqrt(), [1.0]), [[1.0], [4.0], [0.25], [1e6], [0.0]], 4, 4),
    ("cbrt", _r(lambda v: v[0].cbrt(), [1.0]), [[1.0], [8.0], [-27.0], [0.0]], 8, 8),
    ("one_div_x", _r(lambda v: constant(1.0) / v[0], [1.0]), [[1.0], [2.0], [-0.5]], 4, 4),
    ("recip", _r(lambda v: v[0].powi(-1), [2.0]), [[2.0], [-0.5], [0.0]], 4, 4),
    ("neg", _r(lambda v: -v[0], [1.0]), [[1.0], [-3.5], [0.0]], 0, 0),
    ("abs", _r(lambda v: v[0].abs(), [1.0]), [[1.0], [-3.5], [2.0], [0.0]], 0, 0),
    ("exp", _r(lambda v: v[0].exp(), [1.0]), [[0.0], [1.0], [-1.0], [5.0], [1000.0]], 8, 8),
    ("expm1", _r(lambda v: v[0].exp_m1(), [1.0]), [[0.0], [1e-6], [0.5], [-2.0]], 16, 8),
    ("ln", _r(lambda v: v[0].ln(), [1.0]), [[1.0], [2.0], [10.0], [0.5], [0.0]], 8, 8),
    ("ln1p", _r(lambda v: v[0].ln_1p(), [1.0]), [[0.0], [1e-6], [1.0], [-0.5], [-1.0]], 16, 8),
    ("sin", _r(lambda v: v[0].sin(), [1.0]), [[0.0], [0.5], [1.0], [-0.3]], 16, 16),
    ("cos", _r(lambda v: v[0].cos(), [1.0]), [[0.0], [0.5], [1.0], [-0.3]], 16, 16),
    ("tan", _r(lambda v: v[0].tan(), [0.5]), [[0.0], [0.5], [-0.5]], 16, 16),
    ("atan", _r(lambda v: v[0].atan(), [1.0]), [[0.0], [1.0], [-2.5], [100.0]], 8, 8),
    ("atan2", _r(lambda v: v[0].atan2(v[1]), [1.0, 1.0]),
     [[1.0, 1.0], [-1.0, 1.0], [3.0, 4.0], [1e10, 1e10], [0.0, 0.0]], 16, 16),
    ("sinh", _r(lambda v: v[0].sinh(), [1.0]), [[0.0], [1.0], [-2.0], [1000.0]], 16, 16),
    ("cosh", _r(lambda v: v[0].cosh(), [1.0]), [[0.0], [1.0], [-2.0], [1000.0]], 16, 16),
    ("tanh", _r(lambda v: v[0].tanh(), [1.0]), [[0.0], [1.0], [-2.0]], 16, 16),
    ("asinh", _r(lambda v: v[0].asinh(), [1.0]), [[0.0], [1.0], [-3.0], [1e6], [1e20], [-1e20]], 16, 16),
    ("acosh", _r(lambda v: v[0].acosh(), [2.0]), [[1.5], [2.0], [10.0], [1.0], [1e20]], 16, 16),
    ("atanh", _r(lambda v: v[0].atanh(), [0.5]), [[0.0], [0.25], [-0.5], [0.9], [1.0], [-1.0]], 16, 16),
    ("asin", _r(lambda v: v[0].asin(), [0.5]), [[0.0], [0.5], [-0.25], [1.0], [-1.0]], 16, 16),
    ("acos", _r(lambda v: v[0].acos(), [0.5]), [[0.0], [0.5], [-0.25], [1.0], [-1.0]], 16, 16),
    ("exp2", _r(lambda v: v[0].exp2(), [1.0]), [[0.0], [1.0], [-1.0], [3.0]], 8, 8),
    ("log2", _r(lambda v: v[0].log2(), [1.0]), [[1.0], [2.0], [8.0], [0.0]], 8, 8),
    ("log10", _r(lambda v: v[0].log10(), [1.0]), [[1.0], [10.0], [100.0], [0.0]], 8, 8),
    ("powi", _r(lambda v: v[0].powi(3), [2.0]), [[2.0], [-3.0], [0.5], [0.0]], 8, 8),
    ("powf", _r(lambda v: v[0].powf(constant(2.5)), [2.0]), [[2.0], [0.5], [10.0]], 32, 16),
    ("powf_int", _r(lambda v: v[0].powf(constant(3.0)), [2.0]), [[2.0], [-2.0], [-3.0], [0.0]], 16, 16),
    ("powf_var", _r(lambda v: v[0].powf(v[1]), [2.0, 2.0]), [[2.0, 3.0], [0.0, 0.0], [0.0, 2.0], [0.0, 3.0]], 16, 16),
    ("rem", _r(lambda v: v[0] % v[1], [5.0, 2.0]),
     [[5.0, 2.0], [7.5, 2.5], [-3.0, 2.0], [5.0, 0.0], [1e6, 3.0]], 4, 4),
    ("hypot", _r(lambda v: v[0].hypot(v[1]), [3.0, 4.0]),
     [[3.0, 4.0], [1e10, 1e10], [1.0, 0.0], [0.0, 1e-6], [0.0, 0.0]], 8, 8),
    ("max", _r(lambda v: v[0].max(v[1]), [1.0, 2.0]),
     [[1.0, 2.0], [-1.0, -2.0], [3.0, 3.0], [NAN, 1.0], [1.0, NAN]], 0, 0),
    ("min", _r(lambda v: v[0].min(v[1]), [1.0, 2.0]),
     [[1.0, 2.0], [-1.0, -2.0], [3.0, 3.0], [NAN, 1.0], [1.0, NAN]], 0, 0),
    ("rosenbrock", _r(lambda v: (constant(1.0) - v[0]) * (constant(1.0) - v[0])
                      + constant(100.0) * (v[1] - v[0] * v[0]) * (v[1] - v[0] * v[0]), [1.0, 1.0]),
     [[1.0, 1.0], [0.0, 0.0], [-1.2, 1.0]], 64, 32),
    ("sin_x2_mul_exp_neg_x", _r(lambda v: (v[0] * v[0] + constant(1.0)).sin() * (-v[0]).exp(), [1.0]),
     [[0.5], [1.0], [-0.5]], 64, 32),
    ("log_sum_exp", _r(lambda v: (v[0].exp() + v[1].exp()).ln(), [1.0, 0.5]),
     [[0.0, 0.0], [1.0, -1.0], [3.0, 5.0]], 64, 32),
]


def rosenbrock_2(v):
    """f(x, y) = (x-1)^2 + 100(y - x^2)^2 as written in tests/gpu_cuda_tests.rs:17-23."""
    one = constant(1.0)
    hundred = constant(100.0)
    dx = v[0] - one
    t = v[1] - v[0] * v[0]
    return dx * dx + hundred * t * t

