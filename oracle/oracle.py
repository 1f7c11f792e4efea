"""ctypes binding for the oracle (test infrastructure only).

The oracle is the C++ restatement of the reference's CPU BytecodeTape sweeps in
``oracle/oracle.cpp``.  Only the tests, ``__graft_entry__.smoke()`` and bench.py's
CPU-baseline leg load it, and only as the checker.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class _TapeDesc(ctypes.Structure):
    _fields_ = [
        ("opcodes", ctypes.c_void_p),
        ("arg0", ctypes.c_void_p),
        ("arg1", ctypes.c_void_p),
        ("values", ctypes.c_void_p),
        ("num_variables", ctypes.c_uint32),
        ("num_inputs", ctypes.c_uint32),
        ("output_index", ctypes.c_uint32),
        ("output_indices", ctypes.c_void_p),
        ("num_outputs", ctypes.c_uint32),
    ]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
    return _lib


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else ctypes.c_void_p(0)


class OracleTape:
    """Keeps the numpy arrays alive for the descriptor handed to C."""

    def __init__(self, tape, dtype=None):
        dtype = np.dtype(dtype or tape.dtype)
        self.dtype = dtype
        self.suffix = "f64" if dtype == np.float64 else "f32"
        op, a0, a1, vals = tape.arrays()
        self.op, self.a0, self.a1 = op, a0, a1
        self.vals = np.ascontiguousarray(vals, dtype=dtype)
        self.outs = np.asarray(tape.all_output_indices(), dtype=np.uint32)
        self.ni = tape.num_inputs
        self.nout = len(self.outs)
        self.nv = len(op)
        self.desc = _TapeDesc(
            op.ctypes.data, a0.ctypes.data, a1.ctypes.data, self.vals.ctypes.data,
            self.nv, self.ni, tape.output_index, self.outs.ctypes.data, self.nout,
        )

    def _f(self, name):
        return getattr(lib(), f"orc_{name}_{self.suffix}")

    def _arr(self, x):
        return np.ascontiguousarray(x, dtype=self.dtype)

    # -- batch sweeps --
    def forward(self, X, nthreads=1):
        X = self._arr(X).reshape(-1, self.ni) if self.ni else self._arr(X).reshape(-1, 0)
        B = X.shape[0]
        out = np.empty((B, self.nout), dtype=self.dtype)
        self._f("forward")(ctypes.byref(self.desc), _p(X), ctypes.c_uint64(B), _p(out), nthreads)
        return out

    def gradient(self, X, nthreads=1):
        X = self._arr(X).reshape(-1, self.ni)
        B = X.shape[0]
        out = np.empty((B, self.nout), dtype=self.dtype)
        g = np.empty((B, self.ni), dtype=self.dtype)
        self._f("gradient")(ctypes.byref(self.desc), _p(X), ctypes.c_uint64(B), _p(out), _p(g), nthreads)
        return out, g

    def hvp(self, X, V, nthreads=1):
        """Per-point HVP; ``X`` may be a single point (broadcast) or ``[B, ni]``."""
        V = self._arr(V).reshape(-1, self.ni)
        B = V.shape[0]
        X = self._arr(X)
        per_point = 1 if X.size == B * self.ni and B > 1 or X.ndim == 2 else 0
        X = X.reshape(-1, self.ni)
        if X.shape[0] == 1 and B > 1:
            per_point = 0
        g = np.empty((B, self.ni), dtype=self.dtype)
        h = np.empty((B, self.ni), dtype=self.dtype)
        self._f("hvp")(ctypes.byref(self.desc), _p(X), _p(V), ctypes.c_uint64(B), per_point, _p(g), _p(h), nthreads)
        return g, h

    def jvp(self, X, V, nthreads=1):
        X = self._arr(X).reshape(-1, self.ni)
        V = self._arr(V).reshape(-1, self.ni)
        B = X.shape[0]
        val = np.empty((B, self.nout), dtype=self.dtype)
        tan = np.empty((B, self.nout), dtype=self.dtype)
        self._f("jvp")(ctypes.byref(self.desc), _p(X), _p(V), ctypes.c_uint64(B), _p(val), _p(tan), nthreads)
        return val, tan

    def taylor(self, P, S, order, nthreads=1):
        """Returns ``coeffs[k][b*nout + j]`` like ``TaylorKthBatchResult``."""
        P = self._arr(P).reshape(-1, self.ni)
        S = self._arr(S).reshape(-1, self.ni)
        B = P.shape[0]
        c = np.empty((order, B * self.nout), dtype=self.dtype)
        rc = self._f("taylor")(ctypes.byref(self.desc), order, _p(P), _p(S), ctypes.c_uint64(B), _p(c), nthreads)
        if rc != 0:
            raise ValueError(f"oracle: unsupported order {order}")
        return c

    def stde_sparse(self, x, dist, sampled_indices):
        """``stde::stde_sparse`` (``src/stde/sparse.rs:37-78``) at one point over a
        ``SparseSamplingDistribution`` (``echidna_b200.diffop``); returns
        (value, estimate, sample_variance, standard_error, num_samples)."""
        off, vars_, slots, coefs, kout, pref, sign = dist.flatten()
        coefs, pref, sign = (np.ascontiguousarray(a, dtype=self.dtype) for a in (coefs, pref, sign))
        x = self._arr(x).ravel()
        idx = np.ascontiguousarray(sampled_indices, dtype=np.uint64).ravel()
        K = int(kout.max()) + 1
        out = np.empty(5, dtype=self.dtype)
        z = (ctypes.c_double if self.dtype == np.float64 else ctypes.c_float)(float(dist.normalization()))
        rc = self._f("stde_sparse")(ctypes.byref(self.desc), K, _p(x), _p(off), _p(vars_), _p(slots), _p(coefs),
                                     _p(kout), _p(pref), _p(sign), z, _p(idx), ctypes.c_uint64(idx.size), _p(out))
        if rc != 0:
            raise ValueError(f"oracle: unsupported jet order {K}")
        return float(out[0]), float(out[1]), float(out[2]), float(out[3]), int(out[4])

    def hessian(self, x):
        x = self._arr(x)
        n = self.ni
        val = np.zeros(1, dtype=self.dtype)
        g = np.empty(n, dtype=self.dtype)
        H = np.empty((n, n), dtype=self.dtype)
        self._f("hessian")(ctypes.byref(self.desc), _p(x), _p(val), _p(g), _p(H))
        return val[0], g, H

    # -- STDE --
    def laplacian_stats_batch(self, X, dirs, nthreads=1):
        """``estimate(&Laplacian, ...)`` per point. ``dirs``: ``[S, n]`` shared or ``[B, S, n]``."""
        X = self._arr(X).reshape(-1, self.ni)
        B = X.shape[0]
        dirs = self._arr(dirs)
        per_point = 1 if dirs.ndim == 3 else 0
        S = dirs.shape[-2]
        out = np.empty((B, 5), dtype=self.dtype)
        self._f("laplacian_stats_batch")(ctypes.byref(self.desc), _p(X), _p(dirs), ctypes.c_uint64(B),
                                         ctypes.c_uint32(S), per_point, _p(out), nthreads)
        return out

    def laplacian(self, x, dirs):
        x = self._arr(x)
        dirs = self._arr(dirs).reshape(-1, self.ni)
        v = np.zeros(1, dtype=self.dtype)
        lap = np.zeros(1, dtype=self.dtype)
        self._f("laplacian")(ctypes.byref(self.desc), _p(x), _p(dirs), ctypes.c_uint32(dirs.shape[0]), _p(v), _p(lap))
        return v[0], lap[0]

    def hessian_diagonal(self, x):
        x = self._arr(x)
        v = np.zeros(1, dtype=self.dtype)
        d = np.empty(self.ni, dtype=self.dtype)
        self._f("hessian_diagonal")(ctypes.byref(self.desc), _p(x), _p(v), _p(d))
        return v[0], d

    def laplacian_with_control(self, x, dirs, control):
        x = self._arr(x)
        dirs = self._arr(dirs).reshape(-1, self.ni)
        control = self._arr(control)
        out = np.empty(5, dtype=self.dtype)
        self._f("laplacian_with_control")(ctypes.byref(self.desc), _p(x), _p(dirs), ctypes.c_uint32(dirs.shape[0]),
                                          _p(control), _p(out))
        return out

    def estimate_weighted(self, x, dirs, weights):
        x = self._arr(x)
        dirs = self._arr(dirs).reshape(-1, self.ni)
        w = self._arr(weights)
        out = np.empty(5, dtype=self.dtype)
        rc = self._f("estimate_weighted")(ctypes.byref(self.desc), _p(x), _p(dirs), ctypes.c_uint32(dirs.shape[0]),
                                          _p(w), _p(out))
        if rc != 0:
            raise ValueError("estimate_weighted: weights must be non-negative and non-NaN")
        return out

    def diagonal_kth_order_stochastic(self, x, k, indices):
        x = self._arr(x)
        idx = np.ascontiguousarray(indices, dtype=np.uint64)
        out = np.empty(5, dtype=self.dtype)
        rc = self._f("diagonal_kth_order_stochastic")(ctypes.byref(self.desc), _p(x), ctypes.c_uint32(k), _p(idx),
                                                      ctypes.c_uint64(len(idx)), _p(out))
        if rc != 0:
            raise ValueError("unsupported k")
        return out


def hardware_threads() -> int:
    return int(lib().orc_hardware_threads())
