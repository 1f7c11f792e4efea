"""Learned importance proposal for sparse STDE (extension; no reference counterpart).

Uniform sparse STDE (``stde::diagonal_kth_order_stochastic``,
``src/stde/higher_order.rs:173-227``) estimates ``tr(H) = sum_j H_jj`` as
``n * mean(H_jj)`` over uniformly sampled coordinates.  With a proposal ``p(x)``
over the coordinates the estimator ``mean_s(H_{J_s J_s} / p_{J_s})`` (``J_s ~ p``)
stays unbiased, and its variance falls as ``p_j`` approaches ``|H_jj| / sum_k |H_kk|``.
Here ``p(x)`` is a small softmax MLP trained on the GPU (``ech_mlp_*``: BF16
tcgen05 GEMMs, FP32 accumulation, Adam) on exact Hessian diagonals that the
tape's own order-2 jets produce.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .gpu import _check


class ProposalMLP:
    """softmax(W3 relu(W2 relu(W1 x + b1) + b2) + b3), row-major [out][in] weights."""

    def __init__(self, ctx, n_in: int, hidden: int, n_out: int, seed: int = 0):
        rng = np.random.default_rng(seed)

        def he(o, i):
            return (rng.normal(size=(o, i)) * np.sqrt(2.0 / i)).astype(np.float32)

        self.shapes = [(hidden, n_in), (hidden,), (hidden, hidden), (hidden,), (n_out, hidden), (n_out,)]
        w = [he(hidden, n_in), np.zeros(hidden, np.float32), he(hidden, hidden), np.zeros(hidden, np.float32),
             (he(n_out, hidden) * 0.1).astype(np.float32), np.zeros(n_out, np.float32)]
        self._keep = w
        h = ctypes.c_void_p()
        _check(_lib.load().ech_mlp_create(ctx._h, n_in, hidden, n_out, *[_lib.ptr(a) for a in w], ctypes.byref(h)))
        self._h = h
        self._ctx = ctx
        self.n_in, self.hidden, self.n_out = n_in, hidden, n_out
        ctx._children.append(self)

    def train_step(self, x, q, lr: float = 1e-3) -> float:
        """One Adam step on device tensors x [B, n_in], q [B, n_out] (rows sum to 1)."""
        loss = ctypes.c_float(0.0)
        _check(_lib.load().ech_mlp_train_step(self._h, x.data_ptr(), q.data_ptr(), int(x.shape[0]),
                                              ctypes.c_float(lr), ctypes.byref(loss)))
        return float(loss.value)

    def probs(self, x, out=None, stream: int = 0):
        import torch
        B = int(x.shape[0])
        if out is None:
            out = torch.empty((B, self.n_out), dtype=torch.float32, device=x.device)
        _check(_lib.load().ech_mlp_forward(self._h, x.data_ptr(), B, out.data_ptr(), ctypes.c_void_p(stream)))
        if stream == 0:
            torch.cuda.synchronize()
        return out

    def weights(self):
        arrs = [np.empty(s, np.float32) for s in self.shapes]
        _check(_lib.load().ech_mlp_get_weights(self._h, *[_lib.ptr(a) for a in arrs]))
        return arrs

    def close(self):
        if getattr(self, "_h", None) and getattr(self._ctx, "_h", None):
            _lib.load().ech_mlp_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
