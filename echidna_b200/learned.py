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

    def gradients(self, x, q):
        """(loss, [g_w1, g_b1, g_w2, g_b2, g_w3, g_b3]) of the mean cross-entropy on
        device tensors x, q: the step ``train_step`` would take, not applied."""
        grads = [np.empty(s, np.float32) for s in self.shapes]
        loss = ctypes.c_float(0.0)
        _check(_lib.load().ech_mlp_gradients(self._h, x.data_ptr(), q.data_ptr(), int(x.shape[0]),
                                             *[_lib.ptr(a) for a in grads], ctypes.byref(loss)))
        return float(loss.value), grads

    def probs(self, x, out=None, stream=None):
        """softmax(MLP(x)) for a device tensor x [B, n_in], on torch's current stream
        unless ``stream`` is given."""
        import torch
        B = int(x.shape[0])
        if out is None:
            out = torch.empty((B, self.n_out), dtype=torch.float32, device=x.device)
        if stream is None:
            stream = torch.cuda.current_stream().cuda_stream
        _check(_lib.load().ech_mlp_forward(self._h, x.data_ptr(), B, out.data_ptr(), ctypes.c_void_p(stream)))
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


_RESULT_DTYPE = [("value", "f8"), ("estimate", "f8"), ("sample_variance", "f8"), ("standard_error", "f8"),
                 ("num_samples", "u8")]


def _stream(stream):
    """The CUDA stream to enqueue on: torch's current stream unless one is given,
    so the engine's work is ordered with the torch ops around it."""
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return stream


def _settle(ctx, stream):
    """Stream handle 0 means the context's own stream to the C ABI; wait for it so
    that later work on torch's default stream sees the results."""
    if stream == 0:
        _check(_lib.load().ech_ctx_synchronize(ctx._h))


def hessian_diagonals(ctx, tape, X, stream=None):
    """Exact Hessian diagonals of every row of the device tensor X [B, n]
    (``ech_hessian_diagonal_batch_device``); returns a device tensor [B, n]."""
    import torch
    out = torch.empty_like(X)
    st = _stream(stream)
    _check(_lib.load().ech_hessian_diagonal_batch_device(ctx._h, tape._h, int(tape.f64), X.data_ptr(), X.shape[0],
                                                         out.data_ptr(), ctypes.c_void_p(st)))
    _settle(ctx, st)
    return out


def sparse_trace(ctx, tape, X, probs, num_samples: int, seed: int, results=None, stream=None):
    """Per-row sparse STDE trace estimates (``ech_sparse_trace_batch_device``): coordinates
    drawn from ``probs`` [B, n] (fp32 device tensor) or uniformly (``probs=None``).
    Returns a device tensor of B estimator records (5 float64 words each)."""
    import torch
    B = int(X.shape[0])
    if results is None:
        results = torch.empty((B, 5), dtype=torch.float64, device=X.device)
    st = _stream(stream)
    _check(_lib.load().ech_sparse_trace_batch_device(
        ctx._h, tape._h, int(tape.f64), X.data_ptr(), B, None if probs is None else probs.data_ptr(),
        int(num_samples), ctypes.c_uint64(seed & 0xFFFFFFFFFFFFFFFF), results.data_ptr(), ctypes.c_void_p(st)))
    _settle(ctx, st)
    return results


def as_records(results) -> np.ndarray:
    """Device result tensor -> structured numpy array (value, estimate, ..., num_samples)."""
    raw = results.cpu().numpy()
    out = np.zeros(raw.shape[0], dtype=_RESULT_DTYPE)
    for k, (name, _) in enumerate(_RESULT_DTYPE[:4]):
        out[name] = raw[:, k]
    out["num_samples"] = raw[:, 4].view(np.uint64)
    return out


def target_distribution(diag):
    """q_j = |H_jj| / sum_k |H_kk| per row (device tensors)."""
    a = diag.abs().double()
    return (a / a.sum(dim=1, keepdim=True).clamp_min(1e-300)).float()


def samples_to_tolerance(diag, probs, rel: float = 0.01):
    """Samples an importance-sampled trace estimator needs for a relative standard
    error of ``rel``: per-sample variance sum_j d_j^2 / p_j - T^2 over (rel*T)^2.
    ``probs=None`` is the uniform proposal (p_j = 1/n).  Rows of float64 numpy arrays."""
    d = np.asarray(diag, dtype=np.float64)
    n = d.shape[1]
    T = d.sum(axis=1)
    if probs is None:
        second = n * (d * d).sum(axis=1)
    else:
        p = np.asarray(probs, dtype=np.float64)
        p = p / p.sum(axis=1, keepdims=True)
        second = (d * d / np.maximum(p, 1e-300)).sum(axis=1)
    var = np.maximum(second - T * T, 0.0)
    return var / (rel * T) ** 2, var, T


def exact_diagonals(ctx, tape64, X64, chunk: int = 4096):
    """Exact FP64 Hessian diagonals of the rows of X64 [N, n], in chunks."""
    import torch
    parts = [hessian_diagonals(ctx, tape64, X64[i:i + chunk].contiguous()) for i in range(0, X64.shape[0], chunk)]
    return torch.cat(parts)


def diagonal_coloring(pattern):
    """Colors the coordinates so that no two of one color interact: H_jk = 0 for
    every j != k of the same color.  Then, with v_c the indicator vector of color
    c, (H v_c)_j = H_jj for every j of color c, and one HVP per color yields the
    exact diagonal.  Greedy in index order over the structural pattern of
    ``sparse.detect_sparsity`` (a distance-1 coloring of the Hessian's graph; the
    reference's distance-2 ``greedy_coloring``, ``src/sparse.rs:57-98``, is also
    valid here but may use more colors).  Returns (colors [n] uint32, count)."""
    n = int(pattern.dim)
    r = np.asarray(pattern.rows, np.int64)
    c = np.asarray(pattern.cols, np.int64)
    off = r != c
    nbrs = [[] for _ in range(n)]
    for a, b in zip(r[off].tolist(), c[off].tolist()):
        nbrs[a].append(b)
        nbrs[b].append(a)
    colors = np.full(n, -1, np.int64)
    for j in range(n):
        used = {int(colors[k]) for k in nbrs[j] if colors[k] >= 0}
        col = 0
        while col in used:
            col += 1
        colors[j] = col
    return colors.astype(np.uint32), int(colors.max() + 1) if n else 0


def colored_diagonals(ctx, tape64, X64, coloring, chunk: int = 65536, stream=None):
    """Exact FP64 Hessian diagonals of the rows of the device tensor X64 [N, n]
    from one per-point HVP (forward-over-reverse, ``ech_hvp_batch_device``) per
    color of ``coloring`` (``diagonal_coloring``): every diagonal entry is read
    from the HVP of its own color, whose other coordinates do not interact with
    it.  A tridiagonal Hessian takes two HVPs per point instead of n jets.
    Returns a device tensor [N, n]; work runs on torch's current stream."""
    import torch
    colors, nc = coloring
    N, n = int(X64.shape[0]), int(X64.shape[1])
    out = torch.empty_like(X64)
    if N == 0 or nc == 0:
        return out.zero_()
    dev = X64.device
    col_t = torch.as_tensor(np.asarray(colors, np.int64), device=dev)
    seeds = torch.zeros((nc, n), dtype=torch.float64, device=dev)
    seeds[col_t, torch.arange(n, device=dev)] = 1.0
    masks = [col_t == k for k in range(nc)]
    st = _stream(stream)
    lib = _lib.load()
    b_max = min(chunk, N)
    dirs = torch.empty((nc, b_max, n), dtype=torch.float64, device=dev)
    for k in range(nc):
        dirs[k].copy_(seeds[k].expand(b_max, n))
    grads = torch.empty((b_max, n), dtype=torch.float64, device=dev)
    hv = torch.empty((b_max, n), dtype=torch.float64, device=dev)
    for i in range(0, N, b_max):
        b = min(b_max, N - i)
        xs = X64[i:i + b].contiguous()
        for k in range(nc):
            _check(lib.ech_hvp_batch_device(ctx._h, tape64._h, 1, xs.data_ptr(), 1, dirs[k].data_ptr(), b,
                                            grads.data_ptr(), hv.data_ptr(), ctypes.c_void_p(st)))
            _settle(ctx, st)
            out[i:i + b, masks[k]] = hv[:b, masks[k]]
    return out


def train_proposal(ctx, tape64, X64, hidden: int = 256, steps: int = 400, batch: int = 256, lr: float = 1e-3,
                   seed: int = 0):
    """Trains the proposal on exact diagonals of the training points X64 [N, n]
    (FP64 labels from the tape's own jets); returns (mlp, losses)."""
    import torch
    n = int(X64.shape[1])
    q = target_distribution(exact_diagonals(ctx, tape64, X64))
    xf = X64.float()
    mlp = ProposalMLP(ctx, n, hidden, n, seed=seed)
    g = torch.Generator(device=X64.device).manual_seed(seed)
    losses = []
    for _ in range(steps):
        rows = torch.randint(0, X64.shape[0], (batch,), device=X64.device, generator=g)
        losses.append(mlp.train_step(xf[rows].contiguous(), q[rows].contiguous(), lr=lr))
    return mlp, losses
