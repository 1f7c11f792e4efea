"""The tcgen05 BF16 GEMM and the proposal MLP trained with it.

GEMM results are compared with an FP32 torch matmul of the same BF16-rounded
operands: both accumulate in FP32, so they differ only by summation order
(relative 1e-3 of the row scale).  The MLP's loss must fall on a fixed task.
"""
import ctypes

import numpy as np
import pytest

from echidna_b200 import _lib

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _gemm(ctx, A, B, bias=None):
    M, K = A.shape
    N = B.shape[0]
    C = torch.full((M, N), float("nan"), dtype=torch.float32, device="cuda")
    lib = _lib.load()
    st = lib.ech_gemm_bf16(ctx._h, A.data_ptr(), B.data_ptr(), C.data_ptr(),
                           None if bias is None else bias.data_ptr(), M, N, K, K, K, N, None)
    assert st == 0, _lib.last_error()
    torch.cuda.synchronize()
    assert lib.ech_ctx_synchronize(ctx._h) == 0, _lib.last_error()
    return C


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (256, 256, 1024), (200, 384, 256), (64, 1024, 128),
                                   (1024, 1280, 256), (1000, 1200, 192), (4096, 4096, 64), (4096, 4096, 1024),
                                   (2000, 4000, 128), (256, 1030, 64)])
def test_gemm_bf16_matches_fp32_matmul(ctx, M, N, K):
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    bias = torch.randn(N, device="cuda", generator=g)
    C = _gemm(ctx, A, B, bias)
    ref = A.float() @ B.float().T + bias
    scale = ref.abs().max().item()
    assert torch.isfinite(C).all()
    assert (C - ref).abs().max().item() <= 1e-3 * max(1.0, scale)


def test_mlp_learns_a_fixed_proposal(ctx):
    from echidna_b200.learned import ProposalMLP
    rng = np.random.default_rng(3)
    n_in, n_out, B = 128, 128, 256
    # target: a fixed, heavily non-uniform distribution (log-uniform weights)
    w = np.exp(rng.uniform(np.log(1e-3), np.log(1e3), size=n_out))
    q = np.tile(w / w.sum(), (B, 1)).astype(np.float32)
    x = rng.normal(size=(B, n_in)).astype(np.float32)
    mlp = ProposalMLP(ctx, n_in, 64, n_out, seed=1)
    dx, dq = torch.from_numpy(x).cuda(), torch.from_numpy(q).cuda()
    losses = [mlp.train_step(dx, dq, lr=3e-3) for _ in range(300)]
    entropy = float(-(q[0] * np.log(q[0])).sum())
    assert losses[-1] < losses[0]
    assert losses[-1] - entropy < 0.05 * (losses[0] - entropy) + 0.02
    p = mlp.probs(dx).cpu().numpy()
    assert np.allclose(p.sum(axis=1), 1.0, atol=1e-4)


def _bf(a):
    """Round to BF16 (round to nearest even, as __float2bfloat16_rn) and back, in float64."""
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(torch.bfloat16).double().numpy()


def _emulate(x, q, w):
    """The kernels' dataflow in float64: BF16 operands wherever a GEMM reads them
    (x, weights, activations after ReLU, the loss gradient and the back-propagated
    pre-activation gradients), exact products and sums otherwise."""
    W1, b1, W2, b2, W3, b3 = [np.asarray(a, np.float64) for a in w]
    B = x.shape[0]
    xb = _bf(x)
    z1 = xb @ _bf(W1).T + b1
    h1b = _bf(np.maximum(z1, 0.0))
    z2 = h1b @ _bf(W2).T + b2
    h2b = _bf(np.maximum(z2, 0.0))
    logits = h2b @ _bf(W3).T + b3
    m = logits.max(axis=1, keepdims=True)
    logp = logits - m - np.log(np.exp(logits - m).sum(axis=1, keepdims=True))
    p = np.exp(logp)
    loss = float(-(q * logp).sum() / B)
    dl = (p - q) / B
    dlb = _bf(dl)
    g_w3, g_b3 = dlb.T @ h2b, dl.sum(axis=0)
    dz2 = (dlb @ _bf(W3)) * (z2 > 0)
    dz2b = _bf(dz2)
    g_w2, g_b2 = dz2b.T @ h1b, dz2.sum(axis=0)
    dz1 = (dz2b @ _bf(W2)) * (z1 > 0)
    g_w1, g_b1 = _bf(dz1).T @ xb, dz1.sum(axis=0)
    return loss, [g_w1, g_b1, g_w2, g_b2, g_w3, g_b3]


def _autograd(x, q, w):
    """torch FP32 autograd of the BF16-rounded forward: x, the weights and the
    activations the GEMMs read are rounded to BF16 (the activations with an
    identity gradient); the backward runs in FP32 with no rounding."""
    ws = [torch.tensor(_bf(a) if a.ndim == 2 else a, dtype=torch.float32, requires_grad=True) for a in w]
    W1, b1, W2, b2, W3, b3 = ws

    def rnd(t):
        return t + (t.to(torch.bfloat16).float() - t).detach()
    xt = torch.tensor(_bf(x), dtype=torch.float32)
    h = rnd(torch.relu(xt @ W1.T + b1))
    h = rnd(torch.relu(h @ W2.T + b2))
    logp = torch.log_softmax(h @ W3.T + b3, dim=1)
    loss = -(torch.tensor(q) * logp).sum() / x.shape[0]
    loss.backward()
    return float(loss.detach()), [t.grad.double().numpy() for t in ws]


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def test_mlp_backward_and_adam_against_host(ctx):
    """C5 proposal shape (1024 -> 256 -> 256 -> 1024), batch 256: the GPU's loss and
    every weight / bias gradient against (a) a float64 emulation of the kernels'
    dataflow (norm-relative 2e-3: FP32 accumulation, plus the rare BF16 rounding
    that falls the other way), (b) torch FP32 autograd of the BF16-rounded forward
    (norm-relative 1e-2: the kernels also round the back-propagated gradients the
    GEMMs read to BF16, 2^-9 relative per element); then one Adam step against the
    update computed on the host from the GPU's gradients (within 2 ulp)."""
    from echidna_b200.learned import ProposalMLP
    rng = np.random.default_rng(11)
    n_in, hidden, n_out, B = 1024, 256, 1024, 256
    x = rng.normal(size=(B, n_in)).astype(np.float32)
    a = np.exp(rng.uniform(np.log(1e-3), np.log(1e3), size=(B, n_out)))
    q = (a / a.sum(axis=1, keepdims=True)).astype(np.float32)
    mlp = ProposalMLP(ctx, n_in, hidden, n_out, seed=5)
    w0 = mlp.weights()
    dx, dq = torch.from_numpy(x).cuda(), torch.from_numpy(q).cuda()
    loss, grads = mlp.gradients(dx, dq)
    e_loss, e_grads = _emulate(x, q, w0)
    a_loss, a_grads = _autograd(x, q, w0)
    assert abs(loss - e_loss) <= 1e-4 * abs(e_loss)
    assert abs(loss - a_loss) <= 1e-3 * abs(a_loss)
    names = ["w1", "b1", "w2", "b2", "w3", "b3"]
    for name, g, eg, ag in zip(names, grads, e_grads, a_grads):
        assert np.isfinite(g).all(), name
        assert _rel(g, eg) <= 2e-3, (name, _rel(g, eg))
        assert _rel(g, ag) <= 1e-2, (name, _rel(g, ag))
    # the gradients are those of the step: one Adam step from the same state
    lr = 1e-3
    mlp.train_step(dx, dq, lr=lr)
    w1 = mlp.weights()
    b1_, b2_, eps = np.float32(0.9), np.float32(0.999), np.float32(1e-8)
    c1, c2 = np.float32(1) - b1_, np.float32(1) - b2_
    for name, w_old, g, w_new in zip(names, w0, grads, w1):
        m = (np.float32(1) - b1_) * g
        v = (np.float32(1) - b2_) * g * g
        want = w_old - np.float32(lr) * (m / c1) / (np.sqrt(v / c2) + eps)
        np.testing.assert_array_max_ulp(w_new, want.astype(np.float32), maxulp=2)
    mlp.close()
