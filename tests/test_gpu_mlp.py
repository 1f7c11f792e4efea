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


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (256, 256, 1024), (200, 384, 256), (64, 1024, 128)])
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
