"""Sparse STDE with a learned proposal: exact diagonals, unbiased importance-
sampled traces, and the proposal's variance reduction over uniform sampling."""
import numpy as np
import pytest

from echidna_b200 import configs
from echidna_b200.gpu import GpuTapeData
from echidna_b200.learned import (as_records, colored_diagonals, diagonal_coloring, exact_diagonals,
                                  samples_to_tolerance, sparse_trace, train_proposal)
from echidna_b200.sparse import detect_sparsity
from oracle.oracle import OracleTape

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def test_hessian_diagonal_batch_matches_oracle(ctx):
    tape = configs.softplus_chain(64)
    gt = ctx.upload_tape_f64(tape)
    X = np.random.default_rng(1).normal(size=(6, 64))
    got = exact_diagonals(ctx, gt, torch.tensor(X, device="cuda")).cpu().numpy()
    o = OracleTape(tape)
    for b in range(6):
        ref = np.diag(o.hessian(X[b])[2])
        assert np.allclose(got[b], ref, rtol=1e-10, atol=1e-10 * np.abs(ref).max())


@pytest.mark.parametrize("n", [2, 3, 64, 1024])
def test_colored_diagonals_match_jets_and_oracle(ctx, n):
    # the training labels: two HVPs per point (the softplus chain's Hessian is tridiagonal)
    # against the n order-3 jets per point and, for small n, the oracle's dense Hessian
    tape = configs.softplus_chain(n)
    gt = ctx.upload_tape_f64(tape)
    coloring = diagonal_coloring(detect_sparsity(tape))
    assert coloring[1] == (1 if n == 1 else 2)
    B = 300 if n <= 64 else 40
    X = torch.tensor(np.random.default_rng(5).normal(size=(B, n)), device="cuda")
    got = colored_diagonals(ctx, gt, X, coloring, chunk=128).cpu().numpy()
    jets = exact_diagonals(ctx, gt, X).cpu().numpy()
    scale = np.abs(jets).max(axis=1, keepdims=True)
    assert np.all(np.abs(got - jets) <= 1e-12 * scale)
    if n <= 64:
        o = OracleTape(tape)
        for b in range(0, B, 37):
            ref = np.diag(o.hessian(X[b].cpu().numpy())[2])
            assert np.allclose(got[b], ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("learned", [False, True])
def test_sparse_trace_is_unbiased(ctx, learned):
    # many points x 64 samples: standardised errors (est - T) / SE have mean ~0, spread ~1
    n = 64
    tape = configs.softplus_chain(n)
    gt = ctx.upload_tape_f64(tape)
    rng = np.random.default_rng(2)
    X = torch.tensor(rng.normal(size=(1024, n)), device="cuda")
    d = exact_diagonals(ctx, gt, X)
    probs = None
    if learned:  # any strictly positive proposal keeps the estimator unbiased
        a = d.abs().float() + 0.1 * d.abs().float().mean(dim=1, keepdim=True)
        probs = (a / a.sum(dim=1, keepdim=True)).contiguous()
    r = as_records(sparse_trace(ctx, gt, X, probs, 64, seed=9))
    torch.cuda.synchronize()
    T = d.sum(dim=1).cpu().numpy()
    z = (r["estimate"] - T) / np.maximum(r["standard_error"], 1e-300)
    assert np.all(r["num_samples"] == 64)
    assert abs(np.mean(z)) < 0.2
    assert 0.7 < np.std(z) < 1.4


def test_learned_proposal_beats_uniform(ctx):
    n = 128
    tape = configs.softplus_chain(n)
    gt = ctx.upload_tape_f64(tape)
    rng = np.random.default_rng(3)
    Xtr = torch.tensor(rng.normal(size=(4096, n)), device="cuda")
    mlp, losses = train_proposal(ctx, gt, Xtr, hidden=128, steps=300, batch=256, lr=2e-3, seed=4)
    assert losses[-1] < losses[0]
    Xev = torch.tensor(rng.normal(size=(256, n)), device="cuda")
    d = exact_diagonals(ctx, gt, Xev).cpu().numpy()
    p = mlp.probs(Xev.float()).cpu().numpy()
    s_uniform, _, _ = samples_to_tolerance(d, None)
    s_learned, _, _ = samples_to_tolerance(d, p)
    # the best any proposal can do here: p_j = |H_jj| / sum |H_kk| (mixed signs keep it above 0)
    s_best, _, _ = samples_to_tolerance(d, np.abs(d) / np.abs(d).sum(axis=1, keepdims=True))
    print("median samples to 1%: uniform", np.median(s_uniform), "learned", np.median(s_learned),
          "best", np.median(s_best))
    assert np.median(s_learned) < np.median(s_uniform) / 2.5
    assert np.median(s_learned) < 2.0 * np.median(s_best)
