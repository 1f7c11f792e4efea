"""Many tapes in one persistent launch: results equal the per-tape HVP sweep,
bit for bit, and the launch replays from a captured CUDA graph."""
import numpy as np
import pytest

from echidna_b200 import _lib, configs
from echidna_b200.gpu import GpuTapeData, MultiTapeHvp

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _suite(ctx, f64):
    suite = configs.uneven_suite(count=12, seed=77, max_points=3000, max_len=3000, max_dim=48)
    dt = torch.float64 if f64 else torch.float32
    rng = np.random.default_rng(5)
    jobs = []
    for name, tape, n in suite:
        gt = ctx.upload_tape_f64(tape) if f64 else ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
        ni = tape.num_inputs
        x = torch.tensor(rng.uniform(-1, 1, size=(n, ni)), dtype=dt, device="cuda")
        v = torch.tensor(rng.choice([-1.0, 1.0], size=(n, ni)), dtype=dt, device="cuda")
        g = torch.full((n * ni,), float("nan"), dtype=dt, device="cuda")
        h = torch.full((n * ni,), float("nan"), dtype=dt, device="cuda")
        jobs.append((name, gt, n, x, v, g, h))
    return jobs


def _reference(ctx, jobs, f64):
    lib = _lib.load()
    out = []
    for name, gt, n, x, v, _, _ in jobs:
        g = torch.empty_like(x).reshape(-1)
        h = torch.empty_like(x).reshape(-1)
        st = lib.ech_hvp_batch_device(ctx._h, gt._h, int(f64), x.data_ptr(), 1, v.data_ptr(), n, g.data_ptr(),
                                      h.data_ptr(), None)
        assert st == 0, _lib.last_error()
        out.append((g, h))
    assert lib.ech_ctx_synchronize(ctx._h) == 0, _lib.last_error()
    return out


@pytest.mark.parametrize("f64", [False, True])
def test_multi_matches_per_tape_launches(ctx, f64):
    jobs = _suite(ctx, f64)
    torch.cuda.synchronize()
    m = MultiTapeHvp(ctx, [(gt, x.data_ptr(), v.data_ptr(), n, g.data_ptr(), h.data_ptr())
                           for _, gt, n, x, v, g, h in jobs], f64=f64, autotune=True)
    info = m.info()
    assert info["jobs"] == len(jobs) and info["tuned"] == 1
    m.launch()
    assert _lib.load().ech_ctx_synchronize(ctx._h) == 0, _lib.last_error()
    ref = _reference(ctx, jobs, f64)
    for (name, _, _, _, _, g, h), (rg, rh) in zip(jobs, ref):
        assert torch.equal(g, rg), name
        assert torch.equal(h, rh), name
    m.close()


def test_multi_launch_replays_from_cuda_graph(ctx):
    jobs = _suite(ctx, False)
    torch.cuda.synchronize()
    m = MultiTapeHvp(ctx, [(gt, x.data_ptr(), v.data_ptr(), n, g.data_ptr(), h.data_ptr())
                           for _, gt, n, x, v, g, h in jobs], f64=False, autotune=False)
    m.launch()
    assert _lib.load().ech_ctx_synchronize(ctx._h) == 0
    first = [(g.clone(), h.clone()) for _, _, _, _, _, g, h in jobs]
    for _, _, _, _, _, g, h in jobs:
        g.fill_(float("nan"))
        h.fill_(float("nan"))
    s = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s, capture_error_mode="thread_local"):
        m.launch(s.cuda_stream)
    for _ in range(2):
        graph.replay()
    torch.cuda.synchronize()
    assert _lib.load().ech_ctx_synchronize(ctx._h) == 0
    for (g, h), (_, _, _, _, _, g2, h2) in zip(first, jobs):
        assert torch.equal(g, g2) and torch.equal(h, h2)
    del graph
    m.close()


def test_multi_rejects_mixed_precision(ctx):
    tape = configs.rosenbrock(4)
    g64 = ctx.upload_tape_f64(tape)
    x = torch.zeros(8, dtype=torch.float32, device="cuda")
    with pytest.raises(AssertionError, match="precision"):
        MultiTapeHvp(ctx, [(g64, x.data_ptr(), x.data_ptr(), 2, x.data_ptr(), x.data_ptr())], f64=False)
