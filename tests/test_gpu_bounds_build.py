"""The device bounds-checked build (libechidna_b200_bounds.so, -DECH_DEVICE_BOUNDS).

compute-sanitizer is closed on this pool, so the engine carries its own checks:
in the checked build every slot access of the sweeps is tested against its
region (shared registers, global far slots, trajectory) and every input,
output and gradient index against the unit's sizes; a miss sets an error bit
that ech_ctx_synchronize reports, and the access goes to a valid location
instead.  A child process runs the benchmarked kinds of sweeps on the checked
build — narrow shapes with the trajectory in shared memory, tuned MLP shapes,
dense groups, input-direct jets with device signs and shared directions, the
many-tape launch, the allocation-free gradient — and must finish with a clean
error word and results equal, bit for bit, to the ordinary build's.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import ctypes, sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[2])
from echidna_b200 import _lib, configs
from echidna_b200.gpu import CudaContext, GpuTapeData, MultiTapeHvp
from echidna_b200.stde_gpu import DIR_RADEMACHER, DIR_SHARED, laplacian_batch

lib = _lib.load()
ctx = CudaContext.new(0)
out = {}
rng = np.random.default_rng(0xB0)

t = configs.rosenbrock(100)
g = ctx.upload_tape_f64(t)
X = rng.uniform(-2, 2, size=(1024, 100))
out["rosen_v"], out["rosen_g"] = ctx.gradient_batch_f64(g, X, 1024)

t = configs.mlp(64, 64)
g = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(t))
X = rng.normal(size=(20000, 64)).astype(np.float32)
V = rng.choice([-1.0, 1.0], size=(20000, 64)).astype(np.float32)
for _ in range(2):
    out["mlp_v"], out["mlp_g"] = ctx.gradient_batch(g, X, 20000)
    out["mlp_hg"], out["mlp_hv"] = ctx.hvp_batch_points(g, X, V, 20000)

t = configs.logsumexp_tanh(48, 64)
g = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(t))
X = rng.normal(size=(600, 48)).astype(np.float32)
r = laplacian_batch(ctx, g, X, 16, None, DIR_RADEMACHER, seed=3)
out["stde_rad"] = np.stack([r["estimate"], r["sample_variance"]])
D = rng.choice([-1.0, 1.0], size=(16, 48)).astype(np.float32)
r = laplacian_batch(ctx, g, X, 16, D, DIR_SHARED)
out["stde_shared"] = np.stack([r["estimate"], r["sample_variance"]])

suite = configs.uneven_suite(count=9, seed=41, max_points=2000, max_len=2000, max_dim=40)
items, keep = [], []
for k, (name, tp, n) in enumerate(suite):
    gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tp))
    x = torch.tensor(rng.uniform(-1, 1, size=(n, tp.num_inputs)), dtype=torch.float32, device="cuda")
    v = torch.tensor(rng.choice([-1.0, 1.0], size=(n, tp.num_inputs)), dtype=torch.float32, device="cuda")
    gg, hh = torch.empty_like(x), torch.empty_like(x)
    keep.append((gt, x, v, gg, hh))
    items.append((gt, x.data_ptr(), v.data_ptr(), n, gg.data_ptr(), hh.data_ptr()))
torch.cuda.synchronize()
m = MultiTapeHvp(ctx, items, f64=False, autotune=False)
m.launch()
assert lib.ech_ctx_synchronize(ctx._h) == 0, _lib.last_error()
for k, (_, _, _, gg, hh) in enumerate(keep):
    out[f"multi_g{k}"] = gg.cpu().numpy()
    out[f"multi_h{k}"] = hh.cpu().numpy()

t = configs.rosenbrock(30)
g = ctx.upload_tape_f64(t)
X = torch.tensor(rng.uniform(-2, 2, size=(3000, 30)), device="cuda")
o = torch.empty(3000, dtype=torch.float64, device="cuda")
gr = torch.empty(3000 * 30, dtype=torch.float64, device="cuda")
st = lib.ech_gradient_batch_device_noalloc(ctx._h, g._h, 1, X.data_ptr(), 3000, o.data_ptr(), gr.data_ptr(), None)
assert st == 0, _lib.last_error()
st = lib.ech_ctx_synchronize(ctx._h)
assert st == 0, _lib.last_error()
out["noalloc_v"], out["noalloc_g"] = o.cpu().numpy(), gr.cpu().numpy()
np.savez(sys.argv[1], **out)
print("clean")
"""


def _run(tmp_path, variant):
    env = dict(os.environ)
    env.pop("ECHIDNA_B200_VARIANT", None)
    if variant:
        env["ECHIDNA_B200_VARIANT"] = variant
    path = str(tmp_path / f"out_{variant or 'plain'}.npz")
    r = subprocess.run([sys.executable, "-c", CHILD, path, ROOT], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "clean" in r.stdout
    return dict(np.load(path))


def test_bounds_checked_build_is_clean_and_equal(tmp_path):
    lib = os.path.join(ROOT, "echidna_b200", "libechidna_b200_bounds.so")
    assert os.path.exists(lib), "build the checked variant: python -m echidna_b200.build --bounds"
    checked = _run(tmp_path, "bounds")
    plain = _run(tmp_path, "")
    assert checked.keys() == plain.keys()
    for k in plain:
        a, b = checked[k], plain[k]
        assert a.shape == b.shape, k
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8)) or np.array_equal(a, b, equal_nan=True), k
