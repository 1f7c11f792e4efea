"""Golden vectors of tests/golden/config_vectors.json (made by make_golden.py)."""
import json
import os

import numpy as np
import pytest

from echidna_b200 import configs
from oracle.oracle import OracleTape

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "config_vectors.json")) as f:
    CASES = json.load(f)["cases"]
TAPES = {"rosenbrock_n100": lambda: configs.rosenbrock(100), "mlp_n64_w64": lambda: configs.mlp(64, 64)}


def arr(h, shape=None):
    a = np.array([float.fromhex(v) for v in h])
    return a.reshape(shape) if shape else a


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_recorder_and_oracle_reproduce_golden(case):
    tape = TAPES[case["name"]]()
    assert len(tape.opcodes) == case["num_variables"]
    n = case["num_inputs"]
    X, V = arr(case["x"], (-1, n)), arr(case["v"], (-1, n))
    o = OracleTape(tape)
    val, grad = o.gradient(X)
    _, hv = o.hvp(X, V)
    c = o.taylor(X, V, 3)
    assert np.array_equal(val.ravel(), arr(case["value"]))
    assert np.array_equal(grad.ravel(), arr(case["gradient"]))
    assert np.array_equal(hv.ravel(), arr(case["hvp"]))
    assert np.array_equal(c.ravel(), arr(case["taylor3"]))


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_gpu_f64_matches_golden(ctx, case):
    tape = TAPES[case["name"]]()
    n = case["num_inputs"]
    X, V = arr(case["x"], (-1, n)), arr(case["v"], (-1, n))
    B = X.shape[0]
    gt = ctx.upload_tape_f64(tape)
    val, grad = ctx.gradient_batch_f64(gt, X, B)
    _, hv = ctx.hvp_batch_points_f64(gt, X, V, B)
    jets = ctx.taylor_forward_kth_batch_f64(gt, X, V, B, 3)
    # Rosenbrock is +,-,* only: bit-exact.  The MLP goes through CUDA's tanh: 1e-13 relative.
    rel = 0.0 if case["name"].startswith("rosenbrock") else 1e-13
    for got, want in ((val, case["value"]), (grad, case["gradient"]), (hv, case["hvp"]),
                      (np.concatenate(jets.coefficients), case["taylor3"])):
        want = arr(want)
        assert np.max(np.abs(got - want)) <= rel * max(1.0, np.abs(want).max())
