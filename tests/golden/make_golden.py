"""Writes tests/golden/config_vectors.json: oracle outputs on the two plain-method
workloads at a few fixed points, stored as exact hex floats.

The reference is a Rust crate that cannot be built in this environment, so these
vectors come from the oracle (the C++ restatement of its CPU sweeps); the oracle
itself is pinned to the reference's asserted answers by tests/test_known_answers.py.
The fixture catches any later drift of the oracle or of the recorder, and gives
the GPU tests a fixed expected answer.

Run:  python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from echidna_b200 import configs  # noqa: E402
from oracle.oracle import OracleTape  # noqa: E402


def hexes(a):
    return [float(v).hex() for v in np.asarray(a, dtype=np.float64).ravel()]


def case(name, tape, X, V):
    o = OracleTape(tape)
    val, grad = o.gradient(X)
    g2, hv = o.hvp(X, V)
    c = o.taylor(X, V, 3)
    return {"name": name, "num_inputs": int(tape.num_inputs), "num_variables": len(tape.opcodes),
            "x": hexes(X), "v": hexes(V), "value": hexes(val), "gradient": hexes(grad), "hvp": hexes(hv),
            "taylor3": hexes(c)}


def main():
    out = []
    rng = np.random.default_rng(configs.SEEDS["rosenbrock"])
    X = rng.uniform(-2.0, 2.0, size=(4, 100))
    V = rng.choice([-1.0, 1.0], size=(4, 100))
    out.append(case("rosenbrock_n100", configs.rosenbrock(100), X, V))
    rng = np.random.default_rng(configs.SEEDS["mlp"])
    X = rng.normal(size=(2, 64))
    V = rng.choice([-1.0, 1.0], size=(2, 64))
    out.append(case("mlp_n64_w64", configs.mlp(64, 64), X, V))
    with open(os.path.join(HERE, "config_vectors.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "cases": out}, f, indent=1)


if __name__ == "__main__":
    main()
