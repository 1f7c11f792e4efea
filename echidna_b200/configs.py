"""Synthetic workload tapes with the shapes of the benchmark configurations.

Every tape is recorded through :func:`echidna_b200.tape.record`, i.e. with the
reference's recording rules (a fresh ``Const`` slot per constant use, constant
folding, IEEE-exact identities), so slot counts match what echidna's ``record``
would produce for the same Rust closure.  Seeds are fixed per configuration.

* ``rosenbrock(n)``: the bench-style extended Rosenbrock of
  ``benches/common/mod.rs:10-20``.
* ``mlp(n=64, width=64)``: ``h1 = tanh(W1 x + b1)``, ``h2 = tanh(W2 h1 + b2)``,
  ``f = 0.5 * ||h2||^2`` with ``W ~ N(0, 1/64)`` and ``b = 0`` baked in as constants.
* ``logsumexp_tanh(n=256, m=512)``: ``f = ln(sum_j exp(tanh(W x + b)_j))`` with
  ``W ~ N(0, 1/256)``, ``b ~ N(0, 0.1^2)``.  ``|tanh| <= 1`` so the sum needs no
  max-shift.
* ``softplus_chain(n=1024)``: ``f = sum_i a_i softplus(x_i x_{i+1}) + sum_i a_i cos x_i``,
  ``a_i`` log-uniform in ``[1e-3, 1e3]``, softplus recorded as ``ln_1p(exp(z))``.
"""
from __future__ import annotations

import numpy as np

from .tape import constant, record

SEEDS = {"rosenbrock": 0xEC01, "mlp": 0xEC02, "logsumexp_tanh": 0xEC03, "uneven": 0xEC04, "softplus_chain": 0xEC05}


def rosenbrock_fn(x):
    one = constant(1.0)
    hundred = constant(100.0)
    s = constant(0.0)
    for i in range(len(x) - 1):
        t1 = one - x[i]
        t2 = x[i + 1] - x[i] * x[i]
        s = s + t1 * t1 + hundred * t2 * t2
    return s


def rosenbrock(n: int = 100, dtype=np.float64):
    x0 = [0.5 + 0.01 * i for i in range(n)]
    tape, _ = record(rosenbrock_fn, x0, dtype=dtype)
    return tape


def mlp_weights(n=64, width=64, seed=SEEDS["mlp"]):
    rng = np.random.default_rng(seed)
    w1 = rng.normal(0.0, np.sqrt(1.0 / n), size=(width, n))
    w2 = rng.normal(0.0, np.sqrt(1.0 / width), size=(width, width))
    b1 = np.zeros(width)
    b2 = np.zeros(width)
    return w1, b1, w2, b2


def mlp(n: int = 64, width: int = 64, dtype=np.float64, seed=SEEDS["mlp"]):
    w1, b1, w2, b2 = mlp_weights(n, width, seed)

    def f(x):
        def layer(inp, w, b):
            out = []
            for j in range(w.shape[0]):
                z = constant(float(b[j]))
                for i in range(w.shape[1]):
                    z = z + float(w[j, i]) * inp[i]
                out.append(z.tanh())
            return out

        h1 = layer(x, w1, b1)
        h2 = layer(h1, w2, b2)
        s = constant(0.0)
        for h in h2:
            s = s + h * h
        return 0.5 * s

    tape, _ = record(f, [0.1] * n, dtype=dtype)
    return tape


def logsumexp_tanh_weights(n=256, m=512, seed=SEEDS["logsumexp_tanh"]):
    rng = np.random.default_rng(seed)
    w = rng.normal(0.0, np.sqrt(1.0 / n), size=(m, n))
    b = rng.normal(0.0, 0.1, size=m)
    return w, b


def logsumexp_tanh(n: int = 256, m: int = 512, dtype=np.float64, seed=SEEDS["logsumexp_tanh"]):
    w, b = logsumexp_tanh_weights(n, m, seed)

    def f(x):
        s = constant(0.0)
        for j in range(m):
            z = constant(float(b[j]))
            for i in range(n):
                z = z + float(w[j, i]) * x[i]
            s = s + z.tanh().exp()
        return s.ln()

    tape, _ = record(f, [0.1] * n, dtype=dtype)
    return tape


def softplus_chain_coeffs(n=1024, seed=SEEDS["softplus_chain"]):
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(np.log(1e-3), np.log(1e3), size=n))


def softplus_chain(n: int = 1024, dtype=np.float64, seed=SEEDS["softplus_chain"]):
    a = softplus_chain_coeffs(n, seed)

    def f(x):
        s = constant(0.0)
        for i in range(n - 1):
            s = s + float(a[i]) * (x[i] * x[i + 1]).exp().ln_1p()
        for i in range(n):
            s = s + float(a[i]) * x[i].cos()
        return s

    tape, _ = record(f, [0.1] * n, dtype=dtype)
    return tape


def random_dag(n: int, length: int, seed: int, dtype=np.float64):
    """Random DAG tape over {add, mul, sin, exp, log, tanh} with ~``length`` ops.

    Domain rules keep every value finite: ``ln`` is only applied to ``1 + a*a``,
    ``exp`` and ``mul`` only to values bounded by a preceding ``sin``/``tanh``.
    """
    rng = np.random.default_rng(seed)

    def f(x):
        pool = [(xi, False) for xi in x]          # (value, bounded)
        bounded = [xi.tanh() for xi in x[: max(1, min(len(x), 4))]]
        pool += [(b, True) for b in bounded]
        target = max(length - 3 * len(x), 8)
        count = 0
        while count < target:
            k = int(rng.integers(0, 6))
            lo = max(0, len(pool) - 64)
            a, ab = pool[int(rng.integers(lo, len(pool)))]
            b, bb = pool[int(rng.integers(lo, len(pool)))]
            if k == 0:
                v, vb = a + b, False
                count += 1
            elif k == 1:
                if not (ab and bb):
                    a, b = a.tanh(), b.sin()
                    count += 2
                v, vb = a * b, True
                count += 1
            elif k == 2:
                v, vb = a.sin(), True
                count += 1
            elif k == 3:
                if not ab:
                    a = a.tanh()
                    count += 1
                v, vb = a.exp(), False
                count += 1
            elif k == 4:
                v, vb = (1.0 + a * a).ln(), False
                count += 4
            else:
                v, vb = a.tanh(), True
                count += 1
            pool.append((v, vb))
        s = constant(0.0)
        for v, _ in pool[-min(16, len(pool)):]:
            s = s + v
        return s

    x0 = list(np.linspace(-0.5, 0.5, n))
    tape, _ = record(f, x0, dtype=dtype)
    return tape


def ackley_fn(x):
    n = float(len(x))
    s2 = constant(0.0)
    sc = constant(0.0)
    for xi in x:
        s2 = s2 + xi * xi
        sc = sc + (xi * (2.0 * np.pi)).cos()
    return -20.0 * (-0.2 * (s2 / n).sqrt()).exp() - (sc / n).exp() + 20.0 + float(np.e)


def ackley(n: int, dtype=np.float64):
    """Ackley-type sum of exp / cos terms over ``n`` inputs."""
    tape, _ = record(ackley_fn, list(np.linspace(-0.5, 0.5, n)), dtype=dtype)
    return tape


def uneven_suite(count: int = 64, seed: int = SEEDS["uneven"], max_points: int = 100_000, max_len: int = 20_000,
                 max_dim: int = 512):
    """The uneven multi-tape batch: ``count`` (name, tape, n_points) triples.

    Tapes cycle through Rosenbrock, Ackley-type and random DAGs over
    {add, mul, sin, exp, log, tanh}; input dimensions are log-uniform in
    [2, max_dim], DAG lengths log-uniform in [200, max_len] ops and point counts
    log-uniform in [1, max_points].
    """
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = int(round(np.exp(rng.uniform(np.log(2), np.log(max_dim)))))
        pts = int(round(np.exp(rng.uniform(0.0, np.log(max_points)))))
        kind = k % 3
        if kind == 0:
            name, tape = f"rosenbrock{n}", rosenbrock(n)
        elif kind == 1:
            name, tape = f"ackley{n}", ackley(n)
        else:
            length = int(round(np.exp(rng.uniform(np.log(200), np.log(max_len)))))
            name, tape = f"dag{n}x{length}", random_dag(n, length, seed=seed + k)
        out.append((name, tape, max(1, pts)))
    return out
