"""The per-value-kind cost model of the roofline (echidna_b200.opcost) on tapes
whose op counts are known by construction."""
from echidna_b200 import configs, constant, opcost, record


def test_counts_of_a_small_tape():
    # f = sin(x0 * x1) + 3 * x0 - x1 / 2: one var*var mul, one mul by a constant,
    # one div by a constant, one sub, one add, one unary special
    tape, _ = record(lambda v: (v[0] * v[1]).sin() + 3.0 * v[0] - v[1] / constant(2.0), [0.3, 0.7])
    fwd, rev = opcost._classes(tape)
    assert (fwd["mul"], fwd["mul_c"], fwd["div_c"], fwd["add"], fwd["unary"]) == (1, 1, 1, 2, 1)
    assert opcost.sweep_cost(tape, "forward") == (5, 1)
    # Jet K=3: add/sub 3 each, scale 3, div-by-constant 3, mul 9, unary 9
    assert opcost.sweep_cost(tape, "taylor", 3) == (3 + 3 + 3 + 3 + 9 + 9, 1)


def test_dead_ops_do_not_count():
    def f(v):
        _unused = v[0].exp() * v[1]
        return v[0] + v[1]
    tape, _ = record(f, [0.1, 0.2])
    assert opcost.sweep_cost(tape, "forward") == (1, 0)
    assert opcost.sweep_cost(tape, "gradient") == (1 + 2 * 2, 0)


def test_mlp_hvp_is_about_twice_the_gradient():
    tape = configs.mlp(16, 16)
    g, _ = opcost.sweep_cost(tape, "gradient")
    h, _ = opcost.sweep_cost(tape, "hvp")
    assert 1.8 * g <= h <= 2.6 * g


def test_roofline_picks_the_binding_bound():
    r = opcost.roofline(bytes_alg=1e9, flops_alg=1e9, seconds=1e-3, hbm_gbs=1000.0, pipe_ops=1e13)
    assert r["binding"] == "hbm" and abs(r["t_roof_ms"] - 1.0) < 1e-12 and abs(r["frac"] - 1.0) < 1e-12
    r = opcost.roofline(bytes_alg=1e6, flops_alg=1e12, seconds=1.0, hbm_gbs=1000.0, pipe_ops=1e13)
    assert r["binding"] == "pipe" and abs(r["frac"] - 0.1) < 1e-12
