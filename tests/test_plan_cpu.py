"""The host lowering, checked on the CPU: the emulated programs must reproduce
the oracle's outputs and gradients bit for bit at every shared-register cap
(cap 1 forces nearly every value into the global slots)."""
import numpy as np
import pytest

from echidna_b200 import configs, constant, record
from oracle.oracle import OracleTape
from tests.plan_emulator import plan_dump, run_gradient


def _lc_net(seed, n=5):
    """Layers of dot products over earlier values (repeated operands allowed),
    each followed by tanh or by a product with an earlier value, so reverse
    gathers form, break on conflicts and mix with other ops."""
    rng = np.random.default_rng(seed)

    def f(v):
        vals = list(v)
        for _layer in range(3):
            new = []
            for _j in range(4):
                s = constant(float(rng.normal()))
                for i in rng.choice(len(vals), size=int(rng.integers(1, 6)), replace=True):
                    s = s + constant(float(rng.normal())) * vals[int(i)]
                s = s.tanh() if rng.random() < 0.5 else s * vals[int(rng.integers(len(vals)))]
                new.append(s)
            vals = vals + new
        out = constant(0.0)
        for x in vals[-4:]:
            out = out + x * x
        return out
    return record(f, [0.1] * n)[0]


def _tapes():
    yield "rosen10", configs.rosenbrock(10)
    yield "mlp8", configs.mlp(8, 8)
    yield "lcnet1", _lc_net(1)
    yield "lcnet2", _lc_net(2)
    yield "lcnet3", _lc_net(3, n=3)
    yield "mlp4", configs.mlp(4, 4)
    yield "dag", configs.random_dag(6, 300, seed=7)
    yield "dag2", configs.random_dag(3, 120, seed=11)
    yield "square", record(lambda v: v[0] * v[0], [2.0])[0]
    yield "powi", record(lambda v: v[0].powi(3) + v[1].powi(-2), [2.0, 1.5])[0]
    yield "output_is_input", record(lambda v: v[1], [2.0, 3.0])[0]
    yield "const_output", record(lambda v: constant(2.0) * constant(3.0), [2.0])[0]
    yield "unused_input", record(lambda v: v[0].sin() * v[0], [2.0, 5.0])[0]


@pytest.mark.parametrize("dense_max", [1, 2, 16])
@pytest.mark.parametrize("cap", [1, 2, 3, 8, 4096])
@pytest.mark.parametrize("name,tape", list(_tapes()))
def test_lowered_gradient_matches_oracle(name, tape, cap, dense_max):
    rng = np.random.default_rng(3)
    X = rng.uniform(-1.5, 1.5, size=(7, tape.num_inputs))
    out, grad = run_gradient(tape, X, cap, dense_max)
    o = OracleTape(tape)
    ref_out, ref_grad = o.gradient(X)
    np.testing.assert_array_equal(out, ref_out)
    np.testing.assert_array_equal(grad, ref_grad)


@pytest.mark.parametrize("cap", [1, 4, 64, 4096])
def test_register_caps_respected(cap):
    tape = configs.mlp(8, 8)
    fwd, rev, pool, info = plan_dump(tape, "gradient", cap)
    assert info["smem_regs"] <= cap
    # every shared / global index referenced is in range
    for ins in fwd:
        _, ma, mb, md, a, b, d, save, aux, imm = ins
        for m, i in ((ma, a), (mb, b), (md, d)):
            if m == 0:
                assert i < info["smem_regs"]
            elif m == 1:
                assert i < info["far_slots"]
        if save != 0xFFFFFFFF:
            assert save < info["traj_slots"]
    for o in info["dense"]:
        for m, i in ((o["am"], o["ai"]), (o["dm"], o["di"])):
            if m == 0:
                assert i < info["smem_regs"]
            elif m == 1:
                assert i < info["far_slots"]
        if o["save"] != 0xFFFFFFFF:
            assert o["save"] < info["traj_slots"]


def test_mlp_trajectory_is_three_layers_of_width():
    # values read by reverse partials: the 2x64 tanh arguments and the 64 squared outputs
    tape = configs.mlp(64, 64)
    _, _, _, info = plan_dump(tape, "gradient", 4096)
    assert info["traj_slots"] == 3 * 64


def test_dense_layers_reverse_as_gathers():
    # the MLP's two dense layers: every chain reverse becomes a normalisation and
    # each layer one gather (one store per input adjoint)
    tape = configs.mlp(8, 8)
    _, rev, _, info = plan_dump(tape, "gradient", 4096)
    ops = [r[0] for r in rev]
    assert ops.count(85) >= 2 and ops.count(84) == 16 and ops.count(69) <= 1
    headers, q = [], 0
    while q < len(info["gathers"]):
        headers.append(info["gathers"][q])
        q += 1 + info["gathers"][q]["n"]
    assert sorted(h["n"] for h in headers) == [8] * 16


@pytest.mark.parametrize("dense_max,groups", [(16, 8), (8, 16), (2, 64), (1, 0)])
def test_mlp_dense_layers_become_groups(dense_max, groups):
    # each width-64 layer's 64 dot products read the same 64 operands: groups of
    # dense_max chains (one forward instruction each), nothing else grouped
    tape = configs.mlp(64, 64)
    fwd, _, _, info = plan_dump(tape, "gradient", 4096, dense_max)
    dense = [ins for ins in fwd if ins[0] == 86]
    assert len(dense) == groups
    assert sum(ins[8] for ins in dense) == (128 if groups else 0)
    assert all(ins[8] <= dense_max for ins in dense)


def test_dense_group_waits_for_acc0_defined_later():
    # the second dot product's constant term is an earlier result computed after
    # the first dot product starts: it cannot join the group
    def f(v):
        a = constant(0.5) + 2.0 * v[0] + 3.0 * v[1]
        t = a.sin()
        b = t + 4.0 * v[0] + 5.0 * v[1]
        return a * b
    tape = record(f, [0.1, 0.2])[0]
    fwd, _, _, info = plan_dump(tape, "gradient", 4096, 16)
    assert not any(ins[0] == 86 for ins in fwd)
    X = np.random.default_rng(4).uniform(-1, 1, size=(5, 2))
    out, grad = run_gradient(tape, X, 4096, 16)
    ref_out, ref_grad = OracleTape(tape).gradient(X)
    np.testing.assert_array_equal(out, ref_out)
    np.testing.assert_array_equal(grad, ref_grad)
