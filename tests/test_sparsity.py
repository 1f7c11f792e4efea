"""Structural sparsity and coloring: the engine library against the reference's
known answers and, bit-exactly, against the oracle restatement; GPU sparse
Jacobian / Hessian against dense oracle derivatives."""
import numpy as np
import pytest

from echidna_b200 import configs, record, record_multi
from echidna_b200.gpu import GpuTapeData
from echidna_b200.sparse import (JacobianSparsityPattern, SparsityPattern, column_coloring, detect_jacobian_sparsity,
                                 detect_sparsity, greedy_coloring, row_coloring)
from oracle import sparsity as osp
from oracle.oracle import OracleTape


def _pat(dim, rows, cols):
    return SparsityPattern(dim, np.array(rows, np.uint32), np.array(cols, np.uint32))


def _jpat(no, ni, rows, cols):
    return JacobianSparsityPattern(no, ni, np.array(rows, np.uint32), np.array(cols, np.uint32))


# ── tests/sparse_coloring.rs ──

def test_greedy_coloring_known_answers(engine_lib):
    assert greedy_coloring(_pat(0, [], []))[1] == 0                                   # :13-22
    c, n = greedy_coloring(_pat(4, [0, 1, 2, 3], [0, 1, 2, 3]))                        # :25-35
    assert len(c) == 4 and n == 1
    c, n = greedy_coloring(_pat(3, [0, 1, 1, 2, 2, 2], [0, 0, 1, 0, 1, 2]))            # :38-53
    assert n == 3 and len(set(c.tolist())) == 3
    c, n = greedy_coloring(_pat(4, [0, 1, 1, 2, 2, 3, 3], [0, 0, 1, 1, 2, 2, 3]))      # :56-73
    assert n <= 4 and c[0] != c[1] and c[1] != c[2]
    c, n = greedy_coloring(_pat(3, [0, 1, 1, 2, 2], [0, 0, 1, 1, 2]))                  # :76-91
    assert n == 3 and len(set(c.tolist())) == 3


def test_jacobian_coloring_known_answers(engine_lib):
    assert column_coloring(_jpat(0, 0, [], []))[1] == 0                                # :98-108
    assert column_coloring(_jpat(3, 3, [0, 1, 2], [0, 1, 2]))[1] == 1                  # :111-123
    assert column_coloring(_jpat(2, 3, [0, 0, 0, 1, 1, 1], [0, 1, 2, 0, 1, 2]))[1] == 3  # :126-137
    c, n = column_coloring(_jpat(2, 3, [0, 0, 1, 1], [0, 1, 1, 2]))                    # :140-157
    assert n == 2 and c[0] != c[1] and c[1] != c[2] and c[0] == c[2]
    assert row_coloring(_jpat(0, 0, [], []))[1] == 0                                   # :164-174
    assert row_coloring(_jpat(3, 3, [0, 1, 2], [0, 1, 2]))[1] == 1                     # :177-188
    assert row_coloring(_jpat(3, 2, [0, 0, 1, 1, 2, 2], [0, 1, 0, 1, 0, 1]))[1] == 3   # :191-202


def test_detected_jacobian_sparsity_coloring(engine_lib):
    # tests/sparse_coloring.rs:209-226
    tape, _ = record_multi(lambda v: [v[0] * v[1], v[2]], [1.0, 2.0, 3.0])
    p = detect_jacobian_sparsity(tape)
    cc, cn = column_coloring(p)
    rc, rn = row_coloring(p)
    assert cn == 2 and cc[0] != cc[1]
    assert rn == 1 and rc[0] == rc[1]


# ── tests/sparse_jacobian.rs ──

def test_jacobian_patterns_known_answers(engine_lib):
    want = {
        # :18-33: [2 x0 + x1, x1 + 3 x2]
        "linear": (lambda v: [v[0] * 2.0 + v[1], v[1] + v[2] * 3.0], {(0, 0), (0, 1), (1, 1), (1, 2)}),
        # :35-55: [x0 x1, x1 x2, x0^2]
        "nonlinear": (lambda v: [v[0] * v[1], v[1] * v[2], v[0] * v[0]], {(0, 0), (0, 1), (1, 1), (1, 2), (2, 0)}),
    }
    for name, (fn, entries) in want.items():
        tape, _ = record_multi(fn, [1.0, 2.0, 3.0])
        p = detect_jacobian_sparsity(tape)
        for i in range(tape.num_outputs()):
            for j in range(3):
                assert p.contains(i, j) == ((i, j) in entries), (name, i, j)
    # :57-66: an identity map needs one column color
    tape, _ = record_multi(lambda v: [v[0], v[1], v[2]], [1.0, 2.0, 3.0])
    assert column_coloring(detect_jacobian_sparsity(tape))[1] == 1


# ── tests/sparse_hessian.rs ──

def test_hessian_patterns_known_answers(engine_lib):
    p = detect_sparsity(record(lambda v: v[0] * v[0] + v[1] * v[1], [3.0, 4.0])[0])     # :18-29
    assert p.contains(0, 0) and p.contains(1, 1) and not p.contains(0, 1)
    p = detect_sparsity(record(lambda v: v[0] * v[1], [2.0, 3.0])[0])                  # :32-40
    assert p.contains(0, 1) and p.contains(1, 0)
    p = detect_sparsity(record(lambda v: v[0] * v[0] + v[1] * v[2], [1.0, 2.0, 3.0])[0])  # :43-54
    assert p.contains(0, 0) and p.contains(1, 2) and not p.contains(0, 1) and not p.contains(0, 2)


def _tridiag(v):
    s = v[0] - v[0]
    for i in range(len(v) - 1):
        s = s + v[i] * v[i + 1]
    return s


def test_tridiagonal_three_colors(engine_lib):
    # tests/sparse_hessian.rs:57-90
    n = 10
    tape, _ = record(_tridiag, [0.5 + 0.01 * i for i in range(n)])
    p = detect_sparsity(tape)
    for i in range(n - 1):
        assert p.contains(i, i + 1)
    for i in range(n):
        for j in range(n):
            if abs(i - j) > 1:
                assert not p.contains(i, j)
    assert greedy_coloring(p)[1] == 3


TAPES = {
    "rosen20": lambda: configs.rosenbrock(20),
    "dag_a": lambda: configs.random_dag(12, 300, seed=3),
    "dag_b": lambda: configs.random_dag(70, 900, seed=4),
    "mlp8": lambda: configs.mlp(8, 6),
    "tridiag": lambda: record(_tridiag, [0.5 + 0.01 * i for i in range(40)])[0],
}


@pytest.mark.parametrize("name", list(TAPES))
def test_patterns_and_colors_match_oracle_restatement(engine_lib, name):
    tape = TAPES[name]()
    op, a0, a1, _ = tape.arrays()
    ni = tape.num_inputs
    p = detect_sparsity(tape)
    r, c = osp.hessian_pattern(op, a0, a1, ni)
    assert p.rows.tolist() == r and p.cols.tolist() == c
    colors, n = greedy_coloring(p)
    oc, on = osp.greedy_coloring(ni, r, c)
    assert colors.tolist() == oc and n == on
    jp = detect_jacobian_sparsity(tape)
    jr, jc = osp.jacobian_pattern(op, a0, a1, ni, tape.all_output_indices())
    assert jp.rows.tolist() == jr and jp.cols.tolist() == jc
    for fn, ofn in ((column_coloring, osp.column_coloring), (row_coloring, osp.row_coloring)):
        cc, cn = fn(jp)
        occ, ocn = ofn(jp.num_outputs, ni, jr, jc)
        assert cc.tolist() == occ and cn == ocn


def test_diagonal_coloring_separates_interacting_coordinates(engine_lib):
    from echidna_b200.learned import diagonal_coloring
    # tridiagonal: two colors; diagonal only: one; a dense 3x3 lower triangle: three
    assert diagonal_coloring(_pat(5, [0, 1, 1, 2, 2, 3, 3, 4, 4], [0, 0, 1, 1, 2, 2, 3, 3, 4]))[1] == 2
    assert diagonal_coloring(_pat(4, [0, 1, 2, 3], [0, 1, 2, 3]))[1] == 1
    assert diagonal_coloring(_pat(3, [0, 1, 1, 2, 2, 2], [0, 0, 1, 0, 1, 2]))[1] == 3
    assert diagonal_coloring(_pat(0, [], []))[1] == 0
    # the learned-proposal tape (softplus of x_i x_{i+1}): a valid coloring with two colors
    p = detect_sparsity(configs.softplus_chain(257))
    colors, n = diagonal_coloring(p)
    assert n == 2
    off = p.rows != p.cols
    assert np.all(colors[p.rows[off]] != colors[p.cols[off]])


def test_many_colors_fall_back_past_64(engine_lib):
    # a dense 70 x 70 Hessian needs 70 colors: exercises the >= 64 color branch
    n = 70
    rows = [i for i in range(n) for j in range(i + 1)]
    cols = [j for i in range(n) for j in range(i + 1)]
    colors, num = greedy_coloring(_pat(n, rows, cols))
    oc, on = osp.greedy_coloring(n, rows, cols)
    assert num == 70 == on and colors.tolist() == oc


# ── GPU drop-ins: src/gpu/cuda_backend.rs:306-441 ──

def _multi(v):
    return [v[0] * v[1], v[1] + v[2].sin(), v[0] * v[2].exp(), v[3] * v[3]]


@pytest.mark.gpu
def test_gpu_sparse_jacobian_f64_matches_dense(ctx):
    x = np.array([0.3, -1.2, 0.7, 2.0])
    tape, _ = record_multi(_multi, x.tolist())
    gt = ctx.upload_tape_f64(tape)
    vals, pat, jac = ctx.sparse_jacobian_f64(gt, tape, x)
    o = OracleTape(tape)
    ref_vals = o.forward(x[None, :])[0]
    assert np.array_equal(vals, ref_vals) or np.allclose(vals, ref_vals, rtol=1e-15)
    dense = np.stack([o.jvp(x[None, :], np.eye(4)[k][None, :])[1][0] for k in range(4)], axis=1)
    for k in range(pat.nnz()):
        assert abs(jac[k] - dense[pat.rows[k], pat.cols[k]]) <= 1e-14 * max(1.0, abs(dense[pat.rows[k], pat.cols[k]]))


@pytest.mark.gpu
def test_gpu_sparse_hessian_tridiagonal_and_rosenbrock(ctx):
    for tape, x in ((record(_tridiag, [0.5 + 0.01 * i for i in range(10)])[0], 0.5 + 0.01 * np.arange(10)),
                    (configs.rosenbrock(12), np.linspace(-1.0, 1.5, 12))):
        gt = ctx.upload_tape_f64(tape)
        val, grad, pat, hv = ctx.sparse_hessian_f64(gt, tape, x)
        o = OracleTape(tape)
        rv, rg, H = o.hessian(x)
        assert abs(val - rv) <= 1e-12 * max(1.0, abs(rv))
        assert np.allclose(grad, rg, rtol=1e-13, atol=1e-13)
        for k in range(pat.nnz()):
            assert abs(hv[k] - H[pat.rows[k], pat.cols[k]]) <= 1e-10
        # f32 drop-in through the lossy upload
        g32 = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
        v32, gr32, pat32, hv32 = ctx.sparse_hessian(g32, tape, x.astype(np.float32))
        assert pat32.rows.tolist() == pat.rows.tolist()
        assert np.allclose(hv32, hv, rtol=1e-4, atol=1e-3)
