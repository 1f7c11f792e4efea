"""Sparse Jacobian / Hessian drop-ins and the host sparsity / coloring they use.

``CudaContext.sparse_jacobian{,_f64}`` / ``sparse_hessian{,_f64}``
(``src/gpu/cuda_backend.rs:306-441, 696-731, 915-932``): detect the structural
pattern on the host, color it, run one tangent (Jacobian) or HVP (Hessian)
sweep per color on the GPU with the color's indicator vector as the seed, and
scatter the compressed columns into COO values.  Patterns and colors come from
the engine library (``csrc/sparsity.cpp``) and equal the reference's.  Output
values and the value/gradient of the zero-color case come from GPU sweeps too.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Tuple

import numpy as np

from . import _lib


@dataclass
class SparsityPattern:
    """Lower-triangle Hessian pattern, COO sorted by (row, col) (``src/sparse.rs``)."""

    dim: int
    rows: np.ndarray
    cols: np.ndarray

    def nnz(self) -> int:
        return int(self.rows.size)

    def is_empty(self) -> bool:
        return self.rows.size == 0

    def contains(self, i: int, j: int) -> bool:
        r, c = (i, j) if i >= j else (j, i)
        return bool(np.any((self.rows == r) & (self.cols == c)))


@dataclass
class JacobianSparsityPattern:
    num_outputs: int
    num_inputs: int
    rows: np.ndarray
    cols: np.ndarray

    def nnz(self) -> int:
        return int(self.rows.size)

    def is_empty(self) -> bool:
        return self.rows.size == 0

    def contains(self, output_idx: int, input_idx: int) -> bool:
        return bool(np.any((self.rows == output_idx) & (self.cols == input_idx)))


def _check(st: int, what: str):
    if st != _lib.OK:
        raise ValueError(f"{what}: invalid arguments")


def detect_sparsity(tape) -> SparsityPattern:
    """``BytecodeTape::detect_sparsity`` (``src/bytecode_tape/sparse.rs:463-593``)."""
    lib = _lib.load()
    op, a0, a1, _ = tape.arrays()
    nnz = ctypes.c_size_t(0)
    _check(lib.ech_detect_hessian_sparsity(_lib.ptr(op), _lib.ptr(a0), _lib.ptr(a1), len(op), tape.num_inputs,
                                           None, None, 0, ctypes.byref(nnz)), "detect_sparsity")
    rows = np.empty(nnz.value, np.uint32)
    cols = np.empty(nnz.value, np.uint32)
    _check(lib.ech_detect_hessian_sparsity(_lib.ptr(op), _lib.ptr(a0), _lib.ptr(a1), len(op), tape.num_inputs,
                                           _lib.ptr(rows), _lib.ptr(cols), rows.size, ctypes.byref(nnz)),
           "detect_sparsity")
    return SparsityPattern(tape.num_inputs, rows, cols)


def detect_jacobian_sparsity(tape) -> JacobianSparsityPattern:
    """``BytecodeTape::detect_jacobian_sparsity`` (``src/bytecode_tape/sparse.rs:716-776``)."""
    lib = _lib.load()
    op, a0, a1, _ = tape.arrays()
    outs = np.asarray(tape.all_output_indices(), np.uint32)
    nnz = ctypes.c_size_t(0)
    args = (_lib.ptr(op), _lib.ptr(a0), _lib.ptr(a1), len(op), tape.num_inputs, _lib.ptr(outs), outs.size)
    _check(lib.ech_detect_jacobian_sparsity(*args, None, None, 0, ctypes.byref(nnz)), "detect_jacobian_sparsity")
    rows = np.empty(nnz.value, np.uint32)
    cols = np.empty(nnz.value, np.uint32)
    _check(lib.ech_detect_jacobian_sparsity(*args, _lib.ptr(rows), _lib.ptr(cols), rows.size, ctypes.byref(nnz)),
           "detect_jacobian_sparsity")
    return JacobianSparsityPattern(int(outs.size), tape.num_inputs, rows, cols)


def greedy_coloring(p: SparsityPattern) -> Tuple[np.ndarray, int]:
    """``sparse::greedy_coloring`` (``src/sparse.rs:57-98``): distance-2 coloring."""
    colors = np.empty(p.dim, np.uint32)
    n = ctypes.c_uint32(0)
    rows = np.ascontiguousarray(p.rows, np.uint32)
    cols = np.ascontiguousarray(p.cols, np.uint32)
    _check(_lib.load().ech_greedy_coloring(p.dim, _lib.ptr(rows), _lib.ptr(cols), rows.size, _lib.ptr(colors),
                                           ctypes.byref(n)), "greedy_coloring")
    return colors, int(n.value)


def _jac_coloring(p: JacobianSparsityPattern, fn, size: int):
    colors = np.empty(size, np.uint32)
    n = ctypes.c_uint32(0)
    rows = np.ascontiguousarray(p.rows, np.uint32)
    cols = np.ascontiguousarray(p.cols, np.uint32)
    _check(fn(p.num_outputs, p.num_inputs, _lib.ptr(rows), _lib.ptr(cols), rows.size, _lib.ptr(colors),
              ctypes.byref(n)), "coloring")
    return colors, int(n.value)


def column_coloring(p: JacobianSparsityPattern) -> Tuple[np.ndarray, int]:
    """``sparse::column_coloring`` (``src/sparse.rs:292-299``)."""
    return _jac_coloring(p, _lib.load().ech_column_coloring, p.num_inputs)


def row_coloring(p: JacobianSparsityPattern) -> Tuple[np.ndarray, int]:
    """``sparse::row_coloring`` (``src/sparse.rs:309-316``)."""
    return _jac_coloring(p, _lib.load().ech_row_coloring, p.num_outputs)


def _seed_rows(colors: np.ndarray, num_colors: int, ni: int, dtype) -> np.ndarray:
    seeds = np.zeros((num_colors, ni), dtype=dtype)
    if ni:
        seeds[colors, np.arange(ni)] = 1
    return seeds


def sparse_jacobian_gpu(ctx, tape, tape_cpu, x, dtype):
    """``cuda_sparse_jacobian_body`` (``src/gpu/cuda_backend.rs:306-392``):
    returns ``(output values, pattern, jac_values)``."""
    x = np.ascontiguousarray(x, dtype=dtype).ravel()
    ni = tape.num_inputs
    f64 = np.dtype(dtype) == np.float64
    pattern = detect_jacobian_sparsity(tape_cpu)
    colors, num_colors = column_coloring(pattern)
    fwd = ctx.forward_batch_f64 if f64 else ctx.forward_batch
    values = fwd(tape, x, 1)
    if num_colors == 0:
        return values, pattern, np.zeros(0, dtype=dtype)
    seeds = _seed_rows(colors, num_colors, ni, dtype)
    primals = np.tile(x, num_colors)
    tan = ctx.tangent_forward_batch_f64 if f64 else ctx.tangent_forward_batch
    _, tangents = tan(tape, primals, seeds.ravel(), num_colors)
    no = tape.num_outputs
    jac = tangents[colors[pattern.cols].astype(np.int64) * no + pattern.rows.astype(np.int64)]
    return values, pattern, np.ascontiguousarray(jac, dtype=dtype)


def sparse_hessian_gpu(ctx, tape, tape_cpu, x, dtype):
    """``cuda_sparse_hessian_body`` (``src/gpu/cuda_backend.rs:394-436``):
    returns ``(value, gradient, pattern, hess_values)``."""
    x = np.ascontiguousarray(x, dtype=dtype).ravel()
    ni = tape.num_inputs
    f64 = np.dtype(dtype) == np.float64
    pattern = detect_sparsity(tape_cpu)
    colors, num_colors = greedy_coloring(pattern)
    grad_fn = ctx.gradient_batch_f64 if f64 else ctx.gradient_batch
    if num_colors == 0:
        v, g = grad_fn(tape, x, 1)
        return v[0], g, pattern, np.zeros(0, dtype=dtype)
    dirs = _seed_rows(colors, num_colors, ni, dtype)
    hvp = ctx.hvp_batch_f64 if f64 else ctx.hvp_batch
    grads, hvps = hvp(tape, x, dirs.ravel(), num_colors)
    gradient = grads[:ni].copy()
    hess = hvps[colors[pattern.cols].astype(np.int64) * ni + pattern.rows.astype(np.int64)]
    fwd = ctx.forward_batch_f64 if f64 else ctx.forward_batch
    value = fwd(tape, x, 1)[0]
    return value, gradient, pattern, np.ascontiguousarray(hess, dtype=dtype)
