"""Bytecode tape model and recorder.

This module restates the recording half of echidna's BytecodeTape so that a tape
built here has exactly the slot layout the reference's ``record`` produces:

* ``OpCode`` discriminants follow ``src/opcode.rs:21-130`` (pinned again in
  ``src/gpu/mod.rs:427-472``); ``UNUSED`` is ``src/opcode.rs:11``.
* ``BytecodeTape.push_op`` / ``push_const`` / ``push_powi`` / ``new_input`` follow
  ``src/bytecode_tape/mod.rs:240-382``: constant folding when every operand is a
  ``Const``, the IEEE-exact single-constant identities (``x*1``, ``x/1``,
  ``x+(-0.0)``, ``x-(+0.0)``) and the powi rewrites (``x^0``, ``x^1``, ``x^-1``).
* ``BReverse`` follows ``src/breverse.rs:22-30`` and
  ``src/traits/breverse_ops.rs:16-150``: every use of a plain constant pushes a
  fresh ``Const`` slot, in the operand order of the Rust operator impls.
* ``record`` / ``record_multi`` follow ``src/api.rs:197-269``.

Recording-time values are computed in the tape's precision (float64 or float32)
with Rust's scalar semantics (``%`` is fmod, ``max``/``min`` route to the first
operand unless the second is NaN, ``powi`` is square-and-multiply).
"""
from __future__ import annotations

import enum
import json
import math
import threading
from typing import Callable, List, Optional, Sequence

import numpy as np

UNUSED = 0xFFFFFFFF
CONSTANT = 0xFFFFFFFF


class OpCode(enum.IntEnum):
    """Opcode discriminants (``src/opcode.rs:21-130``)."""

    Input = 0
    Const = 1
    Add = 2
    Sub = 3
    Mul = 4
    Div = 5
    Rem = 6
    Powf = 7
    Atan2 = 8
    Hypot = 9
    Max = 10
    Min = 11
    Neg = 12
    Recip = 13
    Sqrt = 14
    Cbrt = 15
    Powi = 16
    Exp = 17
    Exp2 = 18
    ExpM1 = 19
    Ln = 20
    Log2 = 21
    Log10 = 22
    Ln1p = 23
    Sin = 24
    Cos = 25
    Tan = 26
    Asin = 27
    Acos = 28
    Atan = 29
    Sinh = 30
    Cosh = 31
    Tanh = 32
    Asinh = 33
    Acosh = 34
    Atanh = 35
    Abs = 36
    Signum = 37
    Floor = 38
    Ceil = 39
    Round = 40
    Trunc = 41
    Fract = 42
    Custom = 43


BINARY_OPS = frozenset(range(OpCode.Add, OpCode.Min + 1))


def powi_exp_encode(exp: int) -> int:
    """Bit-preserving ``i32 -> u32`` (``src/opcode.rs:528-530``)."""
    return exp & 0xFFFFFFFF


def powi_exp_decode_raw(raw: int) -> int:
    """``u32 -> i32`` reinterpretation (``src/opcode.rs:491-494``)."""
    raw &= 0xFFFFFFFF
    return raw - (1 << 32) if raw >= (1 << 31) else raw


# ---------------------------------------------------------------------------
# Scalar semantics used for recording-time values (Rust f64/f32 behaviour).
# ---------------------------------------------------------------------------

class _Scalar:
    """Rust float semantics in one precision (numpy scalar type ``ft``)."""

    def __init__(self, ft):
        self.ft = ft

    def c(self, x):
        return self.ft(x)

    def powi(self, a, n: int):
        # Square-and-multiply, the llvm.powi lowering used by Rust's powi.
        a = self.ft(a)
        recip = n < 0
        m = -n if n < 0 else n
        r = self.ft(1.0)
        with np.errstate(all="ignore"):
            while True:
                if m & 1:
                    r = self.ft(r * a)
                m >>= 1
                if m == 0:
                    break
                a = self.ft(a * a)
            return self.ft(self.ft(1.0) / r) if recip else r

    def call(self, name: str, a, b=None):
        ft = self.ft
        a = ft(a)
        if b is not None:
            b = ft(b)
        with np.errstate(all="ignore"):
            if name == "add":
                return ft(a + b)
            if name == "sub":
                return ft(a - b)
            if name == "mul":
                return ft(a * b)
            if name == "div":
                return ft(a / b)
            if name == "rem":
                return ft(np.fmod(a, b))
            if name == "powf":
                return ft(np.power(a, b))
            if name == "atan2":
                return ft(np.arctan2(a, b))
            if name == "hypot":
                return ft(np.hypot(a, b))
            if name == "max":
                return a if (a >= b or np.isnan(b)) else b
            if name == "min":
                return a if (a <= b or np.isnan(b)) else b
            if name == "neg":
                return ft(-a)
            if name == "recip":
                return ft(ft(1.0) / a)
            if name == "sqrt":
                return ft(np.sqrt(a))
            if name == "cbrt":
                return ft(np.cbrt(a))
            if name == "exp":
                return ft(np.exp(a))
            if name == "exp2":
                return ft(np.exp2(a))
            if name == "exp_m1":
                return ft(np.expm1(a))
            if name == "ln":
                return ft(np.log(a))
            if name == "log2":
                return ft(np.log2(a))
            if name == "log10":
                return ft(np.log10(a))
            if name == "ln_1p":
                return ft(np.log1p(a))
            if name == "sin":
                return ft(np.sin(a))
            if name == "cos":
                return ft(np.cos(a))
            if name == "tan":
                return ft(np.tan(a))
            if name == "asin":
                return ft(np.arcsin(a))
            if name == "acos":
                return ft(np.arccos(a))
            if name == "atan":
                return ft(np.arctan(a))
            if name == "sinh":
                return ft(np.sinh(a))
            if name == "cosh":
                return ft(np.cosh(a))
            if name == "tanh":
                return ft(np.tanh(a))
            if name == "asinh":
                return ft(np.arcsinh(a))
            if name == "acosh":
                return ft(np.arccosh(a))
            if name == "atanh":
                return ft(np.arctanh(a))
            if name == "abs":
                return ft(np.abs(a))
            if name == "signum":
                return a if np.isnan(a) else ft(np.copysign(ft(1.0), a))
            if name == "floor":
                return ft(np.floor(a))
            if name == "ceil":
                return ft(np.ceil(a))
            if name == "round":
                # Rust round: half away from zero.
                if not np.isfinite(a):
                    return a
                t = ft(np.trunc(a))
                if abs(float(a) - float(t)) >= 0.5:
                    t = ft(t + np.copysign(ft(1.0), a))
                return ft(np.copysign(t, a)) if t == 0 else t
            if name == "trunc":
                return ft(np.trunc(a))
            if name == "fract":
                return ft(a - np.trunc(a))
        raise ValueError(name)


_SCALARS = {np.dtype(np.float64): _Scalar(np.float64), np.dtype(np.float32): _Scalar(np.float32)}


# ---------------------------------------------------------------------------
# The tape.
# ---------------------------------------------------------------------------

class TapeValidationError(ValueError):
    """Structural violation (``src/bytecode_tape/mod.rs:44-53``)."""


class BytecodeTape:
    """Re-evaluable tape: parallel ``opcodes`` / ``arg_indices`` / ``values`` arrays.

    Field meaning follows ``src/bytecode_tape/mod.rs:123-142``.  ``values`` holds the
    recording-time value of every slot; the ``Const`` entries of it are the tape
    constants that every sweep starts from (``forward_into``,
    ``src/bytecode_tape/forward.rs:194-229``).
    """

    def __init__(self, dtype=np.float64):
        self.dtype = np.dtype(dtype)
        self._s = _SCALARS[self.dtype]
        self.opcodes: List[int] = []
        self.arg0: List[int] = []
        self.arg1: List[int] = []
        self.values: list = []
        self.num_inputs = 0
        self.output_index = 0
        self.output_indices: List[int] = []
        self.has_custom_ops = False

    # -- construction (src/bytecode_tape/mod.rs:240-382) ----------------------
    def _push_entry(self, op: int, a0: int, a1: int, value) -> int:
        idx = len(self.opcodes)
        if idx >= 0xFFFFFFFF:
            raise OverflowError("tape entry count overflows u32 indexing")
        self.opcodes.append(int(op))
        self.arg0.append(int(a0))
        self.arg1.append(int(a1))
        self.values.append(self._s.c(value))
        return idx

    def new_input(self, value) -> int:
        self.num_inputs += 1
        return self._push_entry(OpCode.Input, UNUSED, UNUSED, value)

    def push_const(self, value) -> int:
        return self._push_entry(OpCode.Const, UNUSED, UNUSED, value)

    def push_op(self, op: int, arg0: int, arg1: int, value) -> int:
        arg0_const = self.opcodes[arg0] == OpCode.Const
        arg1_const = arg1 == UNUSED or self.opcodes[arg1] == OpCode.Const
        if arg0_const and arg1_const:
            return self.push_const(value)
        if (arg0_const or arg1_const) and arg1 != UNUSED:
            idx = self._try_algebraic_simplify(op, arg0, arg1, arg0_const, arg1_const)
            if idx is not None:
                return idx
        return self._push_entry(op, arg0, arg1, value)

    def _try_algebraic_simplify(self, op, arg0, arg1, arg0_const, arg1_const):
        # src/bytecode_tape/mod.rs:309-354
        if op == OpCode.Add:
            if arg1_const:
                c = self.values[arg1]
                if c == 0 and np.signbit(c):
                    return arg0
            if arg0_const:
                c = self.values[arg0]
                if c == 0 and np.signbit(c):
                    return arg1
        elif op == OpCode.Sub and arg1_const:
            c = self.values[arg1]
            if c == 0 and not np.signbit(c):
                return arg0
        elif op == OpCode.Mul:
            if arg1_const and self.values[arg1] == 1:
                return arg0
            if arg0_const and self.values[arg0] == 1:
                return arg1
        elif op == OpCode.Div and arg1_const and self.values[arg1] == 1:
            return arg0
        return None

    def push_powi(self, arg0: int, exp: int, value) -> int:
        if self.opcodes[arg0] == OpCode.Const:
            return self.push_const(value)
        if exp == 0 and value == 1:
            return self.push_const(1.0)
        if exp == 1:
            return arg0
        if exp == -1:
            return self.push_op(OpCode.Recip, arg0, UNUSED, value)
        return self._push_entry(OpCode.Powi, arg0, powi_exp_encode(exp), value)

    def set_output(self, index: int) -> None:
        self.output_index = int(index)

    def set_outputs(self, indices: Sequence[int]) -> None:
        n = len(self.values)
        for i, idx in enumerate(indices):
            if not (0 <= idx < n):
                raise IndexError(f"set_outputs: indices[{i}] = {idx} is out of range (tape has {n} values)")
        self.output_indices = [int(i) for i in indices]
        if indices:
            self.output_index = int(indices[0])

    # -- queries ---------------------------------------------------------------
    def num_ops(self) -> int:
        return len(self.opcodes)

    num_variables_count = num_ops

    def num_outputs(self) -> int:
        return 1 if not self.output_indices else len(self.output_indices)

    def all_output_indices(self) -> List[int]:
        return [self.output_index] if not self.output_indices else list(self.output_indices)

    def arrays(self):
        """SoA view used by the GPU upload and by the oracle."""
        return (
            np.asarray(self.opcodes, dtype=np.uint32),
            np.asarray(self.arg0, dtype=np.uint32),
            np.asarray(self.arg1, dtype=np.uint32),
            np.asarray(self.values, dtype=self.dtype),
        )

    def validate(self) -> None:
        """Structural invariants of ``BytecodeTape::validate`` (``src/bytecode_tape/mod.rs:575-705``).

        Delegates to the native validator in the library so the host checks and the
        upload checks are one implementation.
        """
        from . import _lib

        op, a0, a1, vals = self.arrays()
        msg = _lib.validate_bytecode_tape(op, a0, a1, len(vals), self.num_inputs, self.output_index,
                                          np.asarray(self.output_indices, dtype=np.uint32),
                                          1 if self.has_custom_ops else 0)
        if msg is not None:
            raise TapeValidationError(msg)

    # -- serialisation (src/bytecode_tape/serde_support.rs:11-100) -------------
    def to_json(self) -> str:
        names = [OpCode(o).name for o in self.opcodes]
        return json.dumps({
            "opcodes": names,
            "arg_indices": [[a, b] for a, b in zip(self.arg0, self.arg1)],
            "values": [float(v) for v in self.values],
            "num_inputs": self.num_inputs,
            "num_variables": len(self.values),
            "output_index": self.output_index,
            "output_indices": list(self.output_indices),
            "custom_second_args": {},
        })

    @classmethod
    def from_json(cls, text: str, dtype=np.float64) -> "BytecodeTape":
        """Deserialize (``src/bytecode_tape/serde_support.rs:35-100``): custom ops and their
        side table are refused, ``num_variables`` must equal the entry count, and the
        whole tape is validated; every corrupt payload raises ``TapeValidationError``."""
        d = json.loads(text)
        try:
            ops = [int(OpCode[o]) if isinstance(o, str) else int(o) for o in d["opcodes"]]
            args = [[int(a[0]), int(a[1])] for a in d["arg_indices"]]
            values = list(d["values"])
            num_inputs = int(d["num_inputs"])
            num_variables = int(d["num_variables"])
            output_index = int(d["output_index"])
            output_indices = [int(i) for i in d.get("output_indices", [])]
            custom_second_args = d.get("custom_second_args", {}) or {}
        except (KeyError, TypeError, ValueError, IndexError) as e:
            raise TapeValidationError(f"malformed tape payload: {e}") from e
        if OpCode.Custom in ops:
            i = ops.index(OpCode.Custom)
            raise TapeValidationError(f"opcodes[{i}] is Custom, which cannot be deserialized "
                                      "(custom ops have no serializable callback)")
        if custom_second_args:
            raise TapeValidationError("custom_second_args must be empty: custom ops cannot be deserialized")
        if num_variables != len(ops):
            raise TapeValidationError(f"num_variables ({num_variables}) != opcodes.len() ({len(ops)})")
        if len(args) != len(ops):
            raise TapeValidationError(f"invalid bytecode tape: arg_indices.len() ({len(args)}) != "
                                      f"opcodes.len() ({len(ops)})")
        if len(values) != len(ops):
            raise TapeValidationError(f"invalid bytecode tape: values.len() ({len(values)}) != "
                                      f"opcodes.len() ({len(ops)})")
        t = cls(dtype)
        t.opcodes = ops
        t.arg0 = [a[0] for a in args]
        t.arg1 = [a[1] for a in args]
        t.values = [t._s.c(v) for v in values]
        t.num_inputs = num_inputs
        t.output_index = output_index
        t.output_indices = output_indices
        t.validate()
        return t


# ---------------------------------------------------------------------------
# Recording front-end.
# ---------------------------------------------------------------------------

_active = threading.local()


def _tape() -> BytecodeTape:
    t = getattr(_active, "tape", None)
    if t is None:
        raise RuntimeError("no active recording; use echidna_b200.record")
    return t


def _ensure_on_tape(x: "BReverse", t: BytecodeTape) -> int:
    # src/breverse.rs:22-30
    if x.index == CONSTANT:
        return t.push_const(x.value)
    return x.index


def _lift(x) -> "BReverse":
    return x if isinstance(x, BReverse) else BReverse.constant(x)


class BReverse:
    """Recording scalar (``src/breverse.rs:56-63``).

    Arithmetic with another ``BReverse`` or a plain number records an opcode on the
    active tape; a plain number becomes a fresh ``Const`` slot at each use.
    """

    __slots__ = ("value", "index")

    def __init__(self, value, index: int):
        self.value = value
        self.index = index

    @staticmethod
    def constant(value) -> "BReverse":
        return BReverse(value, CONSTANT)

    # -- helpers (src/traits/breverse_ops.rs:16-40) --
    def _binary(self, other, op: int, fname: str) -> "BReverse":
        t = _tape()
        other = _lift(other)
        value = t._s.call(fname, self.value, other.value)
        li = _ensure_on_tape(self, t)
        ri = _ensure_on_tape(other, t)
        return BReverse(value, t.push_op(op, li, ri, value))

    def _rbinary(self, other, op: int, fname: str) -> "BReverse":
        # scalar (lhs) OP self: the constant is pushed first.
        t = _tape()
        value = t._s.call(fname, other, self.value)
        c = t.push_const(other)
        ri = _ensure_on_tape(self, t)
        return BReverse(value, t.push_op(op, c, ri, value))

    def _scalar_rhs(self, other, op: int, fname: str) -> "BReverse":
        # self OP scalar: self first, then the constant.
        t = _tape()
        value = t._s.call(fname, self.value, other)
        si = _ensure_on_tape(self, t)
        c = t.push_const(other)
        return BReverse(value, t.push_op(op, si, c, value))

    def _unary(self, op: int, fname: str, value=None) -> "BReverse":
        t = _tape()
        if value is None:
            value = t._s.call(fname, self.value)
        xi = _ensure_on_tape(self, t)
        return BReverse(value, t.push_op(op, xi, UNUSED, value))

    def _arith(self, other, op, fname):
        if isinstance(other, BReverse):
            return self._binary(other, op, fname)
        return self._scalar_rhs(other, op, fname)

    # -- operators --
    def __add__(self, o):
        return self._arith(o, OpCode.Add, "add")

    def __radd__(self, o):
        return self._rbinary(o, OpCode.Add, "add")

    def __sub__(self, o):
        return self._arith(o, OpCode.Sub, "sub")

    def __rsub__(self, o):
        return self._rbinary(o, OpCode.Sub, "sub")

    def __mul__(self, o):
        return self._arith(o, OpCode.Mul, "mul")

    def __rmul__(self, o):
        return self._rbinary(o, OpCode.Mul, "mul")

    def __truediv__(self, o):
        return self._arith(o, OpCode.Div, "div")

    def __rtruediv__(self, o):
        return self._rbinary(o, OpCode.Div, "div")

    def __mod__(self, o):
        return self._arith(o, OpCode.Rem, "rem")

    def __rmod__(self, o):
        return self._rbinary(o, OpCode.Rem, "rem")

    def __neg__(self):
        return self._unary(OpCode.Neg, "neg")

    # comparisons act on values (src/traits/breverse_ops.rs:284-298)
    def __lt__(self, o):
        return self.value < _lift(o).value

    def __le__(self, o):
        return self.value <= _lift(o).value

    def __gt__(self, o):
        return self.value > _lift(o).value

    def __ge__(self, o):
        return self.value >= _lift(o).value

    # -- num_traits::Float methods (src/traits/breverse_num_traits.rs) --
    def recip(self):
        return self._unary(OpCode.Recip, "recip")

    def sqrt(self):
        return self._unary(OpCode.Sqrt, "sqrt")

    def cbrt(self):
        return self._unary(OpCode.Cbrt, "cbrt")

    def powi(self, n: int):
        t = _tape()
        val = t._s.powi(self.value, int(n))
        xi = _ensure_on_tape(self, t)
        return BReverse(val, t.push_powi(xi, int(n), val))

    def powf(self, n):
        return self._binary(_lift(n), OpCode.Powf, "powf")

    def exp(self):
        return self._unary(OpCode.Exp, "exp")

    def exp2(self):
        return self._unary(OpCode.Exp2, "exp2")

    def exp_m1(self):
        return self._unary(OpCode.ExpM1, "exp_m1")

    def ln(self):
        return self._unary(OpCode.Ln, "ln")

    def log2(self):
        return self._unary(OpCode.Log2, "log2")

    def log10(self):
        return self._unary(OpCode.Log10, "log10")

    def ln_1p(self):
        return self._unary(OpCode.Ln1p, "ln_1p")

    def log(self, base):
        return self.ln() / _lift(base).ln()

    def sin(self):
        return self._unary(OpCode.Sin, "sin")

    def cos(self):
        return self._unary(OpCode.Cos, "cos")

    def tan(self):
        return self._unary(OpCode.Tan, "tan")

    def sin_cos(self):
        return self.sin(), self.cos()

    def asin(self):
        return self._unary(OpCode.Asin, "asin")

    def acos(self):
        return self._unary(OpCode.Acos, "acos")

    def atan(self):
        return self._unary(OpCode.Atan, "atan")

    def atan2(self, other):
        return self._binary(_lift(other), OpCode.Atan2, "atan2")

    def sinh(self):
        return self._unary(OpCode.Sinh, "sinh")

    def cosh(self):
        return self._unary(OpCode.Cosh, "cosh")

    def tanh(self):
        return self._unary(OpCode.Tanh, "tanh")

    def asinh(self):
        return self._unary(OpCode.Asinh, "asinh")

    def acosh(self):
        return self._unary(OpCode.Acosh, "acosh")

    def atanh(self):
        return self._unary(OpCode.Atanh, "atanh")

    def __abs__(self):
        return self.abs()

    def abs(self):
        return self._unary(OpCode.Abs, "abs")

    def signum(self):
        return self._unary(OpCode.Signum, "signum")

    def floor(self):
        return self._unary(OpCode.Floor, "floor")

    def ceil(self):
        return self._unary(OpCode.Ceil, "ceil")

    def round(self):
        return self._unary(OpCode.Round, "round")

    def trunc(self):
        return self._unary(OpCode.Trunc, "trunc")

    def fract(self):
        return self._unary(OpCode.Fract, "fract")

    def hypot(self, other):
        return self._binary(_lift(other), OpCode.Hypot, "hypot")

    def max(self, other):
        return self._binary(_lift(other), OpCode.Max, "max")

    def min(self, other):
        return self._binary(_lift(other), OpCode.Min, "min")

    def mul_add(self, a, b):
        return self * a + b

    def __repr__(self):
        return f"BReverse({self.value!r}, index={self.index})"


class _Guard:
    def __init__(self, tape: BytecodeTape):
        self.tape = tape

    def __enter__(self):
        self.prev = getattr(_active, "tape", None)
        _active.tape = self.tape
        return self.tape

    def __exit__(self, *exc):
        _active.tape = self.prev
        return False


def record(f: Callable[[List[BReverse]], BReverse], x: Sequence[float], dtype=np.float64):
    """Record ``f`` at ``x`` (``src/api.rs:197-216``). Returns ``(tape, value)``."""
    tape = BytecodeTape(dtype)
    inputs = [BReverse(tape._s.c(v), tape.new_input(v)) for v in x]
    with _Guard(tape):
        out = f(inputs)
    out = _lift(out)
    tape.set_output(_ensure_on_tape(out, tape))
    return tape, out.value


def record_multi(f, x: Sequence[float], dtype=np.float64):
    """Record a vector-valued ``f`` (``src/api.rs:232-269``)."""
    tape = BytecodeTape(dtype)
    inputs = [BReverse(tape._s.c(v), tape.new_input(v)) for v in x]
    with _Guard(tape):
        outs = f(inputs)
    if not outs:
        raise ValueError("record_multi: closure returned zero outputs")
    outs = [_lift(o) for o in outs]
    idx = [_ensure_on_tape(o, tape) for o in outs]
    tape.set_outputs(idx)
    tape.set_output(idx[0])
    return tape, [o.value for o in outs]


def constant(value) -> BReverse:
    """``BReverse::constant`` (``src/breverse.rs:78-86``)."""
    return BReverse.constant(value)
