"""Algorithmic work per evaluation unit of a tape, by sweep and value kind.

The roofline of a sweep is ``t_roof = max(B_alg / BW_hbm, F_alg / P_pipe)``.
``B_alg`` is the store-all byte model.  Each trajectory value is written once in
the forward sweep and read once in the reverse: ``2 s T_val``.  ``F_alg``
counts the scalar floating-point operations that a direct implementation of
each tape op needs in the sweep's value kind:

* plain values ``T`` (forward, gradient);
* ``Dual<T>`` = (re, eps) (JVP; HVP as forward-over-reverse);
* ``Jet<T,K>`` = (c_0 .. c_{K-1}) (Taylor).

Specials (libm-class calls such as exp, tanh and ln) are counted apart from
flops and are not folded into ``F_alg``.  A multiply whose operand is a
constant is a scale: ``K`` multiplies for a jet, not the Cauchy product of a
constant jet.  Only the ops that reach an output count (dead-op elimination,
as the lowering does).  The reverse sweep counts the ops from which the seed
is reachable.

Per-op costs (flops, specials):

==================  =========  ============  ====================
op class            T          Dual<T>       Jet<T,K>
==================  =========  ============  ====================
add / sub           1          2             K
neg                 1          2             K
mul by constant     1          2             K
mul                 1          4             K(K+1)/2 mul + K(K-1)/2 add = K^2
div by constant     1          2             K
div                 1          5             K^2 + 1
sqrt / recip        1          3             K^2 + 1
unary special       0, 1       1, 1 + 1 mul  K^2, 1
binary special      1, 1       6, 2          2 K^2, 2
cheap unary         1          1             1
==================  =========  ============  ====================

Reverse (gradient in ``T``, HVP in ``Dual<T>``).  Each variable operand takes
one adjoint update ``adj_a += d * adj_r``: 2 flops in ``T``, 6 in ``Dual``
(a Dual multiply and add), or 4 in ``Dual`` when ``d`` is a constant.
Partials cost: div 2 (``T``) or 8 (``Dual``); unary specials 1 special plus
2 flops (``T``) or 2 specials plus 6 flops (``Dual``); binary specials 2
specials plus 4 (``T``) or 12 (``Dual``); add, sub, neg and mul are free.
"""
from __future__ import annotations

import numpy as np

from .tape import OpCode

_CHEAP = {OpCode.Abs, OpCode.Signum, OpCode.Floor, OpCode.Ceil, OpCode.Round, OpCode.Trunc, OpCode.Fract,
          OpCode.Max, OpCode.Min}
_BINSPECIAL = {OpCode.Rem, OpCode.Powf, OpCode.Atan2, OpCode.Hypot}
_ALGEBRAIC = {OpCode.Sqrt, OpCode.Recip, OpCode.Powi}


def _classes(tape):
    """Class counts (forward ops that reach an output; reverse ops that reach the seed),
    cached on the tape object."""
    cached = getattr(tape, "_opcost_classes", None)
    if cached is None:
        cached = _count_classes(tape)
        try:
            tape._opcost_classes = cached
        except AttributeError:
            pass
    return cached


def _count_classes(tape):
    op, a0, a1, _ = tape.arrays()
    nv = len(op)
    outs = tape.all_output_indices()
    binary = (op >= OpCode.Add) & (op <= OpCode.Min)
    is_const = op == OpCode.Const
    # liveness backwards from the outputs
    live = np.zeros(nv, bool)
    live[outs] = True
    for i in range(nv - 1, -1, -1):
        if not live[i] or op[i] <= OpCode.Const:
            continue
        live[a0[i]] = True
        if binary[i]:
            live[a1[i]] = True
    # the seed (first output) reaches ops backwards; an op is in the reverse sweep
    # when its result can reach the seed and it has a variable operand
    reach = np.zeros(nv, bool)
    reach[outs[0]] = True
    for i in range(nv - 1, -1, -1):
        if not reach[i] or op[i] <= OpCode.Const:
            continue
        if not is_const[a0[i]]:
            reach[a0[i]] = True
        if binary[i] and not is_const[a1[i]]:
            reach[a1[i]] = True

    def tally(mask):
        c = dict(add=0, neg=0, mul_c=0, mul=0, div_c=0, div=0, alg=0, unary=0, binspecial=0, cheap=0,
                 var_operands=0, const_partial_operands=0)
        for i in np.nonzero(mask & (op > OpCode.Const))[0]:
            o = int(op[i])
            ca = bool(is_const[a0[i]])
            cb = bool(binary[i] and is_const[a1[i]])
            nvar = (0 if ca else 1) + (1 if binary[i] and not cb else 0)
            c["var_operands"] += nvar
            if o in (OpCode.Add, OpCode.Sub):
                c["add"] += 1
                c["const_partial_operands"] += nvar
            elif o == OpCode.Neg:
                c["neg"] += 1
                c["const_partial_operands"] += nvar
            elif o == OpCode.Mul:
                if ca or cb:
                    c["mul_c"] += 1
                    c["const_partial_operands"] += nvar
                else:
                    c["mul"] += 1
            elif o == OpCode.Div:
                if cb:
                    c["div_c"] += 1
                else:
                    c["div"] += 1
            elif o in _ALGEBRAIC:
                c["alg"] += 1
            elif o in _CHEAP:
                c["cheap"] += 1
            elif o in _BINSPECIAL:
                c["binspecial"] += 1
            else:
                c["unary"] += 1
        return c

    return tally(live), tally(live & reach)


def forward_cost(c, kind: str, K: int = 1):
    """(flops, specials) of one unit's forward sweep for class counts ``c``."""
    if kind == "plain":
        f = c["add"] + c["neg"] + c["mul_c"] + c["mul"] + c["div_c"] + c["div"] + c["alg"] + c["cheap"] \
            + c["binspecial"]
        s = c["unary"] + c["binspecial"]
    elif kind == "dual":
        f = 2 * (c["add"] + c["neg"] + c["mul_c"] + c["div_c"]) + 4 * c["mul"] + 5 * c["div"] + 3 * c["alg"] \
            + c["unary"] + c["cheap"] + 6 * c["binspecial"]
        s = c["unary"] + 2 * c["binspecial"]
    elif kind == "jet":
        f = K * (c["add"] + c["neg"] + c["mul_c"] + c["div_c"]) + K * K * (c["mul"] + c["unary"]) \
            + (K * K + 1) * (c["div"] + c["alg"]) + c["cheap"] + 2 * K * K * c["binspecial"]
        s = c["unary"] + 2 * c["binspecial"]
    else:
        raise ValueError(kind)
    return int(f), int(s)


def reverse_cost(c, kind: str):
    """(flops, specials) of one unit's reverse sweep (``plain`` gradient, ``dual`` HVP)."""
    var, cst = c["var_operands"], c["const_partial_operands"]
    if kind == "plain":
        f = 2 * var + 2 * (c["div"] + c["div_c"]) + 2 * c["unary"] + c["alg"] + 4 * c["binspecial"]
        s = c["unary"] + 2 * c["binspecial"] + c["alg"]
    elif kind == "dual":
        f = 6 * (var - cst) + 4 * cst + 8 * (c["div"] + c["div_c"]) + 6 * c["unary"] + 4 * c["alg"] \
            + 12 * c["binspecial"]
        s = 2 * c["unary"] + 4 * c["binspecial"] + c["alg"]
    else:
        raise ValueError(kind)
    return int(f), int(s)


def sweep_cost(tape, sweep: str, K: int = 3):
    """Per-unit algorithmic (flops, specials) of a sweep: ``forward``, ``gradient``,
    ``hvp`` (per-point, forward-over-reverse), ``jvp`` or ``taylor`` (order ``K``)."""
    fwd, rev = _classes(tape)
    if sweep == "forward":
        return forward_cost(fwd, "plain")
    if sweep == "gradient":
        a, b = forward_cost(fwd, "plain"), reverse_cost(rev, "plain")
        return a[0] + b[0], a[1] + b[1]
    if sweep == "hvp":
        a, b = forward_cost(fwd, "dual"), reverse_cost(rev, "dual")
        return a[0] + b[0], a[1] + b[1]
    if sweep == "jvp":
        return forward_cost(fwd, "dual")
    if sweep == "taylor":
        return forward_cost(fwd, "jet", K)
    raise ValueError(sweep)


def pipe_peak_ops(f64: bool, sm_mhz: float, sms: int = 148) -> float:
    """Scalar FP ops per second of the CUDA-core pipe, one op per lane per clock
    (no FMA: the sweeps round each + and * like the CPU).  FP64 at half rate."""
    return sms * 128 * sm_mhz * 1e6 * (0.5 if f64 else 1.0)


def roofline(bytes_alg: float, flops_alg: float, seconds: float, hbm_gbs: float, pipe_ops: float) -> dict:
    """``t_roof = max(B / BW, F / P)`` and its ratio to the measured time."""
    t_b = bytes_alg / (hbm_gbs * 1e9)
    t_f = flops_alg / pipe_ops
    t_roof = max(t_b, t_f)
    return {"t_roof_ms": t_roof * 1e3, "t_hbm_ms": t_b * 1e3, "t_pipe_ms": t_f * 1e3,
            "binding": "hbm" if t_b >= t_f else "pipe", "frac": t_roof / seconds}
