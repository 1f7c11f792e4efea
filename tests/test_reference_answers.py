"""More of the reference's own asserted answers, transcribed case by case and
checked on the oracle (CPU) and on the engine (GPU-marked copies).

The first group restates the reference's CUDA and GPU-fix tests
(``tests/gpu_cuda_kernel_parity.rs``, ``tests/gpu_kernel_parity.rs``,
``tests/phase7_gpu_fixes.rs``, ``tests/phase7_gpu_parity.rs``): an f64-recorded
tape uploaded with ``from_tape_f64_lossy`` and evaluated in f32, with the
reference's own tolerances.  The second group restates CPU tests of the same
conventions on the bytecode tape in f64:

* ``tests/atan2_extreme_magnitudes.rs`` and ``tests/asinh_acosh_large.rs``;
* ``tests/taylor.rs``: its tape jets and, as jets of one-op tapes, the series
  of its Taylor-type tests;
* ``tests/hypot_leading_zero_parity.rs`` (jets built from polynomials);
* ``tests/opcode_edge_cases.rs`` as forward values and gradients of one-op tapes;
* ``tests/stde_nonfinite_samples.rs`` (the Welford accumulator);
* the tape cases of ``tests/regressions.rs``;
* ``tests/stde_higher_order.rs`` (k-th order diagonals, parabolic diffusion),
  ``tests/stde_pipeline.rs`` (``estimate`` / ``estimate_weighted``),
  ``tests/stde_core.rs`` and ``tests/stde_stats.rs`` (known Hessians, Welford
  statistics, control variate) and ``tests/bytecode_tape.rs`` (gradients
  through shared subexpressions);
* the f32 jet tests of ``tests/gpu_stde.rs`` that the reference runs on its
  CUDA backend.

Dual-number cases become JVPs of the one-op tape (a ``Dual::new(x, 1)`` operand
is a seeded input, a ``Dual::constant`` operand a tape constant).  The oracle
runs every case in the precision the case names (its f32 mode rounds the tape
constants to f32, as ``from_tape_f64_lossy`` does).
"""
import math

import numpy as np
import pytest

from echidna_b200 import constant, record
from echidna_b200.gpu import GpuTapeData
from oracle.oracle import OracleTape

NAN = math.nan
INF = math.inf


def _close(got, want, rel):
    return abs(got - want) <= rel * abs(want)


# name -> (reference, recorder, record point, precision, call, inputs, extra, check)
#   call: "forward" | "gradient" | "hvp" (one x, directions) | "jvp" | "taylor"
#   check(res): res has "value", "grad", "hv", "tan" or "jet" (coefficients of output 0)
CASES = {
    # ── CUDA backend tests (f64 tape, f32 evaluation) ──
    "atan2_1e20": ("gpu_cuda_kernel_parity.rs:20-46", lambda v: v[0].atan2(v[1]), (1.0, 1.0), "f32", "gradient",
                   (1e20, 1e20), None,
                   lambda r: all(math.isfinite(g) and g != 0.0 for g in r["grad"])),
    "asinh_1e20": ("gpu_cuda_kernel_parity.rs:51-68", lambda v: v[0].asinh(), (1.0,), "f32", "gradient", (1e20,),
                   None, lambda r: math.isfinite(r["grad"][0]) and r["grad"][0] > 0
                   and _close(r["grad"][0], 1e-20, 1e-5)),
    "acosh_1e20": ("gpu_cuda_kernel_parity.rs:71-88", lambda v: v[0].acosh(), (2.0,), "f32", "gradient", (1e20,),
                   None, lambda r: math.isfinite(r["grad"][0]) and r["grad"][0] > 0
                   and _close(r["grad"][0], 1e-20, 1e-5)),
    "powf_negative_base": ("gpu_cuda_kernel_parity.rs:93-112", lambda v: v[0].powf(constant(3.0)), (-2.0,), "f32",
                           "gradient", (-2.0,), None,
                           lambda r: math.isfinite(r["grad"][0]) and _close(r["grad"][0], 12.0, 1e-5)),
    "max_nan_operand": ("gpu_cuda_kernel_parity.rs:117-134", lambda v: v[0].max(v[1]), (1.5, NAN), "f32", "gradient",
                        (1.5, NAN), None, lambda r: r["grad"][0] == 1.0 and r["grad"][1] == 0.0),
    "fract_negative": ("gpu_cuda_kernel_parity.rs:139-163", lambda v: v[0].fract(), (-1.3,), "f32", "forward",
                       (-1.3,), None,
                       lambda r: abs(r["value"][0] - float(np.float32(-1.3) - np.trunc(np.float32(-1.3)))) < 1e-6
                       and r["value"][0] < 0.0),
    "abs_signed_zero": ("gpu_kernel_parity.rs abs_signed_zero", lambda v: v[0].abs(), (-0.0,), "f32", "gradient",
                        (-0.0,), None, lambda r: r["grad"][0] == 0.0),
    "atan_1e20": ("phase7_gpu_fixes.rs:87-104", lambda v: v[0].atan(), (1.0,), "f32", "gradient", (1e20,), None,
                  lambda r: math.isfinite(r["grad"][0]) and r["grad"][0] > 0.0),
    "atan_3e9": ("phase7_gpu_fixes.rs:60-83", lambda v: v[0].atan(), (1.0,), "f32", "gradient", (3e9,), None,
                 lambda r: r["grad"][0] > 0.0 and _close(r["grad"][0], 1.0 / (1.0 + 9e18), 1e-3)),
    "div_small_denominator": ("phase7_gpu_fixes.rs:112-135", lambda v: v[0] / v[1], (1.0, 1.0), "f32", "gradient",
                              (1e-10, 1e-20), None, lambda r: math.isfinite(r["grad"][1])),
    "hypot_inf_1": ("phase7_gpu_fixes.rs:148-166", lambda v: v[0].hypot(v[1]), (1.0, 1.0), "f32", "forward",
                    (INF, 1.0), None, lambda r: r["value"][0] == INF),
    "hypot_inf_inf": ("phase7_gpu_fixes.rs:169-188", lambda v: v[0].hypot(v[1]), (1.0, 1.0), "f32", "forward",
                      (INF, INF), None, lambda r: r["value"][0] == INF),
    "hypot_1e20": ("phase7_gpu_fixes.rs:191-222", lambda v: v[0].hypot(v[1]), (1.0, 1.0), "f32", "gradient",
                   (1e20, 1e20), None,
                   lambda r: math.isfinite(r["value"][0]) and all(math.isfinite(g) for g in r["grad"])
                   and _close(r["value"][0], float(np.float32(math.sqrt(2.0)) * np.float32(1e20)), 1e-4)),
    "expm1_small": ("phase7_gpu_fixes.rs:257-285", lambda v: v[0].exp_m1(), (1.0,), "f32", "gradient", (1e-6,), None,
                    lambda r: abs(r["value"][0] - math.expm1(1e-6)) < 1e-12),
    "ln1p_small": ("phase7_gpu_fixes.rs:290-310", lambda v: v[0].ln_1p(), (1.0,), "f32", "gradient", (1e-6,), None,
                   lambda r: abs(r["value"][0] - math.log1p(1e-6)) < 1e-12),
    "powi1_at_zero_hvp": ("phase7_gpu_fixes.rs:322-342", lambda v: v[0].powi(1), (0.0,), "f32", "hvp", (0.0,),
                          (1.0,), lambda r: math.isfinite(r["hv"][0]) and r["hv"][0] == 0.0),
    "powf3_negative_base_hvp": ("phase7_gpu_fixes.rs:373-410", lambda v: v[0].powf(constant(3.0)), (-2.0,), "f32",
                                "hvp", (-2.0,), (1.0,),
                                lambda r: abs(r["grad"][0] - 12.0) < 1e-3 and abs(r["hv"][0] + 12.0) < 1e-3),
    "powi3_negative_base_hvp": ("phase7_gpu_fixes.rs:373-410", lambda v: v[0].powi(3), (-2.0,), "f32", "hvp",
                                (-2.0,), (1.0,),
                                lambda r: abs(r["grad"][0] - 12.0) < 1e-3 and abs(r["hv"][0] + 12.0) < 1e-3),
    "fmad_disabled_bit_exact": ("phase7_gpu_parity.rs l25", lambda v: v[0] * v[1] + v[2],
                                (1.2345678901234567, 9.8765432109876543, 1.1111111111111111), "f32", "gradient",
                                (1.2345678901234567, 9.8765432109876543, 1.1111111111111111), None,
                                lambda r: np.float32(r["value"][0]).tobytes() == (
                                    np.float32(1.2345678901234567) * np.float32(9.8765432109876543)
                                    + np.float32(1.1111111111111111)).tobytes()),
    "rem_quotient": ("phase7_gpu_parity.rs m28", lambda v: v[0] % v[1], (5.0, 2.0), "f32", "gradient", (5.0, 2.0),
                     None, lambda r: abs(r["value"][0] - 1.0) < 1e-5 and abs(r["grad"][0] - 1.0) < 1e-5
                     and abs(r["grad"][1] + 2.0) < 1e-5),
    # ── CPU conventions on the bytecode tape (f64) ──
    "atan2_1e200_reverse": ("atan2_extreme_magnitudes.rs breverse_atan2_large_magnitudes",
                            lambda v: v[0].atan2(v[1]), (1e200, 1e200), "f64", "gradient", (1e200, 1e200), None,
                            lambda r: _close(r["grad"][0], 5e-201, 1e-10) and _close(-r["grad"][1], 5e-201, 1e-10)),
    "atan2_1e200_tangent": ("atan2_extreme_magnitudes.rs dual_atan2_large_magnitudes_finite_tangent",
                            lambda v: v[0].atan2(constant(1e200)), (1e200,), "f64", "jvp", (1e200,), (1.0,),
                            lambda r: math.isfinite(r["value"][0]) and _close(r["tan"][0], 5e-201, 1e-10)),
    "atan2_1e-200_tangent": ("atan2_extreme_magnitudes.rs dual_atan2_tiny_magnitudes_finite_tangent",
                             lambda v: v[0].atan2(constant(1e-200)), (1e-200,), "f64", "jvp", (1e-200,), (1.0,),
                             lambda r: _close(r["tan"][0], 5e199, 1e-10)),
    "atan2_mixed_tangent": ("atan2_extreme_magnitudes.rs dual_atan2_mixed_magnitudes",
                            lambda v: v[0].atan2(constant(1.0)), (1e200,), "f64", "jvp", (1e200,), (1.0,),
                            lambda r: math.isfinite(r["value"][0]) and math.isfinite(r["tan"][0])),
    "atan2_ordinary_tangent": ("atan2_extreme_magnitudes.rs dual_atan2_ordinary_inputs_unchanged",
                               lambda v: v[0].atan2(constant(4.0)), (3.0,), "f64", "jvp", (3.0,), (1.0,),
                               lambda r: abs(r["value"][0] - math.atan2(3.0, 4.0)) < 1e-12
                               and abs(r["tan"][0] - 0.16) < 1e-12),
    "atan2_origin_tangent": ("atan2_extreme_magnitudes.rs dual_atan2_origin_returns_zero_eps",
                             lambda v: v[0].atan2(constant(0.0)), (1.0,), "f64", "jvp", (0.0,), (1.0,),
                             lambda r: r["tan"][0] == 0.0),
    "asinh_1e200_tangent": ("asinh_acosh_large.rs dual_asinh_large_x", lambda v: v[0].asinh(), (1.0,), "f64", "jvp",
                            (1e200,), (1.0,), lambda r: r["tan"][0] > 0 and _close(r["tan"][0], 1e-200, 1e-10)),
    "asinh_-1e200_tangent": ("asinh_acosh_large.rs dual_asinh_large_negative_x", lambda v: v[0].asinh(), (1.0,),
                             "f64", "jvp", (-1e200,), (1.0,), lambda r: _close(r["tan"][0], 1e-200, 1e-10)),
    "asinh_2_tangent": ("asinh_acosh_large.rs dual_asinh_small_x_unchanged", lambda v: v[0].asinh(), (1.0,), "f64",
                        "jvp", (2.0,), (1.0,), lambda r: abs(r["tan"][0] - 1.0 / math.sqrt(5.0)) < 1e-12),
    "acosh_1e200_tangent": ("asinh_acosh_large.rs dual_acosh_large_x", lambda v: v[0].acosh(), (2.0,), "f64", "jvp",
                            (1e200,), (1.0,), lambda r: _close(r["tan"][0], 1e-200, 1e-10)),
    "acosh_2_tangent": ("asinh_acosh_large.rs dual_acosh_small_x_unchanged", lambda v: v[0].acosh(), (2.0,), "f64",
                        "jvp", (2.0,), (1.0,), lambda r: abs(r["tan"][0] - 1.0 / math.sqrt(3.0)) < 1e-12),
    "acosh_1_tangent": ("asinh_acosh_large.rs dual_acosh_at_one_diverges", lambda v: v[0].acosh(), (2.0,), "f64",
                        "jvp", (1.0,), (1.0,), lambda r: r["value"][0] == 0.0 and r["tan"][0] == INF),
    "asinh_1e200_reverse": ("asinh_acosh_large.rs (reverse partial of the same op)", lambda v: v[0].asinh(), (1.0,),
                            "f64", "gradient", (1e200,), None, lambda r: _close(r["grad"][0], 1e-200, 1e-10)),
    "taylor_exp_plus_sin": ("taylor.rs:190-208", lambda v: v[0].exp() + v[0].sin(), (1.0,), "f64", "taylor", (1.0,),
                            ((1.0,), 3),
                            lambda r: abs(r["jet"][0] - (math.e + math.sin(1.0))) < 1e-10
                            and abs(r["jet"][1] - (math.e + math.cos(1.0))) < 1e-10
                            and abs(r["jet"][2] - (math.e - math.sin(1.0)) / 2.0) < 1e-10),
    "taylor_multivar": ("taylor.rs:226-242", lambda v: v[0] * v[1] + v[0].sin(), (1.0, 2.0), "f64", "taylor",
                        (1.0, 2.0), ((1.0, 0.0), 3),
                        lambda r: abs(r["jet"][0] - (2.0 + math.sin(1.0))) < 1e-10
                        and abs(r["jet"][1] - (2.0 + math.cos(1.0))) < 1e-10
                        and abs(r["jet"][2] + math.sin(1.0) / 2.0) < 1e-10),
    "taylor_cube": ("taylor.rs:255-257, 397-405", lambda v: v[0] * v[0] * v[0], (2.0,), "f64", "taylor", (2.0,),
                    ((1.0,), 4), lambda r: list(r["jet"]) == [8.0, 12.0, 6.0, 1.0]),
    # ── regressions.rs, tape cases (f64) ──
    "reg_powi0_at_zero": ("regressions.rs:143-156", lambda v: v[0].powi(0), (0.0,), "f64", "gradient", (0.0,), None,
                          lambda r: r["value"][0] == 1.0 and r["grad"][0] == 0.0),
    "reg_hypot_origin": ("regressions.rs:191-212", lambda v: v[0].hypot(v[1]), (0.0, 0.0), "f64", "gradient",
                         (0.0, 0.0), None, lambda r: r["value"][0] == 0.0 and r["grad"] == [0.0, 0.0]),
    "reg_rem_partials": ("regressions.rs:522-530", lambda v: v[0] % v[1], (7.0, 3.0), "f64", "gradient", (7.0, 3.0),
                         None, lambda r: r["value"][0] == 1.0 and r["grad"] == [1.0, -2.0]),
    "reg_max_nan": ("regressions.rs:546-553", lambda v: v[0].max(v[1]), (5.0, NAN), "f64", "gradient", (5.0, NAN),
                    None, lambda r: r["value"][0] == 5.0 and r["grad"][0] == 1.0),
    "reg_min_nan": ("regressions.rs:555-562", lambda v: v[0].min(v[1]), (5.0, NAN), "f64", "gradient", (5.0, NAN),
                    None, lambda r: r["value"][0] == 5.0 and r["grad"][0] == 1.0),
    "reg_max_nan_replay": ("regressions.rs:564-571", lambda v: v[0].max(v[1]), (3.0, 4.0), "f64", "gradient",
                           (5.0, NAN), None, lambda r: r["grad"][0] == 1.0),
    "reg_atan2_origin": ("regressions.rs:603-610", lambda v: v[0].atan2(v[1]), (0.0, 0.0), "f64", "gradient",
                         (0.0, 0.0), None, lambda r: all(math.isfinite(g) for g in r["grad"])),
    "reg_powf_zero_exponent": ("regressions.rs:664-674", lambda v: v[0].powf(v[1]), (2.0, 0.0), "f64", "gradient",
                               (2.0, 0.0), None, lambda r: r["value"][0] == 1.0 and r["grad"][0] == 0.0
                               and abs(r["grad"][1] - math.log(2.0)) < 1e-12),
    "reg_powf_zero_base": ("regressions.rs:686-692", lambda v: v[0].powf(v[1]), (0.0, 2.0), "f64", "gradient",
                           (0.0, 2.0), None, lambda r: r["value"][0] == 0.0 and r["grad"][0] == 0.0),
}

# opcode_edge_cases.rs (TOL = 1e-10): eval_forward and reverse_partials of one op,
# as the forward value and the gradient of a one-op tape in f64
_T = 1e-10
_ok = lambda got, want: abs(got - want) < _T  # noqa: E731
_UN = lambda f: (lambda v: f(v[0]))  # noqa: E731
_BI = lambda f: (lambda v: f(v[0], v[1]))  # noqa: E731
OPCODE_EDGE = {
    "add_nan": ("opcode_edge_cases.rs:16-19", _BI(lambda a, b: a + b), (NAN, 1.0), "forward", lambda r: math.isnan(r)),
    "mul_nan": ("opcode_edge_cases.rs:22-25", _BI(lambda a, b: a * b), (1.0, NAN), "forward", lambda r: math.isnan(r)),
    "div_nan": ("opcode_edge_cases.rs:37-41", _BI(lambda a, b: a / b), (NAN, 1.0), "forward", lambda r: math.isnan(r)),
    "neg_nan": ("opcode_edge_cases.rs:28-34", _UN(lambda a: -a), (NAN,), "forward", lambda r: math.isnan(r)),
    "exp_nan": ("opcode_edge_cases.rs:28-34", _UN(lambda a: a.exp()), (NAN,), "forward", lambda r: math.isnan(r)),
    "sin_nan": ("opcode_edge_cases.rs:28-34", _UN(lambda a: a.sin()), (NAN,), "forward", lambda r: math.isnan(r)),
    "sqrt_nan": ("opcode_edge_cases.rs:28-34", _UN(lambda a: a.sqrt()), (NAN,), "forward", lambda r: math.isnan(r)),
    "abs_nan": ("opcode_edge_cases.rs:28-34", _UN(lambda a: a.abs()), (NAN,), "forward", lambda r: math.isnan(r)),
    "exp_large": ("opcode_edge_cases.rs:47-49", _UN(lambda a: a.exp()), (1000.0,), "forward", lambda r: math.isinf(r)),
    "ln_zero": ("opcode_edge_cases.rs:52-55", _UN(lambda a: a.ln()), (0.0,), "forward", lambda r: r == -INF),
    "div_zero": ("opcode_edge_cases.rs:58-61", _BI(lambda a, b: a / b), (1.0, 0.0), "forward", lambda r: math.isinf(r)),
    "recip_zero": ("opcode_edge_cases.rs:64-67", _UN(lambda a: a.recip()), (0.0,), "forward", lambda r: math.isinf(r)),
    "sqrt_negative": ("opcode_edge_cases.rs:70-72", _UN(lambda a: a.sqrt()), (-1.0,), "forward",
                      lambda r: math.isnan(r)),
    "ln_negative": ("opcode_edge_cases.rs:75-77", _UN(lambda a: a.ln()), (-1.0,), "forward", lambda r: math.isnan(r)),
    "max_35": ("opcode_edge_cases.rs:84-89", _BI(lambda a, b: a.max(b)), (3.0, 5.0), "forward", lambda r: r == 5.0),
    "max_53": ("opcode_edge_cases.rs:84-89", _BI(lambda a, b: a.max(b)), (5.0, 3.0), "forward", lambda r: r == 5.0),
    "min_35": ("opcode_edge_cases.rs:84-89", _BI(lambda a, b: a.min(b)), (3.0, 5.0), "forward", lambda r: r == 3.0),
    "min_53": ("opcode_edge_cases.rs:84-89", _BI(lambda a, b: a.min(b)), (5.0, 3.0), "forward", lambda r: r == 3.0),
    "max_equal": ("opcode_edge_cases.rs:92-95", _BI(lambda a, b: a.max(b)), (4.0, 4.0), "forward", lambda r: r == 4.0),
    "min_equal": ("opcode_edge_cases.rs:92-95", _BI(lambda a, b: a.min(b)), (4.0, 4.0), "forward", lambda r: r == 4.0),
    "abs_zero": ("opcode_edge_cases.rs:98-101", _UN(lambda a: a.abs()), (0.0,), "forward", lambda r: r == 0.0),
    "abs_neg_zero": ("opcode_edge_cases.rs:98-101", _UN(lambda a: a.abs()), (-0.0,), "forward", lambda r: r == 0.0),
    "abs_neg": ("opcode_edge_cases.rs:104-107", _UN(lambda a: a.abs()), (-3.5,), "forward", lambda r: r == 3.5),
    "powi_0": ("opcode_edge_cases.rs:114-117", _UN(lambda a: a.powi(0)), (5.0,), "forward", lambda r: _ok(r, 1.0)),
    "powi_3": ("opcode_edge_cases.rs:120-123", _UN(lambda a: a.powi(3)), (2.0,), "forward", lambda r: _ok(r, 8.0)),
    "powi_-2": ("opcode_edge_cases.rs:126-129", _UN(lambda a: a.powi(-2)), (2.0,), "forward",
                lambda r: _ok(r, 0.25)),
    "floor": ("opcode_edge_cases.rs:147-153", _UN(lambda a: a.floor()), (2.7,), "forward", lambda r: r == 2.0),
    "ceil": ("opcode_edge_cases.rs:147-153", _UN(lambda a: a.ceil()), (2.3,), "forward", lambda r: r == 3.0),
    "round_half": ("opcode_edge_cases.rs:147-153", _UN(lambda a: a.round()), (2.5,), "forward", lambda r: r == 3.0),
    "trunc": ("opcode_edge_cases.rs:147-153", _UN(lambda a: a.trunc()), (-2.7,), "forward", lambda r: r == -2.0),
    "fract": ("opcode_edge_cases.rs:147-153", _UN(lambda a: a.fract()), (2.7,), "forward", lambda r: _ok(r, 0.7)),
    # reverse_partials -> gradient of the one-op tape
    "d_add": ("opcode_edge_cases.rs:160-165", _BI(lambda a, b: a + b), (2.0, 3.0), "gradient", (1.0, 1.0)),
    "d_sub": ("opcode_edge_cases.rs:167-172", _BI(lambda a, b: a - b), (5.0, 3.0), "gradient", (1.0, -1.0)),
    "d_mul": ("opcode_edge_cases.rs:174-179", _BI(lambda a, b: a * b), (3.0, 4.0), "gradient", (4.0, 3.0)),
    "d_div": ("opcode_edge_cases.rs:181-186", _BI(lambda a, b: a / b), (6.0, 3.0), "gradient", (1 / 3, -6 / 9)),
    "d_exp": ("opcode_edge_cases.rs:188-194", _UN(lambda a: a.exp()), (1.5,), "gradient", (math.exp(1.5),)),
    "d_ln": ("opcode_edge_cases.rs:196-202", _UN(lambda a: a.ln()), (2.0,), "gradient", (0.5,)),
    "d_sin": ("opcode_edge_cases.rs:204-210", _UN(lambda a: a.sin()), (0.7,), "gradient", (math.cos(0.7),)),
    "d_cos": ("opcode_edge_cases.rs:212-218", _UN(lambda a: a.cos()), (0.7,), "gradient", (-math.sin(0.7),)),
    "d_sqrt": ("opcode_edge_cases.rs:220-226", _UN(lambda a: a.sqrt()), (4.0,), "gradient", (0.25,)),
    "d_neg": ("opcode_edge_cases.rs:228-233", _UN(lambda a: -a), (5.0,), "gradient", (-1.0,)),
    "d_recip": ("opcode_edge_cases.rs:235-239", _UN(lambda a: a.recip()), (2.0,), "gradient", (-0.25,)),
    "d_powi": ("opcode_edge_cases.rs:241-247", _UN(lambda a: a.powi(3)), (2.0,), "gradient", (12.0,)),
    "d_hypot": ("opcode_edge_cases.rs:252-256", _BI(lambda a, b: a.hypot(b)), (3.0, 4.0), "gradient", (0.6, 0.8)),
    "d_atan2": ("opcode_edge_cases.rs:258-265", _BI(lambda a, b: a.atan2(b)), (1.0, 1.0), "gradient", (0.5, -0.5)),
    "d_max_first": ("opcode_edge_cases.rs:267-271", _BI(lambda a, b: a.max(b)), (5.0, 3.0), "gradient", (1.0, 0.0)),
    "d_max_second": ("opcode_edge_cases.rs:273-277", _BI(lambda a, b: a.max(b)), (3.0, 5.0), "gradient", (0.0, 1.0)),
    "d_min_first": ("opcode_edge_cases.rs:279-283", _BI(lambda a, b: a.min(b)), (3.0, 5.0), "gradient", (1.0, 0.0)),
    "d_abs_positive": ("opcode_edge_cases.rs:285-288", _UN(lambda a: a.abs()), (3.0,), "gradient", (1.0,)),
}


def _edge_check(name, value, grad):
    _, _, _, call, want = OPCODE_EDGE[name]
    if call == "forward":
        assert want(float(value)), (name, value)
    else:
        assert all(abs(float(g) - w) < _T for g, w in zip(grad, want)), (name, list(grad), want)


@pytest.mark.parametrize("name", sorted(OPCODE_EDGE))
def test_oracle_opcode_edge_cases(name):
    _, fn, x, call, _ = OPCODE_EDGE[name]
    tape = record(fn, list(x))[0]
    v, g = OracleTape(tape).gradient(np.asarray([x]))
    _edge_check(name, v[0, 0], g[0])


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(OPCODE_EDGE))
def test_gpu_opcode_edge_cases(ctx, name):
    _, fn, x, call, _ = OPCODE_EDGE[name]
    tape = record(fn, list(x))[0]
    gt = ctx.upload_tape_f64(tape)
    xa = np.asarray(x, dtype=np.float64)
    fwd = ctx.forward_batch_f64(gt, xa, 1)
    v, g = ctx.gradient_batch_f64(gt, xa, 1)
    assert np.array_equal(fwd, v, equal_nan=True)
    _edge_check(name, v[0], g)


def _poly(t, coeffs):
    """sum_k c_k t^k on the tape, built so that its jet at t = 0 along 1 is
    exactly (c_0, c_1, ..): t^k is the jet e_k, and c_k e_k and the sums of
    such small integers are exact."""
    acc = t - t
    tk = None
    for k, c in enumerate(coeffs):
        tk = t if k == 1 else (tk * t if k > 1 else None)
        if c != 0.0:
            acc = acc + (constant(c) if k == 0 else constant(c) * tk)
    return acc


# hypot_leading_zero_parity.rs: Taylor::<f64, 6> hypot of two given jets; the
# engine's jets go to order 5, so the first five coefficients are compared,
# exactly (the reference's assert is a == e)
HYPOT_JETS = {
    "peel_m2": ("hypot_leading_zero_parity.rs:30-36", [0., 0., 1., 2., 0.], [0., 0., 0., 1., 0.],
                [0., 0., 1., 2., 0.5]),
    "nondegenerate": ("hypot_leading_zero_parity.rs:88-101", [1., 2., 3., 4., 5.], [7., 8., 9., 10., 11.],
                      [7.0710678118654755, 8.20243866176395, 9.384721199907856, 10.60976955617793,
                       11.870557917596285]),
    "all_zero": ("hypot_leading_zero_parity.rs:83-85", [0.] * 5, [0.] * 5, [0.] * 5),
}


def _hypot_tape(a, b):
    return record(lambda v: _poly(v[0], a).hypot(_poly(v[0], b)), [0.5])[0]


def _tape(case):
    _, fn, x0, *_ = case
    return record(fn, list(x0))[0]


def _run_oracle(case):
    _, _, _, prec, call, x, extra, _ = case
    tape = _tape(case)
    o = OracleTape(tape, dtype=np.float32 if prec == "f32" else np.float64)
    X = np.asarray([x])
    if call == "forward":
        return {"value": o.forward(X)[0]}
    if call == "gradient":
        v, g = o.gradient(X)
        return {"value": v[0], "grad": g[0]}
    if call == "hvp":
        g, h = o.hvp(np.asarray(x), np.asarray([extra]))
        return {"grad": g[0], "hv": h[0]}
    if call == "jvp":
        v, t = o.jvp(X, np.asarray([extra]))
        return {"value": v[0], "tan": t[0]}
    dirs, order = extra
    c = o.taylor(X, np.asarray([dirs]), order)
    return {"jet": [float(c[k][0]) for k in range(order)]}


def _run_gpu(ctx, case):
    _, _, _, prec, call, x, extra, _ = case
    tape = _tape(case)
    f32 = prec == "f32"
    gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape)) if f32 else ctx.upload_tape_f64(tape)
    xa = np.asarray(x, dtype=np.float32 if f32 else np.float64)
    if call == "forward":
        return {"value": (ctx.forward_batch if f32 else ctx.forward_batch_f64)(gt, xa, 1)}
    if call == "gradient":
        v, g = (ctx.gradient_batch if f32 else ctx.gradient_batch_f64)(gt, xa, 1)
        return {"value": v, "grad": g}
    if call == "hvp":
        g, h = (ctx.hvp_batch if f32 else ctx.hvp_batch_f64)(gt, xa, np.asarray(extra, dtype=xa.dtype), 1)
        return {"grad": g, "hv": h}
    if call == "jvp":
        v, t = (ctx.tangent_forward_batch if f32 else ctx.tangent_forward_batch_f64)(
            gt, xa, np.asarray(extra, dtype=xa.dtype), 1)
        return {"value": v, "tan": t}
    dirs, order = extra
    fn = ctx.taylor_forward_kth_batch if f32 else ctx.taylor_forward_kth_batch_f64
    res = fn(gt, xa, np.asarray(dirs, dtype=xa.dtype), 1, order)
    return {"jet": [float(res.coefficients[k][0]) for k in range(order)]}


def _as_float(res):
    return {k: (v if k == "jet" else [float(e) for e in np.asarray(v, dtype=np.float64).ravel()])
            for k, v in res.items()}


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_reference_answers(name):
    case = CASES[name]
    res = _as_float(_run_oracle(case))
    assert case[-1](res), (name, case[0], res)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_gpu_reference_answers(ctx, name):
    case = CASES[name]
    res = _as_float(_run_gpu(ctx, case))
    assert case[-1](res), (name, case[0], res)


# taylor.rs:11-157 (epsilon 1e-12): Taylor::<f64, K>::variable(x0) through one op,
# i.e. the jet of a one-op tape at x0 along 1; polynomial jets built with _poly
_C1 = lambda: constant(1.0)  # noqa: E731
TAYLOR_OPS = {
    "exp_at_0": ("taylor.rs:11-20", lambda t: t.exp(), 0.0, [1.0, 1.0, 0.5, 1 / 6, 1 / 24]),
    "sin_at_0": ("taylor.rs:23-32", lambda t: t.sin(), 0.0, [0.0, 1.0, 0.0, -1 / 6, 0.0]),
    "cos_at_0": ("taylor.rs:35-44", lambda t: t.cos(), 0.0, [1.0, 0.0, -0.5, 0.0, 1 / 24]),
    "ln_1p_at_0": ("taylor.rs:47-57", lambda t: (_C1() + t).ln(), 0.0, [0.0, 1.0, -0.5, 1 / 3, -0.25]),
    "geometric": ("taylor.rs:60-68", lambda t: _C1() / (_C1() - t), 0.0, [1.0] * 5),
    "exp_at_1.5": ("taylor.rs:75-83", lambda t: t.exp(), 1.5, [math.exp(1.5), math.exp(1.5)]),
    "sin_at_0.7": ("taylor.rs:86-92", lambda t: t.sin(), 0.7, [math.sin(0.7), math.cos(0.7)]),
    "ln_at_2": ("taylor.rs:95-101", lambda t: t.ln(), 2.0, [math.log(2.0), 0.5]),
    "sqrt_at_4": ("taylor.rs:104-110", lambda t: t.sqrt(), 4.0, [2.0, 0.25]),
    "atan_at_0.5": ("taylor.rs:113-119", lambda t: t.atan(), 0.5, [math.atan(0.5), 1 / 1.25]),
    "tanh_at_0.3": ("taylor.rs:122-128", lambda t: t.tanh(), 0.3, [math.tanh(0.3), 1 / math.cosh(0.3) ** 2]),
    "cauchy_product": ("taylor.rs:135-146", lambda t: _poly(t, [1.0, 1.0]) * _poly(t, [1.0, 1.0]), 0.0,
                       [1.0, 2.0, 1.0]),
    "recursive_division": ("taylor.rs:149-157", lambda t: _poly(t, [1.0, 2.0, 1.0]) / _poly(t, [1.0, 1.0]), 0.0,
                           [1.0, 1.0, 0.0]),
}


def _taylor_op_tape(name):
    _, fn, x0, _ = TAYLOR_OPS[name]
    return record(lambda v: fn(v[0]), [x0 + 0.25])[0]


@pytest.mark.parametrize("name", sorted(TAYLOR_OPS))
def test_oracle_taylor_op_rules(name):
    _, _, x0, want = TAYLOR_OPS[name]
    c = OracleTape(_taylor_op_tape(name)).taylor(np.asarray([[x0]]), np.asarray([[1.0]]), len(want))
    got = [float(c[k][0]) for k in range(len(want))]
    assert all(abs(g - w) < 1e-12 for g, w in zip(got, want)), (name, got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(TAYLOR_OPS))
def test_gpu_taylor_op_rules(ctx, name):
    _, _, x0, want = TAYLOR_OPS[name]
    gt = ctx.upload_tape_f64(_taylor_op_tape(name))
    res = ctx.taylor_forward_kth_batch_f64(gt, np.asarray([x0]), np.ones(1), 1, len(want))
    got = [float(res.coefficients[k][0]) for k in range(len(want))]
    assert all(abs(g - w) < 1e-12 for g, w in zip(got, want)), (name, got, want)


@pytest.mark.parametrize("name", sorted(HYPOT_JETS))
def test_oracle_hypot_jets_leading_zeros(name):
    _, a, b, want = HYPOT_JETS[name]
    c = OracleTape(_hypot_tape(a, b)).taylor(np.asarray([[0.0]]), np.asarray([[1.0]]), 5)
    assert [float(c[k][0]) for k in range(5)] == want


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(HYPOT_JETS))
def test_gpu_hypot_jets_leading_zeros(ctx, name):
    _, a, b, want = HYPOT_JETS[name]
    gt = ctx.upload_tape_f64(_hypot_tape(a, b))
    res = ctx.taylor_forward_kth_batch_f64(gt, np.zeros(1), np.ones(1), 1, 5)
    assert [float(res.coefficients[k][0]) for k in range(5)] == want


@pytest.mark.gpu
def test_gpu_upload_with_empty_output_indices(ctx):
    # phase7_gpu_fixes.rs:227-250: output_indices cleared before upload; the
    # upload falls back to [output_index] and f(2) = 2*2 + 2 = 6
    tape = record(lambda v: v[0] * v[0] + v[0], [2.0])[0]
    data = GpuTapeData.from_tape_f64_lossy(tape)
    data.output_indices = np.zeros(0, dtype=np.uint32)
    gt = ctx.upload_tape(data)
    r, _ = ctx.gradient_batch(gt, np.asarray([2.0], np.float32), 1)
    assert r.size == 1 and abs(r[0] - 6.0) < 1e-5


# stde_nonfinite_samples.rs: f = exp(x0 x1) at (1, 700).  A direction through x0
# overflows the second-order coefficient (e^700 * 700^2 / 2), a non-finite sample
# that the Welford accumulator skips; the zero direction gives the finite sample 0.
LIVE, DEAD = [1.0, 0.0], [0.0, 0.0]
NONFINITE = {
    "skips_nonfinite": ("stde_nonfinite_samples.rs:28-39", [LIVE, DEAD, DEAD], 2, 0.0),
    "all_nonfinite": ("stde_nonfinite_samples.rs:42-55", [LIVE, LIVE], 0, "nan"),
}


def _exp_prod_tape():
    return record(lambda v: (v[0] * v[1]).exp(), [1.0, 700.0])[0]


def _check_estimate(num_samples, estimate, se, want_n, want_est):
    assert num_samples == want_n
    if want_est == "nan":
        assert math.isnan(estimate)
    else:
        assert estimate == want_est and math.isfinite(se)


@pytest.mark.parametrize("name", sorted(NONFINITE))
def test_oracle_laplacian_skips_nonfinite_samples(name):
    _, dirs, want_n, want_est = NONFINITE[name]
    r = OracleTape(_exp_prod_tape()).laplacian_stats_batch(np.asarray([[1.0, 700.0]]), np.asarray([dirs]))[0]
    _check_estimate(int(r[4]), float(r[1]), float(r[3]), want_n, want_est)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(NONFINITE))
def test_gpu_laplacian_skips_nonfinite_samples(ctx, name):
    from echidna_b200.stde_gpu import DIR_PER_POINT, laplacian_batch
    _, dirs, want_n, want_est = NONFINITE[name]
    gt = ctx.upload_tape_f64(_exp_prod_tape())
    r = laplacian_batch(ctx, gt, np.asarray([[1.0, 700.0]]), len(dirs), np.asarray([dirs]), DIR_PER_POINT)[0]
    _check_estimate(int(r["num_samples"]), float(r["estimate"]), float(r["standard_error"]), want_n, want_est)


def test_oracle_estimate_weighted_nonfinite_and_zero_weights():
    o = OracleTape(_exp_prod_tape())
    x = np.asarray([1.0, 700.0])
    # stde_nonfinite_samples.rs:58-69: the non-finite sample is skipped
    r = o.estimate_weighted(x, np.asarray([LIVE, DEAD]), np.asarray([1.0, 1.0]))
    assert int(r[4]) == 1 and r[1] == 0.0
    # :72-82: nothing contributes -> NaN
    r = o.estimate_weighted(x, np.asarray([LIVE]), np.asarray([1.0]))
    assert int(r[4]) == 0 and math.isnan(r[1])
    # :85-99: zero weights still count as samples
    q = OracleTape(record(lambda v: v[0] * v[0] + v[1] * v[1], [1.0, 2.0])[0])
    r = q.estimate_weighted(np.asarray([1.0, 2.0]), np.asarray([[1.0, 0.0], [0.0, 1.0]]), np.asarray([1.0, 0.0]))
    assert int(r[4]) == 2 and math.isfinite(r[1])
    # :103-111: a negative weight is rejected
    with pytest.raises(ValueError):
        q.estimate_weighted(np.asarray([1.0, 2.0]), np.asarray([[1.0, 0.0]]), np.asarray([-1.0]))


# stde_higher_order.rs: diagonal_kth_order(_stochastic) and parabolic diffusion.
# diagonal_kth_order(tape, x, k)[j] is the stochastic estimate over the single
# index j divided by n (the estimator rescales the mean by n / |J| * |J|).
def _exp_1d():
    return record(lambda v: v[0].exp(), [1.0])[0]


def _quartic():
    return record(lambda v: v[0] * v[0] * v[0] * v[0] + v[1] * v[1] * v[1] * v[1], [2.0, 3.0])[0]


def _cubic_mix():
    return record(lambda v: v[0] * v[0] * v[1] + v[1] * v[1] * v[1], [1.0, 2.0, 3.0])[0]


E = math.e
# name: (source, tape, x, k, sampled indices, estimate, tolerance)
KTH_ORDER = {
    **{f"exp_k{k}": ("stde_higher_order.rs:39-51", _exp_1d, [1.0], k, [0], E, 10.0 ** -(12 - k))
       for k in (2, 3, 4, 5)},
    # :53-68: d^4/dx^4 (x^4 + y^4) = 24 each; the order-5 derivatives vanish
    "quartic_k4_x": ("stde_higher_order.rs:53-68", _quartic, [2.0, 3.0], 4, [0], 2 * 24.0, 1e-6),
    "quartic_k4_y": ("stde_higher_order.rs:53-68", _quartic, [2.0, 3.0], 4, [1], 2 * 24.0, 1e-6),
    "quartic_k5": ("stde_higher_order.rs:53-68", _quartic, [2.0, 3.0], 5, [0, 1], 0.0, 1e-4),
    # :83-93 and :95-103: the full sample and the n/|J| scaling both give 48
    "full_sample": ("stde_higher_order.rs:83-93", _quartic, [2.0, 3.0], 4, [0, 1], 48.0, 1e-4),
    "scaling": ("stde_higher_order.rs:95-103", _quartic, [2.0, 3.0], 4, [0], 48.0, 1e-4),
    # :70-81: k = 2 is the Hessian diagonal, (2y, 6y, 0) at (1, 2, 3); summed: 16
    "cubic_mix_k2": ("stde_higher_order.rs:70-81", _cubic_mix, [1.0, 2.0, 3.0], 2, [0, 1, 2], 16.0, 1e-10),
}


def _kth_check(name, value, estimate):
    _, mk, x, k, idx, want, tol = KTH_ORDER[name]
    assert _close(value, float(OracleTape(mk()).forward(np.asarray([x]))[0][0]), 1e-12), name
    assert abs(estimate - want) <= tol * max(1.0, abs(want)), (name, estimate, want)


@pytest.mark.parametrize("name", sorted(KTH_ORDER))
def test_oracle_diagonal_kth_order(name):
    _, mk, x, k, idx, _, _ = KTH_ORDER[name]
    r = OracleTape(mk()).diagonal_kth_order_stochastic(np.asarray(x), k, idx)
    _kth_check(name, float(r[0]), float(r[1]))


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(KTH_ORDER))
def test_gpu_diagonal_kth_order(ctx, name):
    from echidna_b200.stde_gpu import diagonal_kth_order_stochastic_gpu
    _, mk, x, k, idx, _, _ = KTH_ORDER[name]
    r = diagonal_kth_order_stochastic_gpu(ctx, ctx.upload_tape_f64(mk()), x, k, idx)
    assert r.num_samples == len(idx)
    _kth_check(name, r.value, r.estimate)


@pytest.mark.gpu
def test_gpu_diagonal_kth_order_limits(ctx):
    # stde_higher_order.rs:105-118 and higher_order.rs:13-22: the reference's k
    # range, then the engine's jet limit (order 9) for 9 <= k <= 18
    from echidna_b200.gpu import GpuError
    from echidna_b200.stde_gpu import diagonal_kth_order_stochastic_gpu
    gt = ctx.upload_tape_f64(_exp_1d())
    with pytest.raises(GpuError, match="k must be >= 2"):
        diagonal_kth_order_stochastic_gpu(ctx, gt, [1.0], 1, [0])
    with pytest.raises(GpuError, match="k must be <= 18"):
        diagonal_kth_order_stochastic_gpu(ctx, gt, [1.0], 19, [0])
    with pytest.raises(GpuError, match="k must be <= 12 for f32"):
        f32_tape = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(_exp_1d()))
        diagonal_kth_order_stochastic_gpu(ctx, f32_tape, [1.0], 13, [0])
    with pytest.raises(GpuError, match="unsupported Taylor order 10"):
        diagonal_kth_order_stochastic_gpu(ctx, gt, [1.0], 9, [0])
    # the highest order the engine runs: d^8/dx^8 exp(x) = e
    r = diagonal_kth_order_stochastic_gpu(ctx, gt, [1.0], 8, [0])
    assert abs(r.estimate - E) <= 1e-3


# stde_higher_order.rs:150-181: sigma = I on x^2 + y^2 at (1, 2) gives the value
# 5 and the diffusion 1/2 tr(H) = 2; the full stochastic sample matches it.
@pytest.mark.gpu
def test_gpu_parabolic_diffusion_identity_sigma(ctx):
    from echidna_b200.stde_gpu import parabolic_diffusion_gpu, parabolic_diffusion_stochastic_gpu
    gt = ctx.upload_tape_f64(record(lambda v: v[0] * v[0] + v[1] * v[1], [1.0, 2.0])[0])
    sig = np.eye(2)
    value, diffusion = parabolic_diffusion_gpu(ctx, gt, [1.0, 2.0], sig)
    assert abs(value - 5.0) <= 1e-10 and abs(diffusion - 2.0) <= 1e-10
    r = parabolic_diffusion_stochastic_gpu(ctx, gt, [1.0, 2.0], sig, [0, 1])
    assert abs(r.estimate - diffusion) <= 1e-10


# gpu_stde.rs, section 2 (run by the reference on its CUDA backend too): f32 jets
# of one-op tapes from taylor_forward_2nd_batch along 1, uploaded with
# from_tape_f64_lossy.  check_1d (:187-226) compares c0, c1, c2 against the f64 CPU
# jet with an absolute floor of 1e-2 and relative 1e-4, 1e-4, 1e-3.
_U1 = {
    "exp": lambda t: t.exp(), "ln": lambda t: t.ln(), "exp2": lambda t: t.exp2(), "log2": lambda t: t.log2(),
    "log10": lambda t: t.log10(), "ln_1p": lambda t: t.ln_1p(), "exp_m1": lambda t: t.exp_m1(),
    "sqrt": lambda t: t.sqrt(), "cbrt": lambda t: t.cbrt(), "sin": lambda t: t.sin(), "cos": lambda t: t.cos(),
    "tan": lambda t: t.tan(), "sinh": lambda t: t.sinh(), "cosh": lambda t: t.cosh(), "tanh": lambda t: t.tanh(),
    "asin": lambda t: t.asin(), "acos": lambda t: t.acos(), "atan": lambda t: t.atan(),
    "asinh": lambda t: t.asinh(), "acosh": lambda t: t.acosh(), "atanh": lambda t: t.atanh(),
    "abs": lambda t: t.abs(), "powi3": lambda t: t.powi(3), "powf25": lambda t: t.powf(constant(2.5)),
    "powf3": lambda t: t.powf(constant(3.0)),
    "arith": lambda t: (t + _C1()) * (constant(2.0) - t) + t.recip(),
    "div": lambda t: (t * t + _C1()) / (t + _C1()),
    "signum": lambda t: t.signum(), "round": lambda t: t.round(),
}
JET_1D = {f"{op}@{x0}": (op, x0) for op, x0 in [
    # :363-480
    ("exp", 1.5), ("ln", 2.0), ("exp2", 1.0), ("log2", 3.0), ("log10", 2.0), ("ln_1p", 0.5), ("exp_m1", 0.3),
    ("sqrt", 4.0), ("cbrt", 8.0), ("sin", 1.0), ("cos", 1.0), ("tan", 0.5), ("sinh", 1.0), ("cosh", 1.0),
    ("tanh", 0.5), ("asin", 0.5), ("acos", 0.5), ("atan", 1.0), ("asinh", 1.0), ("acosh", 2.0), ("atanh", 0.5),
    ("powf25", 2.0), ("powi3", 2.0), ("powi3", -2.0), ("powf3", -2.0), ("arith", 1.5), ("div", 2.0),
    ("abs", -2.0), ("abs", 2.0),
    # :482-497, near |x| = 1
    ("asin", 0.9), ("acos", 0.9), ("atanh", 0.9), ("asin", 0.99), ("acos", 0.99), ("atanh", 0.99)]}


def _jet1(op, x0):
    return record(lambda v: _U1[op](v[0]), [x0])[0]


def _f32_jets(run, tape, x, seed):
    """(c0, c1, c2) of output 0 of one f32 point: ``run`` is "oracle" or a context."""
    xs, ss = np.asarray([x], np.float32), np.asarray([seed], np.float32)
    if run == "oracle":
        c = OracleTape(tape, dtype=np.float32).taylor(xs, ss, 3)
        return tuple(float(c[k][0]) for k in range(3))
    r = run.taylor_forward_2nd_batch(run.upload_tape(GpuTapeData.from_tape_f64_lossy(tape)), xs.ravel(),
                                     ss.ravel(), 1)
    return float(r.values[0]), float(r.c1s[0]), float(r.c2s[0])


def _check_1d(run, name):
    op, x0 = JET_1D[name]
    tape = _jet1(op, x0)
    got = _f32_jets(run, tape, [x0], [1.0])
    c = OracleTape(tape).taylor(np.asarray([[x0]]), np.asarray([[1.0]]), 3)
    want = [float(c[k][0]) for k in range(3)]
    for g, w, rel in zip(got, want, (1e-4, 1e-4, 1e-3)):
        assert abs(g - w) < max(1e-2, abs(w) * rel), (name, got, want)


@pytest.mark.parametrize("name", sorted(JET_1D))
def test_oracle_f32_jets_match_f64(name):
    _check_1d("oracle", name)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(JET_1D))
def test_gpu_f32_jets_match_f64(ctx, name):
    _check_1d(ctx, name)


_NEXT_BELOW_HALF = float(np.frombuffer(np.uint32(0x3EFFFFFF).tobytes(), np.float32)[0])
# name: (source, op or binary fn, inputs, seed, expected (c0, c1, c2) with None = any;
# "nan", "+inf", "-inf" classes, or (value, rel) for a relative check of c0 against
# the f64 truth at the f32-rounded input)
JET_EDGE = {
    # :498-535 (check_primal_rel, tolerance 1e-3) and the overflow limit
    "expm1@1e-6": (":498-500", "exp_m1", [1e-6], [1.0], ("rel", math.expm1), None, None),
    "expm1@1e-7": (":498-500", "exp_m1", [1e-7], [1.0], ("rel", math.expm1), None, None),
    "ln1p@1e-6": (":498-500", "ln_1p", [1e-6], [1.0], ("rel", math.log1p), None, None),
    "ln1p@1e-7": (":498-500", "ln_1p", [1e-7], [1.0], ("rel", math.log1p), None, None),
    "expm1@87": (":531", "exp_m1", [87.0], [1.0], ("rel", math.expm1), None, None),
    "expm1@90": (":512-526", "exp_m1", [90.0], [1.0], "+inf", None, None),
    # :537-564: all-NaN jets strictly outside the real domain
    **{f"{op}@{x}_nan": (":537-564", op, [x], [1.0], "nan", "nan", "nan") for op, x in [
        ("ln", -2.0), ("log2", -2.0), ("log10", -2.0), ("ln_1p", -2.0), ("acosh", -2.0), ("atanh", 1.5),
        ("asin", 1.5), ("acos", 1.5), ("acosh", 0.5)]},
    # :566-600: the domain boundary keeps its branch-point value
    "acosh@1": (":573-577", "acosh", [1.0], [1.0], 0.0, None, None),
    "atanh@1": (":578-582", "atanh", [1.0], [1.0], "+inf", None, None),
    "atanh@-1": (":585-589", "atanh", [-1.0], [1.0], "-inf", None, None),
    "ln1p@-1": (":590-594", "ln_1p", [-1.0], [1.0], "-inf", None, None),
    "ln@0": (":595-599", "ln", [0.0], [1.0], "-inf", None, None),
    # :603-627: max / min keep the finite operand against NaN
    "max_nan": (":611-618", lambda v: v[0].max(v[1]), [1.0, NAN], [1.0, 0.0], 1.0, None, None),
    "min_nan": (":619-626", lambda v: v[0].min(v[1]), [1.0, NAN], [1.0, 0.0], 1.0, None, None),
    # :629-641: rem by a zero-leading divisor is an all-NaN jet
    "rem_zero": (":637-641", lambda v: v[0] % v[1], [3.0, 0.0], [1.0, 0.0], "nan", "nan", "nan"),
    # :643-683: signum(-0) = -1 and round ties away from zero
    "signum@-0": (":657-659", "signum", [-0.0], [1.0], -1.0, None, None),
    "round@2.5": (":662-663", "round", [2.5], [1.0], 3.0, None, None),
    "round@-2.5": (":664-665", "round", [-2.5], [1.0], -3.0, None, None),
    "round@0.5": (":666-670", "round", [0.5], [1.0], 1.0, None, None),
    "round@8388609": (":673-678", "round", [8388609.0], [1.0], 8388609.0, None, None),
    "round@below_half": (":679-682", "round", [_NEXT_BELOW_HALF], [1.0], 0.0, None, None),
    # :687-715: sqrt at 0 has a uniform +Inf jet
    "sqrt@0": (":687-715", "sqrt", [0.0], [1.0], 0.0, "+inf", "+inf"),
}


def _edge_tape(fn, x):
    f = (lambda v: _U1[fn](v[0])) if isinstance(fn, str) else fn
    return record(f, list(x))[0]


def _check_class(got, want, x, label):
    if want is None:
        return
    if isinstance(want, tuple):
        truth = want[1](float(np.float32(x)))
        assert abs(got - truth) / max(abs(truth), 2.2e-308) < 1e-3, (label, got, truth)
    elif want == "nan":
        assert math.isnan(got), (label, got)
    elif want in ("+inf", "-inf"):
        assert math.isinf(got) and (got > 0) == (want == "+inf"), (label, got)
    else:
        assert got == want, (label, got, want)


def _jet_edge(run, name):
    _, fn, x, seed, *want = JET_EDGE[name]
    got = _f32_jets(run, _edge_tape(fn, x), x, seed)
    for k in range(3):
        _check_class(got[k], want[k], x[0], (name, k))


@pytest.mark.filterwarnings("ignore:overflow encountered in cast")  # the recorded e^90 in f32
@pytest.mark.parametrize("name", sorted(JET_EDGE))
def test_oracle_f32_jet_edge_cases(name):
    _jet_edge("oracle", name)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(JET_EDGE))
def test_gpu_f32_jet_edge_cases(ctx, name):
    _jet_edge(ctx, name)


# gpu_stde.rs:864-913: x^2 + y^2 at (3, 4) in f32.  The four Rademacher
# directions give the Laplacian 4 exactly; the Hessian diagonal is (2, 2), value 25.
@pytest.mark.gpu
def test_gpu_polynomial_exact_laplacian_and_diagonal(ctx):
    from echidna_b200.stde_gpu import hessian_diagonal_gpu, laplacian_gpu
    gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(record(lambda v: v[0] * v[0] + v[1] * v[1],
                                                                [3.0, 4.0])[0]))
    dirs = [[1.0, 1.0], [1.0, -1.0], [-1.0, 1.0], [-1.0, -1.0]]
    assert abs(laplacian_gpu(ctx, gt, [3.0, 4.0], dirs).estimate - 4.0) < 1e-3
    val, diag = hessian_diagonal_gpu(ctx, gt, [3.0, 4.0])
    assert abs(val - 25.0) < 1e-3 and abs(diag[0] - 2.0) < 1e-3 and abs(diag[1] - 2.0) < 1e-3


# gpu_stde.rs:1353-2093, the cases the reference runs with its CUDA backend: f32
# jets from taylor_forward_kth_batch (tape recorded at `rec`, evaluated at `x`).
# Expectations per coefficient: a number (exact), ("near", v, tol), "nan",
# "+inf", "inf" (either sign), or "cpu": check_hypot_jet's finiteness plus the
# check_1d tolerances against the f64 CPU jet.
_HYP = lambda v: v[0].hypot(v[1])  # noqa: E731
_CPU3 = ("cpu", "cpu", "cpu")
CUDA_JETS = {
    # :1532-1558 (check_hypot_jet)
    "hypot(3,4)_dx": (":1534-1541", _HYP, [3.0, 4.0], [3.0, 4.0], [1.0, 0.0], _CPU3),
    "hypot(3,4)_dy": (":1534-1541", _HYP, [3.0, 4.0], [3.0, 4.0], [0.0, 1.0], _CPU3),
    "hypot(1e20,1e19)_dx": (":1545-1551", _HYP, [1e20, 1e19], [1e20, 1e19], [1.0, 0.0], _CPU3),
    "hypot(0,0)_dx": (":1555-1558", _HYP, [0.0, 0.0], [0.0, 0.0], [1.0, 0.0], _CPU3),
    # :1504-1515: a NaN operand makes the whole jet NaN (tape recorded at (1, 1))
    "hypot(nan,0)": (":1506-1514", _HYP, [1.0, 1.0], [NAN, 0.0], [1.0, 0.0], ("nan", "nan", "nan")),
    "hypot(0,nan)": (":1506-1514", _HYP, [1.0, 1.0], [0.0, NAN], [1.0, 0.0], ("nan", "nan", "nan")),
    "hypot(nan,1)": (":1506-1514", _HYP, [1.0, 1.0], [NAN, 1.0], [1.0, 0.0], ("nan", "nan", "nan")),
    # :1731-1757 and :1784-1801
    "hypot(inf,1)": (":1733-1757", _HYP, [INF, 1.0], [INF, 1.0], [1.0, 0.0], ("inf", "nan", "nan")),
    "hypot(1,inf)": (":1733-1757", _HYP, [1.0, INF], [1.0, INF], [1.0, 0.0], ("inf", "nan", "nan")),
    "hypot_identically_zero": (":1786-1801", _HYP, [0.0, 0.0], [0.0, 0.0], [0.0, 0.0], (0.0, 0.0, 0.0)),
    # :1853-1877: fract is x - trunc(x)
    "fract(-2.3)": (":1853-1877", lambda v: v[0].fract(), [-2.3], [-2.3], [1.0],
                    (("near", -0.3, 1e-5), ("near", 1.0, 1e-6), None)),
    # :1880-1901: hypot(t^2, 0) = t^2, a depth-two shift
    "hypot_depth_two": (":1880-1901", lambda v: (v[0] * v[0]).hypot(v[1]), [0.0, 0.0], [0.0, 0.0], [1.0, 0.0],
                        tuple(("near", e, 1e-6) for e in (0.0, 0.0, 1.0, 0.0, 0.0))),
    # :1904-1922: x^10 seeded at 0 has valuation 10 > K - 1
    "powi10_at_0": (":1904-1922", lambda v: v[0].powi(10), [0.0], [0.0], [1.0], (0.0,) * 5),
    # :1987-2011: x^2.5 at 0 (recorded at 1): zero below the branch order, +Inf above
    "powf2.5_at_0": (":1987-2011", lambda v: v[0].powf(constant(2.5)), [1.0], [0.0], [1.0],
                     (0.0, 0.0, 0.0, "+inf", "+inf")),
}


def _f32_kth(run, tape, x, seed, K):
    xs, ss = np.asarray([x], np.float32), np.asarray([seed], np.float32)
    if run == "oracle":
        c = OracleTape(tape, dtype=np.float32).taylor(xs, ss, K)
        return [float(c[k][0]) for k in range(K)]
    r = run.taylor_forward_kth_batch(run.upload_tape(GpuTapeData.from_tape_f64_lossy(tape)), xs.ravel(),
                                     ss.ravel(), 1, K)
    return [float(r.coefficients[k][0]) for k in range(K)]


def _cuda_jet(run, name):
    _, fn, rec, x, seed, want = CUDA_JETS[name]
    tape = record(fn, list(rec))[0]
    got = _f32_kth(run, tape, x, seed, len(want))
    cpu = None
    if "cpu" in want:
        c = OracleTape(tape).taylor(np.asarray([x]), np.asarray([seed]), len(want))
        cpu = [float(c[k][0]) for k in range(len(want))]
    for k, (g, w) in enumerate(zip(got, want)):
        label = (name, k, got)
        if w == "cpu":
            rel = 1e-3 if k == 2 else 1e-4
            assert math.isfinite(g) and abs(g - cpu[k]) < max(1e-2, abs(cpu[k]) * rel), (label, cpu)
        elif w == "inf":
            assert math.isinf(g), label
        elif isinstance(w, tuple):
            assert abs(g - w[1]) < w[2], label
        elif w is not None:
            _check_class(g, w, x[0], label)


@pytest.mark.parametrize("name", sorted(CUDA_JETS))
def test_oracle_f32_cuda_backend_jets(name):
    _cuda_jet("oracle", name)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CUDA_JETS))
def test_gpu_f32_cuda_backend_jets(ctx, name):
    _cuda_jet(ctx, name)


def _sqrt_hypot_tape():
    return record(lambda v: v[0].hypot(v[1]).sqrt(), [3.0, 4.0])[0]


# gpu_stde.rs:2038-2090: sqrt'(0) = Inf reaches hypot's origin node, whose partials
# are exactly 0: gradient and HVP are 0 there; away from it the replay holds.
_ZM_X = 0.6 * 0.5 / math.sqrt(5.0)


def test_oracle_f32_zero_multiplier_absorbs_inf_adjoint():
    o = OracleTape(_sqrt_hypot_tape(), dtype=np.float32)
    _, g = o.gradient(np.asarray([[0.0, 0.0]], np.float32))
    assert list(g[0]) == [0.0, 0.0]
    _, g = o.gradient(np.asarray([[3.0, 4.0]], np.float32))
    assert abs(g[0][0] - _ZM_X) < 1e-5
    hg, hv = o.hvp(np.asarray([0.0, 0.0], np.float32), np.asarray([[1.0, 0.0]], np.float32))
    assert list(hg[0]) == [0.0, 0.0] and list(hv[0]) == [0.0, 0.0]


@pytest.mark.gpu
def test_gpu_f32_zero_multiplier_absorbs_inf_adjoint(ctx):
    gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(_sqrt_hypot_tape()))
    _, g = ctx.gradient_batch(gt, np.asarray([0.0, 0.0], np.float32), 1)
    assert list(np.asarray(g, np.float64)) == [0.0, 0.0]
    _, g = ctx.gradient_batch(gt, np.asarray([3.0, 4.0], np.float32), 1)
    assert abs(float(g[0]) - _ZM_X) < 1e-5
    hg, hv = ctx.hvp_batch(gt, np.asarray([0.0, 0.0], np.float32), np.asarray([1.0, 0.0], np.float32), 1)
    assert list(np.asarray(hg, np.float64)) == [0.0, 0.0] and list(np.asarray(hv, np.float64)) == [0.0, 0.0]


# stde_higher_order.rs:39-81 and :185-263 on the exact vector form
# (diagonal_kth_order and its const-order twin): (value, [d^k f / dx_j^k]).
KTH_DIAG = {
    **{f"exp_k{k}": (_exp_1d, [1.0], k, E, [E], 10.0 ** -(12 - k)) for k in (2, 3, 4, 5)},
    "quartic_k4": (_quartic, [2.0, 3.0], 4, 97.0, [24.0, 24.0], 1e-6),
    "quartic_k5": (_quartic, [2.0, 3.0], 5, 97.0, [0.0, 0.0], 1e-4),
    "cubic_mix_k2": (_cubic_mix, [1.0, 2.0, 3.0], 2, 10.0, [4.0, 12.0, 0.0], 1e-10),
}


@pytest.mark.parametrize("name", sorted(KTH_DIAG))
def test_oracle_diagonal_kth_order_vector(name):
    # the oracle's single-index estimate is n * d^k f / dx_j^k
    mk, x, k, _, want, tol = KTH_DIAG[name]
    o = OracleTape(mk())
    got = [float(o.diagonal_kth_order_stochastic(np.asarray(x), k, [j])[1]) / len(x) for j in range(len(x))]
    assert all(abs(g - w) <= tol * max(1.0, abs(w)) for g, w in zip(got, want)), (name, got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(KTH_DIAG))
def test_gpu_diagonal_kth_order_vector(ctx, name):
    from echidna_b200.stde_gpu import diagonal_kth_order_gpu
    mk, x, k, value, want, tol = KTH_DIAG[name]
    v, d = diagonal_kth_order_gpu(ctx, ctx.upload_tape_f64(mk()), x, k)
    assert abs(v - value) <= 1e-10 * max(1.0, abs(value))
    assert all(abs(g - w) <= tol * max(1.0, abs(w)) for g, w in zip(d, want)), (name, list(d), want)


@pytest.mark.gpu
def test_gpu_diagonal_kth_order_vector_edges(ctx):
    from echidna_b200.gpu import GpuError
    from echidna_b200.stde_gpu import diagonal_kth_order_gpu
    # higher_order.rs:59-62: a zero-input tape returns its primal and no diagonal
    gt = ctx.upload_tape_f64(record(lambda v: constant(3.0) * constant(2.0), [])[0])
    v, d = diagonal_kth_order_gpu(ctx, gt, [], 3)
    assert v == 6.0 and d.size == 0
    # the highest order the engine runs, and f32
    v, d = diagonal_kth_order_gpu(ctx, ctx.upload_tape_f64(_exp_1d()), [1.0], 8)
    assert abs(d[0] - E) <= 1e-3
    v, d = diagonal_kth_order_gpu(ctx, ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(_exp_1d())), [1.0], 2)
    assert abs(d[0] - E) <= 1e-5 * E
    with pytest.raises(GpuError, match="k must be >= 2"):
        diagonal_kth_order_gpu(ctx, ctx.upload_tape_f64(_exp_1d()), [1.0], 1)
    from echidna_b200 import record_multi
    two = record_multi(lambda v: [v[0] * v[1], v[0] + v[1]], [1.0, 2.0])[0]
    with pytest.raises(GpuError, match="scalar-output"):
        diagonal_kth_order_gpu(ctx, ctx.upload_tape_f64(two), [1.0, 2.0], 2)


# stde_pipeline.rs:37-172: estimate / estimate_weighted with both estimators.
_RADEMACHER4 = [[1.0, 1.0], [1.0, -1.0], [-1.0, 1.0], [-1.0, -1.0]]


def _sum_sq(x0):
    return record(lambda v: v[0] * v[0] + v[1] * v[1], x0)[0]


@pytest.mark.gpu
def test_gpu_estimate_pipeline(ctx):
    from echidna_b200.stde_gpu import GRADIENT_SQUARED_NORM, LAPLACIAN, estimate_gpu, laplacian_gpu
    # :37-54: the Laplacian estimator equals laplacian() (value 5, estimate 4, 4 samples)
    gt = ctx.upload_tape_f64(_sum_sq([1.0, 2.0]))
    r = estimate_gpu(ctx, gt, [1.0, 2.0], _RADEMACHER4, LAPLACIAN)
    assert abs(r.value - 5.0) <= 1e-10 and abs(r.estimate - 4.0) <= 1e-10 and r.num_samples == 4
    f32 = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(_sum_sq([1.0, 2.0])))
    lap = laplacian_gpu(ctx, f32, [1.0, 2.0], _RADEMACHER4)
    r32 = estimate_gpu(ctx, f32, [1.0, 2.0], _RADEMACHER4, LAPLACIAN)
    assert r32.estimate == lap.estimate and r32.value == lap.value
    # :56-76: GradientSquaredNorm at (3, 4): value 25, E[(g.v)^2] = |g|^2 = 100
    gt = ctx.upload_tape_f64(_sum_sq([3.0, 4.0]))
    r = estimate_gpu(ctx, gt, [3.0, 4.0], _RADEMACHER4, GRADIENT_SQUARED_NORM)
    assert abs(r.value - 25.0) <= 1e-10 and abs(r.estimate - 100.0) <= 1e-10
    # :78-101: unit weights reproduce the unweighted estimate
    cm = ctx.upload_tape_f64(_cubic_mix())
    dirs = [[1.0, 1.0, 1.0], [1.0, -1.0, 1.0], [-1.0, 1.0, -1.0], [1.0, 1.0, -1.0]]
    a = estimate_gpu(ctx, cm, [1.0, 2.0, 3.0], dirs)
    b = estimate_gpu(ctx, cm, [1.0, 2.0, 3.0], dirs, weights=[1.0] * 4)
    assert abs(a.estimate - b.estimate) <= 1e-10 and a.num_samples == b.num_samples
    # :103-124: weights (3, 1) on x^2 + y^2: both samples 4, so 4
    gt = ctx.upload_tape_f64(_sum_sq([1.0, 2.0]))
    r = estimate_gpu(ctx, gt, [1.0, 2.0], _RADEMACHER4[:2], weights=[3.0, 1.0])
    assert abs(r.estimate - 4.0) <= 1e-10 and r.num_samples == 2
    # :130-168: x^2 + 3 y^2, samples 2 and 6 with weights (3, 1): mean 3, SE over n_eff = 1.6
    t = record(lambda v: v[0] * v[0] + (v[1] * v[1]) * constant(3.0), [1.0, 2.0])[0]
    r = estimate_gpu(ctx, ctx.upload_tape_f64(t), [1.0, 2.0], [[1.0, 0.0], [0.0, 1.0]], weights=[3.0, 1.0])
    assert abs(r.estimate - 3.0) <= 1e-10
    assert abs(r.standard_error - math.sqrt(r.sample_variance / 1.6)) <= 1e-10
    assert abs(r.standard_error - math.sqrt(r.sample_variance / 2.0)) > 1e-6


@pytest.mark.gpu
def test_gpu_estimate_weighted_matches_oracle_and_nonfinite(ctx):
    from echidna_b200.gpu import GpuError
    from echidna_b200.stde_gpu import estimate_gpu
    from echidna_b200 import configs
    # a random tape, random directions and weights with zeros: the oracle's West update
    tape = configs.random_dag(6, 300, seed=77)
    rng = np.random.default_rng(77)
    x = rng.uniform(-0.7, 0.7, size=6)
    dirs = rng.choice([-1.0, 1.0], size=(40, 6))
    w = rng.uniform(0.0, 2.0, size=40)
    w[::7] = 0.0
    r = estimate_gpu(ctx, ctx.upload_tape_f64(tape), x, dirs, weights=w)
    o = OracleTape(tape).estimate_weighted(x, dirs, w)
    for got, want in zip((r.value, r.estimate, r.sample_variance, r.standard_error), o[:4]):
        assert abs(got - float(want)) <= 1e-10 * max(1.0, abs(float(want)))
    assert r.num_samples == int(o[4])
    # stde_nonfinite_samples.rs:58-111 through the GPU jets
    gt = ctx.upload_tape_f64(_exp_prod_tape())
    r = estimate_gpu(ctx, gt, [1.0, 700.0], [LIVE, DEAD], weights=[1.0, 1.0])
    assert r.num_samples == 1 and r.estimate == 0.0
    r = estimate_gpu(ctx, gt, [1.0, 700.0], [LIVE], weights=[1.0])
    assert r.num_samples == 0 and math.isnan(r.estimate)
    with pytest.raises(GpuError, match="weights must be non-negative"):
        estimate_gpu(ctx, gt, [1.0, 700.0], [LIVE], weights=[-1.0])
    with pytest.raises(GpuError, match="directions must not be empty"):
        estimate_gpu(ctx, gt, [1.0, 700.0], np.zeros((0, 2)))


# stde_core.rs:61-297 on the oracle (the GPU forms are checked against it in
# test_gpu_taylor_stde.py and above): laplacian, hessian_diagonal and the
# directional derivatives of the stde module's known Hessians.
_R3 = [[a, b, c] for a in (1.0, -1.0) for b in (1.0, -1.0) for c in (1.0, -1.0)]
STDE_CORE = {
    # name: (tape maker, x, Rademacher dirs or None, value, laplacian or None, diagonal or None)
    "sum_of_squares": (lambda: _sum_sq([1.0, 2.0]), [1.0, 2.0], _RADEMACHER4[:2], 5.0, 4.0, [2.0, 2.0]),
    "product": (lambda: record(lambda v: v[0] * v[1], [3.0, 4.0])[0], [3.0, 4.0], _RADEMACHER4[:2], 12.0, 0.0,
                [0.0, 0.0]),
    "cubic_mix": (_cubic_mix, [1.0, 2.0, 3.0], _R3, 10.0, 16.0, [4.0, 12.0, 0.0]),
    "cube_1d": (lambda: record(lambda v: v[0] * v[0] * v[0], [2.0])[0], [2.0], None, 8.0, None, [12.0]),
    "linear": (lambda: record(lambda v: v[0] + v[1], [1.0, 2.0])[0], [1.0, 2.0], _RADEMACHER4[:2], 3.0, 0.0,
               [0.0, 0.0]),
}


@pytest.mark.parametrize("name", sorted(STDE_CORE))
def test_oracle_stde_core_known_hessians(name):
    mk, x, dirs, value, lap, diag = STDE_CORE[name]
    o = OracleTape(mk())
    if dirs is not None:
        v, got = o.laplacian(np.asarray(x), np.asarray(dirs))
        assert abs(v - value) <= 1e-10 and abs(got - lap) <= 1e-10, (name, v, got)
    v, d = o.hessian_diagonal(np.asarray(x))
    assert abs(v - value) <= 1e-10 and np.allclose(d, diag, rtol=0, atol=1e-10), (name, v, d)
    # :159-214: the diagonal and the trace agree with the full Hessian
    _, _, H = o.hessian(np.asarray(x))
    assert np.allclose(np.diag(H), d, rtol=0, atol=1e-10)


def test_oracle_stde_core_directional_derivatives():
    # :285-298: along e0 on x^2 + y^2 at (1, 2), c1 = 2 and c2 = e0^T H e0 / 2 = 1;
    # :221-237: along each e_j, c1 is the gradient entry
    o = OracleTape(_sum_sq([1.0, 2.0]))
    c = o.taylor(np.asarray([[1.0, 2.0]]), np.asarray([[1.0, 0.0]]), 3)
    assert abs(c[1][0] - 2.0) <= 1e-10 and abs(c[2][0] - 1.0) <= 1e-10
    q = OracleTape(_cubic_mix())
    _, g = q.gradient(np.asarray([[1.0, 2.0, 3.0]]))
    for j in range(3):
        e = np.zeros((1, 3))
        e[0, j] = 1.0
        cj = q.taylor(np.asarray([[1.0, 2.0, 3.0]]), e, 2)
        assert abs(cj[1][0] - g[0][j]) <= 1e-10
    assert np.allclose(g[0], [4.0, 13.0, 0.0], rtol=0, atol=1e-10)


# stde_stats.rs:95-343 on the oracle: the Hessian diagonal of exp(x) + sin(y), the
# Welford statistics of laplacian_with_stats and the control-variate estimate.
_CM_DIRS = [[1.0, 1.0, 1.0], [1.0, -1.0, 1.0], [-1.0, 1.0, -1.0], [1.0, 1.0, -1.0]]


def test_oracle_stde_stats_known_answers():
    # :95-103
    t = record(lambda v: v[0].exp() + v[1].sin(), [1.0, 2.0])[0]
    _, d = OracleTape(t).hessian_diagonal(np.asarray([1.0, 2.0]))
    assert abs(d[0] - math.exp(1.0)) <= 1e-10 and abs(d[1] + math.sin(2.0)) <= 1e-10
    cm = OracleTape(_cubic_mix())
    x3 = np.asarray([[1.0, 2.0, 3.0]])
    # :146-163: off-diagonal Hessian entries give a positive variance
    r = cm.laplacian_stats_batch(x3, np.asarray(_CM_DIRS))[0]
    assert r[2] > 0.0 and r[3] > 0.0
    # :178-189: SE = sqrt(var / n)
    r = cm.laplacian_stats_batch(x3, np.asarray(_CM_DIRS[:3]))[0]
    assert abs(r[3] - math.sqrt(r[2] / r[4])) <= 1e-14
    ss = OracleTape(_sum_sq([1.0, 2.0]))
    x2 = np.asarray([[1.0, 2.0]])
    # :166-176: one sample has zero variance and SE
    r = ss.laplacian_stats_batch(x2, np.asarray([[1.0, 1.0]]))[0]
    assert int(r[4]) == 1 and r[2] == 0.0 and r[3] == 0.0
    # :192-205: a diagonal Hessian gives 4 with zero variance; :128-143 it equals laplacian()
    r = ss.laplacian_stats_batch(x2, np.asarray(_RADEMACHER4))[0]
    v, lap = ss.laplacian(np.asarray([1.0, 2.0]), np.asarray(_RADEMACHER4))
    assert abs(r[1] - 4.0) <= 1e-10 and abs(r[2]) <= 1e-10 and r[1] == lap and r[0] == v and int(r[4]) == 4
    # :212-231: the control variate keeps the exact 16 over all 8 Rademacher vectors
    _, diag = cm.hessian_diagonal(np.asarray([1.0, 2.0, 3.0]))
    r = cm.laplacian_with_control(np.asarray([1.0, 2.0, 3.0]), np.asarray(_R3), diag)
    assert abs(r[1] - 16.0) <= 1e-10
    # :333-344: a linear function: value 3, estimate 0, variance 0
    lin = OracleTape(record(lambda v: v[0] + v[1], [1.0, 2.0])[0])
    r = lin.laplacian_stats_batch(x2, np.asarray(_RADEMACHER4))[0]
    assert abs(r[0] - 3.0) <= 1e-10 and abs(r[1]) <= 1e-10 and abs(r[2]) <= 1e-10


# bytecode_tape.rs:34-72 on the oracle: gradients through shared subexpressions.
def _chain8(x):
    a = x * x
    b = a * a
    return b * b


BYTECODE_GRADS = {
    "x_squared": (lambda v: v[0] * v[0], [3.0], [6.0]),
    "x_times_y": (lambda v: v[0] * v[1], [3.0, 4.0], [4.0, 3.0]),
    "diamond": (lambda v: v[0] * v[0] + v[0] * v[0] * v[0], [2.0], [16.0]),
    "fan_out": (lambda v: v[0] + v[0] + v[0], [5.0], [3.0]),
    "chain_depth": (lambda v: _chain8(v[0]), [2.0], [8.0 * 2.0 ** 7]),
}


@pytest.mark.parametrize("name", sorted(BYTECODE_GRADS))
def test_oracle_bytecode_tape_gradients(name):
    fn, x, want = BYTECODE_GRADS[name]
    _, g = OracleTape(record(fn, x)[0]).gradient(np.asarray([x]))
    assert all(abs(a - b) <= 1e-12 * abs(b) for a, b in zip(g[0], want)), (name, g[0], want)
