"""Host-only checks of the C ABI: exports, validation messages, argument checks.

No GPU is needed: the library loads without a device, validation is host code,
and context creation must fail cleanly with NO_DEVICE on a machine without one.
"""
import ctypes
import os
import re

import numpy as np
import pytest

from echidna_b200 import _lib, record
from echidna_b200.gpu import GpuError, GpuTapeData
from echidna_b200.tape import UNUSED, BytecodeTape, OpCode, TapeValidationError

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "echidna_b200.h")


def _declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"ECH_API\s+[\w\s\*]+?\b(ech_\w+)\s*\(", text)))


def test_header_declares_the_abi():
    names = _declared_symbols()
    assert len(names) >= 40
    for must in ("ech_ctx_create", "ech_upload_tape_f32", "ech_upload_tape_f64", "ech_forward_batch_f64",
                 "ech_gradient_batch_f64", "ech_hvp_batch_f64", "ech_taylor_forward_kth_batch_f32",
                 "ech_laplacian_gpu_f32", "ech_hessian_diagonal_gpu_f32", "ech_laplacian_with_control_gpu_f32"):
        assert must in names


def test_library_exports_every_declared_symbol(engine_lib):
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in _declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_ctypes_signatures_cover_the_header(engine_lib):
    declared = set(_declared_symbols())
    bound = set(_lib._SIGS)
    assert bound <= declared, bound - declared


def test_version_string(engine_lib):
    assert b"sm_100a" in engine_lib.ech_version()


def test_ctx_create_without_device_is_no_device(engine_lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    assert engine_lib.ech_ctx_create(0, ctypes.byref(h)) == _lib.NO_DEVICE
    assert h.value is None
    assert "no suitable GPU device" in _lib.last_error()


# ── GpuTapeData::validate (src/gpu/mod.rs:397-564), cases of tests/gpu_upload_validation.rs:12-76 ──

def _data(**changes):
    d = dict(opcodes=np.array([0, 1, 4], np.uint32), arg0=np.array([UNUSED, UNUSED, 0], np.uint32),
             arg1=np.array([UNUSED, UNUSED, 1], np.uint32), constants=np.array([0.0, 3.0, 0.0], np.float32),
             num_ops=3, num_inputs=1, num_variables=3, output_index=2, output_indices=np.array([2], np.uint32))
    d.update(changes)
    return GpuTapeData(**d)


def test_gpu_tape_data_valid(engine_lib):
    _data().validate()


@pytest.mark.parametrize("mutate, text", [
    (lambda d: d.arg0.__setitem__(2, 9999), "arg0[2] (9999) must reference an earlier slot"),
    (lambda d: (d.opcodes.__setitem__(2, 24), d.arg1.__setitem__(2, 9999)),
     "arg1[2] (9999) should be the UNUSED sentinel for unary opcode 24"),
    (lambda d: (setattr(d, "output_index", UNUSED), setattr(d, "output_indices", np.zeros(0, np.uint32))),
     "output_index (4294967295) >= num_variables (3)"),
    (lambda d: setattr(d, "output_indices", np.array([3], np.uint32)), "output_indices[0] (3) >= num_variables (3)"),
    (lambda d: d.opcodes.__setitem__(2, 43), "opcodes[2] (43) is not a GPU-executable opcode"),
    (lambda d: setattr(d, "num_ops", 4), "opcodes.len() (3) != num_ops (4)"),
])
def test_gpu_tape_data_rejects(engine_lib, mutate, text):
    d = _data()
    mutate(d)
    with pytest.raises(GpuError) as e:
        d.validate()
    assert "invalid GpuTapeData" in str(e.value)
    assert text in str(e.value)


# ── BytecodeTape::validate (src/bytecode_tape/mod.rs:575-705) ──

def _tape(op, a0, a1, vals, ni, out):
    t = BytecodeTape()
    t.opcodes = list(op)
    t.arg0 = list(a0)
    t.arg1 = list(a1)
    t.values = list(vals)
    t.num_inputs = ni
    t.output_index = out
    t.output_indices = []
    return t


def test_bytecode_validate_accepts_recorded_tapes():
    tape, _ = record(lambda v: (v[0] * v[1]).sin() + v[0].powi(3), [0.5, 1.5])
    tape.validate()


@pytest.mark.parametrize("args, text", [
    (([0, 0, 4], [UNUSED, UNUSED, 0], [UNUSED, UNUSED, 1], [1.0, 2.0, 2.0], 1, 2),
     "opcodes[1] is Input, but only the first 1 entries may be inputs"),
    (([0, 1, 4], [UNUSED, UNUSED, 2], [UNUSED, UNUSED, 1], [1.0, 2.0, 2.0], 1, 2),
     "arg_indices[2][0] (2) must reference an earlier slot"),
    (([0, 1, 24], [UNUSED, UNUSED, 0], [UNUSED, UNUSED, 1], [1.0, 2.0, 0.8], 1, 2),
     "arg_indices[2][1] (1) should be UNUSED for unary op Sin"),
    (([0, 1, 4], [UNUSED, UNUSED, 0], [UNUSED, UNUSED, 1], [1.0, 2.0, 2.0], 1, 3),
     "output_index (3) >= tape length (3)"),
    (([0, 1, 4], [UNUSED, 5, 0], [UNUSED, UNUSED, 1], [1.0, 2.0, 2.0], 1, 2),
     "must be [UNUSED, UNUSED] for a Const entry"),
    (([0, 1, 4], [UNUSED, UNUSED, 0], [UNUSED, UNUSED, 1], [1.0, 2.0, 2.0], 4, 2),
     "num_inputs (4) > tape length (3)"),
])
def test_bytecode_validate_rejects(args, text):
    t = _tape(*args)
    with pytest.raises(TapeValidationError) as e:
        t.validate()
    assert text in str(e.value)


def test_powi_exponent_is_exempt_from_the_earlier_slot_rule():
    # opcode.rs:491-522: Powi stores its i32 exponent in arg1
    tape, _ = record(lambda v: v[0].powi(-7), [1.3])
    op, a0, a1, _ = tape.arrays()
    k = int(np.flatnonzero(op == OpCode.Powi)[0])
    assert a1[k] > k
    tape.validate()


def test_upload_without_context_is_invalid_arg(engine_lib):
    op = np.array([0, 1, 4], np.uint32)
    a = np.array([UNUSED, UNUSED, 0], np.uint32)
    b = np.array([UNUSED, UNUSED, 1], np.uint32)
    v = np.array([0.0, 3.0, 0.0])
    outs = np.array([2], np.uint32)
    h = ctypes.c_void_p()
    st = engine_lib.ech_upload_tape_f64(None, _lib.ptr(op), _lib.ptr(a), _lib.ptr(b), _lib.ptr(v), 3, 1, 2,
                                        _lib.ptr(outs), 1, 0, ctypes.byref(h))
    assert st == _lib.INVALID_ARG
