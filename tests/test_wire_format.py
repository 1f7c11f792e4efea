"""Tape wire format (src/bytecode_tape/serde_support.rs): JSON round trips that
keep derivatives, and clean errors for corrupt payloads (tests/serde.rs)."""
import json

import numpy as np
import pytest

from echidna_b200 import configs, record, record_multi
from echidna_b200.tape import BytecodeTape, TapeValidationError
from oracle.oracle import OracleTape


def _rosen(v):
    s = v[0] - v[0]
    for i in range(len(v) - 1):
        s = s + (1.0 - v[i]) * (1.0 - v[i]) + 100.0 * (v[i + 1] - v[i] * v[i]) * (v[i + 1] - v[i] * v[i])
    return s


def test_roundtrip_keeps_gradient_and_hessian():
    # tests/serde.rs:14-66
    tape, _ = record(_rosen, [1.5, 2.5])
    back = BytecodeTape.from_json(tape.to_json())
    assert back.opcodes == tape.opcodes and back.arg0 == tape.arg0 and back.arg1 == tape.arg1
    X = np.array([[1.5, 2.5], [0.3, -0.7]])
    a, b = OracleTape(tape), OracleTape(back)
    for x in X:
        assert np.array_equal(a.gradient(x[None])[1], b.gradient(x[None])[1])
        assert np.array_equal(a.hessian(x)[2], b.hessian(x)[2])


def test_payload_fields_and_names():
    # tests/serde.rs:222-228: num_variables is carried; opcodes are variant names
    tape, _ = record(lambda v: (v[0] * v[0]).sin() + v[1], [0.5, 1.0])
    v = json.loads(tape.to_json())
    assert v["num_variables"] == len(v["opcodes"])
    assert "Sin" in v["opcodes"] and v["opcodes"][0] == "Input"
    assert set(v) == {"opcodes", "arg_indices", "values", "num_inputs", "num_variables", "output_index",
                      "output_indices", "custom_second_args"}


def test_roundtrip_f32_and_multi_output():
    # tests/serde.rs:120-153
    tape, _ = record(_rosen, [1.5, 2.5], dtype=np.float32)
    back = BytecodeTape.from_json(tape.to_json(), dtype=np.float32)
    assert np.array_equal(np.asarray(back.values, np.float32), np.asarray(tape.values, np.float32))
    mt, _ = record_multi(lambda v: [v[0] * v[1], v[1].sin(), v[0] + v[2]], [1.0, 2.0, 3.0])
    back = BytecodeTape.from_json(mt.to_json())
    assert back.all_output_indices() == mt.all_output_indices()
    x = np.array([[0.2, -0.4, 1.1]])
    assert np.array_equal(OracleTape(mt).jvp(x, np.ones_like(x))[1], OracleTape(back).jvp(x, np.ones_like(x))[1])


def test_large_config_tape_roundtrips():
    tape = configs.mlp(8, 6)
    back = BytecodeTape.from_json(tape.to_json())
    X = np.random.default_rng(1).normal(size=(4, 8))
    assert np.array_equal(OracleTape(tape).gradient(X)[1], OracleTape(back).gradient(X)[1])


def _value():
    tape, _ = record(_rosen, [1.5, 2.5])
    return json.loads(tape.to_json())


@pytest.mark.parametrize("mutate, text", [
    (lambda v: v.__setitem__("num_variables", v["num_variables"] + 1), "num_variables"),
    (lambda v: v["opcodes"].__setitem__(5, "Custom"), "is Custom"),
    (lambda v: v.__setitem__("custom_second_args", {"3": 1}), "custom_second_args must be empty"),
    (lambda v: v["arg_indices"].pop(), "arg_indices.len()"),
    (lambda v: v["values"].pop(), "values.len()"),
    (lambda v: v["arg_indices"].__setitem__(len(v["arg_indices"]) - 1, [10 ** 6, 0]), "earlier slot"),
    (lambda v: v.__setitem__("output_index", 10 ** 6), "output_index"),
    (lambda v: v.__setitem__("num_inputs", 10 ** 6), "num_inputs"),
])
def test_corrupt_payloads_are_rejected(mutate, text):
    # tests/serde.rs:175-400: every corruption gives a clean error
    v = _value()
    mutate(v)
    with pytest.raises(TapeValidationError) as e:
        BytecodeTape.from_json(json.dumps(v))
    assert text in str(e.value)


def test_regression_26_mismatched_lengths():
    # tests/serde.rs:175-183
    payload = ('{"opcodes":[0,1],"arg_indices":[[0,0]],"values":[0.0,1.0],"num_inputs":1,"num_variables":2,'
               '"output_index":1,"output_indices":[1],"custom_ops":{},"custom_second_args":{}}')
    with pytest.raises(TapeValidationError):
        BytecodeTape.from_json(payload)
