"""B200-native batched BytecodeTape engine (forward, gradient, HVP, Taylor jets, STDE)."""
from .tape import BReverse, BytecodeTape, OpCode, UNUSED, TapeValidationError, record, record_multi, constant

__all__ = ["BReverse", "BytecodeTape", "OpCode", "UNUSED", "TapeValidationError", "record", "record_multi", "constant"]
