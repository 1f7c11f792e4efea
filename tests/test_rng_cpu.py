"""Host replay of the device direction stream (echidna_b200.rng): Philox-4x32-10
against the published known-answer vectors of its authors' Random123 suite
(first output word), and the Rademacher mapping."""
import numpy as np

from echidna_b200.rng import philox_bits, rademacher_directions


def test_philox_known_answers():
    # (key, counter) -> first word: zeros, all ones, and the digits of pi
    assert int(philox_bits(0, 0, 0, 0)) == 0x6627E8D5
    ones = np.uint64(0xFFFFFFFFFFFFFFFF)
    assert int(philox_bits(0xFFFFFFFFFFFFFFFF, ones, 0xFFFFFFFF, 0xFFFFFFFF)) == 0x408F276D
    assert int(philox_bits(0x299F31D0A4093822, np.uint64(0x85A308D3243F6A88), 0x13198A2E, 0x03707344)) == 0xD16CFE09


def test_rademacher_directions_shape_and_balance():
    d = rademacher_directions(123, np.arange(64), 16, 50)
    assert d.shape == (64, 16, 50)
    assert set(np.unique(d)) == {-1.0, 1.0}
    assert abs(d.mean()) < 0.05
    w = philox_bits(123, 5, 3, 7)
    assert d[5, 3, 7] == (1.0 if int(w) & 1 else -1.0)
