"""Host replay of the device's counter-based direction stream.

The kernels draw Rademacher directions and coordinate samples from
Philox-4x32-10 (Salmon, Moraes, Dror and Shaw, "Parallel random numbers: as
easy as 1, 2, 3", SC'11) keyed by the caller's 64-bit seed, with the counter
(point low word, point high word, direction, coordinate).  These functions give
the same words on the host, so a device-RNG launch can be reproduced with
host-supplied directions.
"""
from __future__ import annotations

import numpy as np

_M32 = np.uint64(0xFFFFFFFF)


def philox_bits(seed: int, point, direction, i):
    """First output word of Philox-4x32-10 for each (point, direction, i); the
    arguments broadcast against each other (numpy uint64 arithmetic)."""
    point = np.asarray(point, dtype=np.uint64)
    c0 = point & _M32
    c1 = point >> np.uint64(32)
    c2 = np.asarray(direction, dtype=np.uint64) & _M32
    c3 = np.asarray(i, dtype=np.uint64) & _M32
    c0, c1, c2, c3 = (a.copy() for a in np.broadcast_arrays(c0, c1, c2, c3))
    k0 = np.uint64(seed & 0xFFFFFFFF)
    k1 = np.uint64((seed >> 32) & 0xFFFFFFFF)
    for _ in range(10):
        p0 = np.uint64(0xD2511F53) * c0
        p1 = np.uint64(0xCD9E8D57) * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & _M32
        hi1, lo1 = p1 >> np.uint64(32), p1 & _M32
        c0, c1, c2, c3 = hi1 ^ c1 ^ k0, lo1, hi0 ^ c3 ^ k1, lo0
        k0 = (k0 + np.uint64(0x9E3779B9)) & _M32
        k1 = (k1 + np.uint64(0xBB67AE85)) & _M32
    return c0


def rademacher_directions(seed: int, points, num_directions: int, n: int, dtype=np.float64):
    """The device's Rademacher directions ``[len(points), S, n]`` for a point-direction
    launch with device RNG: +1 where bit 0 of the word is set, else -1."""
    p = np.asarray(points, dtype=np.uint64)[:, None, None]
    s = np.arange(num_directions, dtype=np.uint64)[None, :, None]
    i = np.arange(n, dtype=np.uint64)[None, None, :]
    return np.where(philox_bits(seed, p, s, i) & np.uint64(1), 1.0, -1.0).astype(dtype)
