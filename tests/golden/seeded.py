"""Seeded test vectors that any machine can regenerate cheaply.

The bench-size fixtures (FCI(12e,12o) to FCI(16e,16o), up to 165 636 900
determinants) cannot hold their input vectors, so the inputs are defined by
a counter hash: element i of vector `seed` is splitmix64(i + seed * golden
ratio), mapped to a double in [-1, 1).  The same function runs in the
fixture script and in the tests, chunked so a 1.3 GB vector is built in a
few seconds.
"""
from __future__ import annotations

import numpy as np

_M64 = (1 << 64) - 1
_GOLDEN = 0x9E3779B97F4A7C15


def hash_vector(n: int, seed: int, chunk: int = 1 << 24) -> np.ndarray:
    """n doubles in [-1, 1), element i = splitmix64(i + seed * 0x9E37...) / 2^63 - 1."""
    out = np.empty(n, np.float64)
    base = np.uint64((seed * _GOLDEN) & _M64)
    c1, c2 = np.uint64(0xBF58476D1CE4E5B9), np.uint64(0x94D049BB133111EB)
    s30, s27, s31, s11 = np.uint64(30), np.uint64(27), np.uint64(31), np.uint64(11)
    with np.errstate(over="ignore"):
        for s0 in range(0, n, chunk):
            z = np.arange(s0, min(n, s0 + chunk), dtype=np.uint64) + base
            z = (z ^ (z >> s30)) * c1
            z = (z ^ (z >> s27)) * c2
            z ^= z >> s31
            out[s0:s0 + len(z)] = (z >> s11).astype(np.float64) * (2.0 ** -52) - 1.0
    return out


def sample_rows(n: int, count: int, seed: int) -> np.ndarray:
    """Sorted distinct determinant indices: the first and last rows plus
    `count` rows drawn uniformly (numpy default_rng(seed))."""
    rng = np.random.default_rng(seed)
    pick = rng.choice(n, size=min(count, n), replace=False)
    return np.unique(np.concatenate([[0, n - 1], pick])).astype(np.int64)
