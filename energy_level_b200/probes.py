"""Host mirror of the library's counter-based Rademacher probes.

The device draws probe p, row r as the sign of
splitmix64(splitmix64(seed ^ (p+1) * 0xD1B54A32D192ED03) + r) (top bit set ->
-1), independent of launch shape and chunking.  This numpy restatement lets a
CPU checker use exactly the probes the GPU used.
"""
from __future__ import annotations

import numpy as np

_M = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix64(x):
    x = (x + np.uint64(0x9E3779B97F4A7C15)) & _M
    x = ((x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & _M
    x = ((x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & _M
    return x ^ (x >> np.uint64(31))


def rademacher_host(seed: int, probe0: int, nvec: int, dim: int) -> np.ndarray:
    """int8 [nvec, dim] of +-1 equal to the device probes probe0..probe0+nvec-1."""
    out = np.empty((nvec, dim), dtype=np.int8)
    rows = np.arange(dim, dtype=np.uint64)
    with np.errstate(over="ignore"):
        for v in range(nvec):
            stream = np.uint64(probe0 + v + 1)
            key = _splitmix64(np.uint64(seed) ^ ((stream * np.uint64(0xD1B54A32D192ED03)) & _M))
            h = _splitmix64((key + rows) & _M)
            out[v] = np.where((h >> np.uint64(63)) != 0, -1, 1).astype(np.int8)
    return out
