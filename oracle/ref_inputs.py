"""Seeded inputs of the benchmark configurations (test infrastructure only).

The same splitmix64 streams as oracle/ref_configs.cu, so that a result of
this library on these inputs can be compared with the digest of the
reference build's result on the same inputs (tests/golden/ref_fixtures.json,
made by oracle/make_ref_fixtures.py).

  c2_inputs()       4096 uneven pairs: per operand e in 3..11 and a length
                    2^e + r, r < 2^e (log-uniform over [8, 4096) octave by
                    octave), then the limbs of every A, then of every B
  c3_inputs(log2L)  two L-limb operands (L = 2^log2L)
  c4_input()        one 2^25-limb fraction (2^30 bits)
"""
from __future__ import annotations

import hashlib

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, start: int, count: int) -> np.ndarray:
    """Outputs start .. start+count-1 of the splitmix64 stream of `seed`
    (output k mixes seed + (k+1) * golden)."""
    with np.errstate(over="ignore"):
        k = np.arange(start + 1, start + count + 1, dtype=np.uint64)
        z = np.uint64(seed) + k * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def limbs(seed: int, start: int, n: int) -> np.ndarray:
    """n limbs from stream outputs start, start+1, ...: low half then high half."""
    z = splitmix64(seed, start, (n + 1) // 2)
    out = np.empty(2 * z.size, dtype=np.uint32)
    out[0::2] = (z & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    out[1::2] = (z >> np.uint64(32)).astype(np.uint32)
    return out[:n]


def c2_inputs(n: int = 4096):
    z = splitmix64(0xC2, 0, n)
    ea = np.uint64(3) + z % np.uint64(9)
    eb = np.uint64(3) + (z >> np.uint64(8)) % np.uint64(9)
    one = np.uint64(1)
    La = (one << ea) + ((z >> np.uint64(16)) & ((one << ea) - one))
    Lb = (one << eb) + ((z >> np.uint64(40)) & ((one << eb) - one))
    La, Lb = La.astype(np.uint32), Lb.astype(np.uint32)
    ta, tb = int(La.sum()), int(Lb.sum())
    A = limbs(0xC2, n, ta)
    B = limbs(0xC2, n + (ta + 1) // 2, tb)
    return La, Lb, A, B


def c3_inputs(log2L: int = 27):
    L = 1 << log2L
    A = limbs(0xC3, 0, L)
    B = limbs(0xC3, (L + 1) // 2, L)
    return A, B


def c4_input():
    return limbs(0xC4, 0, 1 << 25)


def digest(data) -> dict:
    """SHA-256, byte length and the first / last 16 bytes of a result."""
    b = memoryview(np.ascontiguousarray(data)).cast("B") if not isinstance(data, (bytes, bytearray)) else data
    return {"sha256": hashlib.sha256(b).hexdigest(), "bytes": len(b), "head": bytes(b[:16]).hex(),
            "tail": bytes(b[-16:]).hex()}
