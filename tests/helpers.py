"""Shared test helpers: seeded operand generation and device round trips."""
from __future__ import annotations

import numpy as np

import gpupi_b200 as g

M32 = (1 << 32) - 1


def rand_buf(rng: np.random.Generator, rows: int, stride: int, length: int, pad_canary: int = 0xA5A5A5A5):
    """rows x stride words; the first `length` words of each row random, the
    padding filled with a canary so that writes outside L_c are detected."""
    words = max(rows * stride, 1)
    buf = np.full(words, pad_canary, dtype=np.uint32)
    for r in range(rows):
        if length:
            buf[r * stride: r * stride + length] = rng.integers(0, 1 << 32, size=length, dtype=np.uint64).astype(np.uint32)
    return buf


def to_dev(a: np.ndarray) -> g.DeviceLimbs:
    return g.DeviceLimbs.from_numpy(a)
