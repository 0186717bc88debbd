"""Parity of decimal conversion: the leaf kernel (batch_decimal_naive) and the
divide-and-conquer converter (convert_decimal_equal_split) against the CPU
oracle, which restates the reference algorithm exactly (including its
truncating splits).  Cases follow batch_decimal_naive_test.cu:266-283 and
convert_decimal_test.cu:301-304.
"""
import numpy as np
import pytest

import batch_ref as ref
import pi_ref
from helpers import rand_buf, to_dev

pytestmark = pytest.mark.gpu

NAIVE_CASES = [(1, 1, 0), (2, 1, 7), (4, 2, 0), (70000, 1, 2), (7, 3, 5), (8, 4, 0), (5, 5, 9), (9, 8, 3),
               (3, 15, 0), (6, 31, 11), (2, 63, 0), (1, 127, 13), (4, 255, 0), (2, 511, 17), (1, 1023, 0),
               (1, 2047, 19)]


@pytest.mark.parametrize("N,L,extra", NAIVE_CASES)
def test_decimal_naive(N, L, extra):
    import gpupi_b200 as g
    rng = np.random.default_rng(N * 7919 + L)
    L_dec = int(L * 32 * 0.30103) + extra
    A = rand_buf(rng, N, L, L)
    dA = to_dev(A)
    out = g.DeviceBytes(N * L_dec)
    g.decimal_naive(N, dA.ptr, L, L, out.ptr, L_dec, L_dec)
    want = ref.decimal_naive(N, A, L, L, L_dec, L_dec, bytearray(N * L_dec))
    assert out.text().encode() == bytes(want)


def _xorshift_words(n, seed, bits):
    """The seeded fraction generator of convert_decimal_test.cu:56-78."""
    state = seed or 1
    words = []
    M = (1 << 64) - 1
    for _ in range(n):
        state ^= state >> 12
        state ^= (state << 25) & M
        state ^= state >> 27
        words.append(((state * 2685821657736338717) & M) >> 32)
    extra = bits & 31
    if extra:
        words[-1] &= (1 << extra) - 1
    if words and words[-1] == 0:
        words[-1] = 1 if not extra else 1 & ((1 << extra) - 1)
    return words


@pytest.mark.parametrize("digits,seed", [(477, 0x1234), (954, 0x2345), (1908, 0x3456), (3816, 0x4567)])
def test_convert_decimal_reference_cases(ctx, digits, seed):
    """convert_decimal_test.cu:301-304: leaf 477, input bits = bits(digits) + 64."""
    import gpupi_b200 as g
    bits = pi_ref.bits_for_digits(digits) + 64
    limbs = (bits + 31) // 32
    words = _xorshift_words(limbs, seed, bits)
    X = np.array(words, dtype=np.uint32)
    dX = to_dev(X)
    out = g.DeviceBytes(digits)
    ctx.convert_decimal(dX.ptr, limbs, bits, digits, 477, out.ptr)
    want = pi_ref.convert_decimal(pi_ref.from_limbs(words), limbs, bits, digits, 477)
    assert out.text() == want


@pytest.mark.parametrize("total,leaf", [(1000, 500), (20032, 313), (65536 * 3, 384), (100096, 391)])
def test_convert_decimal_random(ctx, total, leaf):
    import gpupi_b200 as g
    rng = np.random.default_rng(total)
    bits = pi_ref.bits_for_digits(total) + 96
    limbs = (bits + 31) // 32
    X = rand_buf(rng, 1, limbs, limbs)
    dX = to_dev(X)
    out = g.DeviceBytes(total)
    ctx.convert_decimal(dX.ptr, limbs, limbs * 32, total, leaf, out.ptr)
    want = pi_ref.convert_decimal(pi_ref.from_limbs(X), limbs, limbs * 32, total, leaf)
    assert out.text() == want
