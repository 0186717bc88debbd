"""CPU restatement of gpupi's batched limb operations.

TEST INFRASTRUCTURE ONLY: used by tests/ and __graft_entry__.smoke() as the
checker of the CUDA kernels; never on the product path.

Operands are numpy uint32 buffers holding N rows at ``row * stride``; lengths
and strides follow gpupi's BatchMPArray (batch_arith.h:10-22).  Each function
returns the buffer the reference would leave in C (only the first ``L_c``
limbs of each row are written; other words are untouched), computed with
Python integers.  File:line citations are into the gpupi project.
"""
from __future__ import annotations

import sys

import numpy as np

sys.set_int_max_str_digits(0)   # decimal strings of very long integers

M32 = (1 << 32) - 1


def row_int(buf: np.ndarray, row: int, length: int, stride: int) -> int:
    base = row * stride
    if length == 0:
        return 0
    return int.from_bytes(np.ascontiguousarray(buf[base:base + length], dtype=np.uint32).tobytes(), "little")


def put_row(buf: np.ndarray, row: int, length: int, stride: int, value: int) -> None:
    base = row * stride
    if length == 0:
        return
    value &= (1 << (32 * length)) - 1
    buf[base:base + length] = np.frombuffer(value.to_bytes(4 * length, "little"), dtype=np.uint32)


# Size-independent product check for operands too large for an exact Python
# product: residues modulo fixed primes below 2^61 plus the exact low limbs.
CHECK_PRIMES = (2305843009213693951, 2305843009213693921, 2305843009213693907, 4611686018427387847)


def mul_check(N, A, La, sA, B, Lb, sB, C, sC, low_limbs=4096) -> bool:
    Lc = La + Lb
    for r in range(N):
        a, b, c = row_int(A, r, La, sA), row_int(B, r, Lb, sB), row_int(C, r, Lc, sC)
        for p in CHECK_PRIMES:
            if (a % p) * (b % p) % p != c % p:
                return False
        k = min(low_limbs, Lc)
        m = (1 << (32 * k)) - 1
        if ((a & m) * (b & m)) & m != c & m:
            return False
        if c.bit_length() > 32 * Lc:
            return False
    return True


def _rows(op, N, C, Lc, sC):
    out = C.copy()
    for r in range(N):
        put_row(out, r, Lc, sC, op(r) & ((1 << (32 * Lc)) - 1))
    return out


def add(N, A, La, sA, B, Lb, sB, C, Lc, sC):
    """batch_add.h:6-17: sum over max(La,Lb)+1 limbs, truncated/zero-extended."""
    return _rows(lambda r: row_int(A, r, La, sA) + row_int(B, r, Lb, sB), N, C, Lc, sC)


def sub(N, A, La, sA, B, Lb, sB, C, Lc, sC):
    """batch_sub.h:6-13: A - B mod 2^(32 Lc)."""
    return _rows(lambda r: row_int(A, r, La, sA) - row_int(B, r, Lb, sB), N, C, Lc, sC)


def add_small(N, A, La, sA, b, C, Lc, sC):
    """batch_add_small.h:6-14."""
    return _rows(lambda r: row_int(A, r, La, sA) + b, N, C, Lc, sC)


def sub_small(N, A, La, sA, b, C, Lc, sC):
    """batch_sub_small.h:6-13."""
    return _rows(lambda r: row_int(A, r, La, sA) - b, N, C, Lc, sC)


def mul_small(N, A, La, sA, b, C, Lc, sC):
    """batch_mul_small.h:6-14."""
    return _rows(lambda r: row_int(A, r, La, sA) * b, N, C, Lc, sC)


def shift_add(N, A, La, sA, B, Lb, sB, shift, C, Lc, sC):
    """batch_shift_add.h:6-21."""
    return _rows(lambda r: (row_int(A, r, La, sA) << shift) + row_int(B, r, Lb, sB), N, C, Lc, sC)


def shift_sub(N, A, La, sA, B, Lb, sB, shift, C, Lc, sC):
    """batch_shift_sub.h:6-14."""
    return _rows(lambda r: (row_int(A, r, La, sA) << shift) - row_int(B, r, Lb, sB), N, C, Lc, sC)


def mul(N, A, La, sA, B, Lb, sB, C, sC):
    """batch_mul_naive.h:7-15 / batch_mul_ntt.h:13-22: exact product, La+Lb limbs."""
    return _rows(lambda r: row_int(A, r, La, sA) * row_int(B, r, Lb, sB), N, C, La + Lb, sC)


def shift_bits(N, A, La, sA, B, Lb, sB, shift):
    """batch_shift.cu:22-86: signed shift of the La-limb value, truncated to Lb."""
    def f(r):
        v = row_int(A, r, La, sA)
        return v << shift if shift >= 0 else v >> (-shift)
    return _rows(f, N, B, Lb, sB)


def exactdiv_small(N, A, La, sA, b):
    """batch_exactdiv_small.cu:15-141: q with q*b == A mod 2^(32 La)."""
    inv = pow(b, -1, 1 << (32 * La)) if La else 0
    return _rows(lambda r: row_int(A, r, La, sA) * inv, N, A, La, sA)


def bitlength_max(N, A, La, sA):
    """batch_bitlength.cu:186-225 (bit mode)."""
    return max([row_int(A, r, La, sA).bit_length() for r in range(N)] + [0])


def limblength_max(N, A, La, sA):
    """batch_bitlength.cu limb mode: smallest limb count holding every row."""
    return max([(row_int(A, r, La, sA).bit_length() + 31) // 32 for r in range(N)] + [0])


def decimal_naive(N, A, L_limb, sA, L_dec, s_out, out: bytearray):
    """batch_decimal_naive.cu:16-217: truncated digits of X/2^(32 L_limb),
    least significant first (out[0] is the 10^-L_dec place)."""
    for r in range(N):
        x = row_int(A, r, L_limb, sA)
        v = (x * 10 ** L_dec) >> (32 * L_limb)
        s = str(v).rjust(L_dec, "0")[-L_dec:]
        out[r * s_out: r * s_out + L_dec] = s[::-1].encode()
    return out
