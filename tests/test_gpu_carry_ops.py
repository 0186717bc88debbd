"""Parity of the carry-chain family (add, sub, *_small, mul_small, shift_add,
shift_sub), shift and bitlength kernels against the CPU oracle.

Cases follow the reference's own tests: fixed (N, L_a, L_b, L_c, strides)
tables (batch_add_test.cu:632-642), output-padding canaries, in-place
aliasing (:397), long carry chains (:175-248) and zero-length operands.
All comparisons are bit-exact.
"""
import numpy as np
import pytest

import batch_ref as ref
from helpers import rand_buf, to_dev

pytestmark = pytest.mark.gpu

# (N, La, Lb, Lc, sA, sB, sC) -- batch_add_test.cu:632-642 plus long rows
# that take the multi-tile path and huge batches of short rows.
FIXED = [
    (37, 7, 5, 9, 11, 9, 13),
    (19, 17, 23, 12, 20, 29, 16),
    (11, 31, 30, 31, 35, 34, 36),
    (9, 64, 47, 80, 69, 52, 84),
    (128, 300, 300, 301, 300, 300, 301),
    (4, 5000, 4097, 5001, 5000, 4097, 5001),
    (3, 6000, 6000, 7000, 6000, 6000, 7008),
    (2, 8192, 8191, 4096, 8192, 8191, 4096),
    (5, 0, 23, 24, 3, 27, 29),
    (5000, 3, 4, 6, 3, 4, 6),
    (4099, 9, 11, 13, 10, 12, 15),
    (3001, 16, 16, 16, 16, 16, 17),
    (2500, 20, 31, 32, 21, 31, 33),
    (1, 100000, 99999, 100001, 100000, 99999, 100001),
]


@pytest.mark.parametrize("case", FIXED)
@pytest.mark.parametrize("op", ["add", "sub"])
def test_add_sub(ctx, case, op):
    N, La, Lb, Lc, sA, sB, sC = case
    rng = np.random.default_rng(123456789 + La)
    A, B, C = rand_buf(rng, N, sA, La), rand_buf(rng, N, sB, Lb), rand_buf(rng, N, sC, 0)
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C)
    getattr(ctx, op)(N, dA.ptr, La, sA, dB.ptr, Lb, sB, dC.ptr, Lc, sC)
    want = getattr(ref, op)(N, A, La, sA, B, Lb, sB, C, Lc, sC)
    assert np.array_equal(dC.numpy(), want)


@pytest.mark.parametrize("L", [1, 31, 32, 33, 4095, 4096, 4097, 20000, 70000])
def test_long_carry_chain(ctx, L):
    """All-ones + 1 carries through every limb and every tile
    (batch_add_test.cu:175-248); the borrow mirror for subtraction."""
    N = 2
    A = np.full(N * L, 0xFFFFFFFF, dtype=np.uint32)
    B = np.zeros(N * L, dtype=np.uint32)
    B[0] = 1
    B[L] = 1
    C = np.zeros(N * (L + 1), dtype=np.uint32)
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C)
    ctx.add(N, dA.ptr, L, L, dB.ptr, L, L, dC.ptr, L + 1, L + 1)
    assert np.array_equal(dC.numpy(), ref.add(N, A, L, L, B, L, L, C, L + 1, L + 1))
    Z = np.zeros(N * L, dtype=np.uint32)
    dZ, dD = to_dev(Z), to_dev(C)
    ctx.sub(N, dZ.ptr, L, L, dB.ptr, L, L, dD.ptr, L, L + 1)
    assert np.array_equal(dD.numpy(), ref.sub(N, Z, L, L, B, L, L, C, L, L + 1))


def test_carry_chain_mixed_runs(ctx):
    """Random runs of all-ones limbs so tile boundaries see every carry state."""
    rng = np.random.default_rng(7)
    N, L = 3, 50000
    A = rand_buf(rng, N, L, L)
    for r in range(N):
        for _ in range(40):
            s = int(rng.integers(0, L - 9000))
            A[r * L + s: r * L + s + int(rng.integers(1, 9000))] = 0xFFFFFFFF
    B = np.zeros(N * L, dtype=np.uint32)
    B[::L] = rng.integers(1, 1 << 32, size=N, dtype=np.uint64).astype(np.uint32)
    C = np.zeros(N * (L + 1), dtype=np.uint32)
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C)
    ctx.add(N, dA.ptr, L, L, dB.ptr, L, L, dC.ptr, L + 1, L + 1)
    assert np.array_equal(dC.numpy(), ref.add(N, A, L, L, B, L, L, C, L + 1, L + 1))


@pytest.mark.parametrize("op", ["add", "sub"])
def test_in_place(ctx, op):
    """C aliases A with the same length and stride (batch_add.h:15-16)."""
    rng = np.random.default_rng(11)
    N, L = 7, 4097
    A, B = rand_buf(rng, N, L, L), rand_buf(rng, N, L, L)
    dA, dB = to_dev(A), to_dev(B)
    getattr(ctx, op)(N, dA.ptr, L, L, dB.ptr, L, L, dA.ptr, L, L)
    assert np.array_equal(dA.numpy(), getattr(ref, op)(N, A, L, L, B, L, L, A, L, L))


@pytest.mark.parametrize("case", [(37, 7, 9, 11, 13), (5, 300, 301, 300, 301), (3, 9000, 9001, 9000, 9001),
                                  (4096, 5, 6, 5, 6), (2, 0, 3, 1, 3)])
@pytest.mark.parametrize("op", ["add_small", "sub_small", "mul_small"])
def test_small_ops(ctx, case, op):
    N, La, Lc, sA, sC = case
    rng = np.random.default_rng(99 + La)
    b = int(rng.integers(1, 1 << 32))
    A, C = rand_buf(rng, N, sA, La), rand_buf(rng, N, sC, 0)
    dA, dC = to_dev(A), to_dev(C)
    getattr(ctx, op)(N, dA.ptr, La, sA, b, dC.ptr, Lc, sC)
    assert np.array_equal(dC.numpy(), getattr(ref, op)(N, A, La, sA, b, C, Lc, sC))


@pytest.mark.parametrize("shift", [0, 1, 15, 31, 32, 33, 255, 1000])
@pytest.mark.parametrize("op", ["shift_add", "shift_sub"])
def test_shift_addsub(ctx, shift, op):
    rng = np.random.default_rng(5 + shift)
    for (N, La, Lb, sA, sB) in [(64, 10, 9, 10, 9), (3, 5000, 5100, 5000, 5100), (3000, 6, 9, 12, 9)]:
        Lc = max(La + shift // 32 + 1, Lb) + 1
        A, B, C = rand_buf(rng, N, sA, La), rand_buf(rng, N, sB, Lb), rand_buf(rng, N, Lc, 0)
        dA, dB, dC = to_dev(A), to_dev(B), to_dev(C)
        getattr(ctx, op)(N, dA.ptr, La, sA, dB.ptr, Lb, sB, shift, dC.ptr, Lc, Lc)
        assert np.array_equal(dC.numpy(), getattr(ref, op)(N, A, La, sA, B, Lb, sB, shift, C, Lc, Lc))


@pytest.mark.parametrize("shift", [-1000, -33, -32, -31, -1, 0, 1, 31, 32, 33, 1000])
def test_shift_bits(ctx, shift):
    rng = np.random.default_rng(1234 + shift)
    for (N, La, Lb, sA, sB) in [(21, 13, 17, 15, 19), (2, 7000, 6900, 7000, 6900), (3000, 4, 5, 4, 5)]:
        A, B = rand_buf(rng, N, sA, La), rand_buf(rng, N, sB, 0)
        dA, dB = to_dev(A), to_dev(B)
        ctx.shift_bits(N, dA.ptr, La, sA, dB.ptr, Lb, sB, shift)
        assert np.array_equal(dB.numpy(), ref.shift_bits(N, A, La, sA, B, Lb, sB, shift))


@pytest.mark.parametrize("divisor", [1, 3, 5, 0xFFFFFFFF, 0xFFFFFFFD, 0x13579BDF, 830297, 156590819])
def test_exactdiv(ctx, divisor):
    """Cases of batch_exactdiv_small_test.cu:279-305: exact multiples of b."""
    rng = np.random.default_rng(0x6FDDC0FFEE123456 & 0xFFFFFFFF)
    for (N, L, stride) in [(1, 1, 4), (7, 2, 5), (19, 7, 11), (33, 8, 12), (65, 32, 37), (96, 64, 70),
                           (37, 127, 127), (68, 128, 128)]:
        A = rand_buf(rng, N, stride, 0)
        for r in range(N):
            q = int(rng.integers(0, 1 << 62)) << (32 * L - 64) if L >= 2 else int(rng.integers(0, 1 << 32))
            q = (q * 0x9E3779B97F4A7C15 + r) % (1 << (32 * L))
            v = (q * divisor) % (1 << (32 * L))
            ref.put_row(A, r, L, stride, v)
        dA = to_dev(A)
        ctx.exactdiv_small(N, dA.ptr, L, stride, divisor)
        assert np.array_equal(dA.numpy(), ref.exactdiv_small(N, A, L, stride, divisor))


def test_bitlength(ctx):
    rng = np.random.default_rng(3)
    # both kernels: chunked (long rows, or few rows) and one thread per row
    # (short rows, or 65536 rows and more)
    for (N, L, stride) in [(1, 1, 1), (100, 17, 20), (5, 9000, 9000), (40000, 3, 3), (5000, 100, 101),
                           (4096, 3000, 3000), (70000, 70, 70), (8192, 64, 64)]:
        A = rand_buf(rng, N, stride, L)
        for r in range(N):
            cut = int(rng.integers(0, L + 1))
            A[r * stride + cut: r * stride + L] = 0
        dA = to_dev(A)
        assert ctx.bitlength_max(N, dA.ptr, L, stride) == ref.bitlength_max(N, A, L, stride)
        assert ctx.limblength_max(N, dA.ptr, L, stride) == ref.limblength_max(N, A, L, stride)
    Z = np.zeros(64, dtype=np.uint32)
    dZ = to_dev(Z)
    assert ctx.limblength_max(4, dZ.ptr, 16, 16) == 0
    # many long rows, all but one far shorter than the batch length
    N, L = 4096, 20000
    A = np.zeros(N * L, dtype=np.uint32)
    A[np.arange(N) * L + 7] = 1
    A[1234 * L + 19000] = 5
    dA = to_dev(A)
    assert ctx.limblength_max(N, dA.ptr, L, L) == 19001
    assert ctx.bitlength_max(N, dA.ptr, L, L) == 19000 * 32 + 3


def test_invalid_metadata(ctx):
    """Malformed views return cudaErrorInvalidValue (batch_arith_test.cu:155-167)."""
    import gpupi_b200 as g
    d = to_dev(np.zeros(64, dtype=np.uint32))
    with pytest.raises(g.GpupiError):
        ctx.add(2, d.ptr, 9, 8, d.ptr, 1, 8, d.ptr, 4, 8)          # length > stride
    with pytest.raises(g.GpupiError):
        ctx.mul(1, d.ptr, 3, 3, d.ptr, 3, 3, d.ptr, 5, 6)          # Lc != La + Lb
    with pytest.raises(g.GpupiError):
        ctx.exactdiv_small(1, d.ptr, 2, 2, 4)                     # even divisor
    with pytest.raises(g.GpupiError):
        ctx.shift_add(1, d.ptr, 2, 2, d.ptr + 64, 2, 2, 3, d.ptr, 4, 4)   # C aliases A
