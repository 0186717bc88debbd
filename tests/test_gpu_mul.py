"""Parity of the batched multiply (schoolbook tiers, three-prime NTT with one,
two and three passes, broadcast and squaring) against exact Python integers.

Mirrors batch_mul_ntt_test.cu (random strides with padding :289-293, size
sweeps :373-402, large-L cases :543-556) and batch_arith_test.cu's crossover
cases (:98-102).  Bit-exact.
"""
import numpy as np
import pytest

import batch_ref as ref
from helpers import rand_buf, to_dev

pytestmark = pytest.mark.gpu


def _check_mul(ctx, N, La, Lb, sA, sB, sC, rng, path="auto", extreme=False):
    A, B, C = rand_buf(rng, N, sA, La), rand_buf(rng, N, sB, Lb), rand_buf(rng, N, sC, 0)
    if extreme:   # all-ones operands: largest coefficients and longest carries
        for r in range(N):
            A[r * sA: r * sA + La] = 0xFFFFFFFF
            B[r * sB: r * sB + Lb] = 0xFFFFFFFF
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C)
    if path == "ntt":
        ctx.mul_ntt(N, dA.ptr, La, sA, dB.ptr, Lb, sB, dC.ptr, sC)
    elif path == "naive":
        import gpupi_b200 as g
        g.mul_naive(N, dA.ptr, La, sA, dB.ptr, Lb, sB, dC.ptr, sC)
    else:
        ctx.mul(N, dA.ptr, La, sA, dB.ptr, Lb, sB, dC.ptr, La + Lb, sC)
    got = dC.numpy()
    if La + Lb <= 300000:
        assert np.array_equal(got, ref.mul(N, A, La, sA, B, Lb, sB, C, sC))
    else:
        # too large for an exact Python product: residues mod 4 primes + exact low limbs
        assert ref.mul_check(N, A, La, sA, B, Lb, sB, got, sC)


@pytest.mark.parametrize("La,Lb", [(1, 1), (3, 3), (4, 3), (6, 4), (8, 8), (12, 5), (16, 16), (17, 3), (3, 17),
                                   (20, 12), (31, 1), (17, 16), (21, 16), (64, 64), (65, 64), (150, 50),
                                   (33, 31), (100, 7), (256, 256), (511, 513), (1000, 24)])
def test_schoolbook(ctx, La, Lb):
    rng = np.random.default_rng(La * 1000 + Lb)
    N = 300 if La + Lb < 64 else 17
    _check_mul(ctx, N, La, Lb, La + 3, Lb + 1, La + Lb + 2, rng, path="naive")
    _check_mul(ctx, 3, La, Lb, La, Lb, La + Lb, rng, path="naive", extreme=True)


@pytest.mark.parametrize("La,Lb", [(3, 3), (6, 4), (11, 11), (15, 15), (18, 15), (11, 18), (21, 21), (34, 29),
                                   (41, 3), (42, 42), (68, 59)])
def test_schoolbook_many_rows(ctx, La, Lb):
    """The splitting tree's lower-level shapes in batches of thousands of rows,
    the operands as every other row of a wider array (the level's even and
    odd views): every row-tile and lane-group boundary of the kernels."""
    rng = np.random.default_rng(7 * La + Lb)
    N = 5003
    _check_mul(ctx, N, La, Lb, 2 * La, 2 * Lb + 1, La + Lb, rng, path="naive")
    _check_mul(ctx, 129, La, Lb, La, Lb, La + Lb, rng, path="naive", extreme=True)


@pytest.mark.parametrize("La,Lb", [(1, 1), (2, 3), (100, 100), (513, 511), (1000, 1000), (2048, 2048),
                                   (3000, 1097), (2049, 2048)])
def test_ntt_single_pass(ctx, La, Lb):
    rng = np.random.default_rng(100 + La + Lb)
    _check_mul(ctx, 5, La, Lb, La + 1, Lb + 2, La + Lb + 3, rng, path="ntt")
    _check_mul(ctx, 2, La, Lb, La, Lb, La + Lb, rng, path="ntt", extreme=True)


@pytest.mark.parametrize("La,Lb,N", [(4097, 1, 2), (4096, 4097, 3), (20000, 30000, 2), (100000, 70000, 1),
                                     (1 << 20, 1 << 20, 1)])
def test_ntt_two_pass(ctx, La, Lb, N):
    rng = np.random.default_rng(La ^ Lb)
    _check_mul(ctx, N, La, Lb, La, Lb, La + Lb, rng, path="ntt")


def test_ntt_extreme_coefficients(ctx):
    """All-ones operands make every convolution coefficient maximal."""
    rng = np.random.default_rng(0)
    _check_mul(ctx, 1, 150000, 150000, 150000, 150000, 300000, rng, path="ntt", extreme=True)
    _check_mul(ctx, 1, 1 << 21, 1 << 21, 1 << 21, 1 << 21, 1 << 22, rng, path="ntt", extreme=True)


def test_ntt_three_pass(ctx):
    """K = 2^23 points: two column passes + the row pass."""
    rng = np.random.default_rng(2 ** 22)
    _check_mul(ctx, 1, 3_000_000, 2_500_000, 3_000_000, 2_500_000, 5_500_000, rng, path="ntt")


def test_broadcast_and_square(ctx):
    """stride 0 broadcast of B (convert_decimal.cu:401-406) and A*A."""
    rng = np.random.default_rng(77)
    N, La, Lb = 9, 6000, 5000
    A, B, C = rand_buf(rng, N, La, La), rand_buf(rng, 1, Lb, Lb), rand_buf(rng, N, La + Lb, 0)
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C)
    ctx.mul(N, dA.ptr, La, La, dB.ptr, Lb, 0, dC.ptr, La + Lb, La + Lb)
    assert np.array_equal(dC.numpy(), ref.mul(N, A, La, La, B, Lb, 0, C, La + Lb))
    S = rand_buf(rng, 1, 2 * La, 0)
    dS = to_dev(S)
    ctx.mul(1, dA.ptr, La, La, dA.ptr, La, La, dS.ptr, 2 * La, 2 * La)
    assert np.array_equal(dS.numpy(), ref.mul(1, A, La, La, A, La, La, S, 2 * La))


@pytest.mark.parametrize("L", [447, 448, 449, 510, 511, 512, 513, 1023, 1024, 1025])
def test_crossover_boundary(ctx, L):
    """Products on both sides of the schoolbook/NTT crossover (batch_arith_test.cu:98-102)."""
    rng = np.random.default_rng(L)
    _check_mul(ctx, 4, L // 2, L - L // 2, L // 2, L - L // 2, L, rng)


def test_uneven_pairs_sample(ctx):
    """A sample of the 4096-uneven-pairs workload: log-uniform lengths in
    [8, 4096] per operand, one call per pair (the reference API takes a single
    length per batch)."""
    rng = np.random.default_rng(0xC2)
    for _ in range(24):
        La = int(2 ** rng.uniform(3, 12))
        Lb = int(2 ** rng.uniform(3, 12))
        _check_mul(ctx, 1, La, Lb, La, Lb, La + Lb, rng)


def test_ntt_cosets(ctx):
    """Products longer than 2^25 points (the largest transform): M cosets of
    K = 2^25 points, residues mod x^K - g^(iK), recombined per coefficient
    through the inverse Vandermonde matrix.  M = 2, 3, 5 and 8 (the limit)."""
    rng = np.random.default_rng(28)
    La, Lb = (1 << 24) + 7, (1 << 24) + 5                      # M = 2
    _check_mul(ctx, 1, La, Lb, La, Lb, La + Lb, rng, path="ntt")
    La, Lb = (1 << 26) + (1 << 24), 5000                       # M = 3, A spans 3 blocks
    _check_mul(ctx, 1, La, Lb, La, Lb, La + Lb, rng, path="ntt")
    L = (1 << 26) + 1                                          # M = 5
    _check_mul(ctx, 1, L, L, L, L, 2 * L, rng, path="ntt")
    _check_mul(ctx, 1, L + 1000, L - 999, L + 1000, L - 999, 2 * L + 1, rng, path="ntt", extreme=True)
    L = 1 << 27                                                # M = 8: need = 2^28 - 1
    _check_mul(ctx, 1, L, L, L, L, 2 * L, rng, path="ntt", extreme=True)


def _all_ones_product(a, b):
    """Limbs of (2^(32a) - 1)(2^(32b) - 1), a >= b >= 1."""
    c = np.full(a + b, 0xFFFFFFFF, dtype=np.uint32)
    c[0] = 1
    c[1:b] = 0
    c[a] = 0xFFFFFFFE
    return c


def test_all_ones_product_formula():
    for a, b in [(1, 1), (3, 2), (5, 2), (4, 4), (6, 3), (9, 1)]:
        v = ((1 << (32 * a)) - 1) * ((1 << (32 * b)) - 1)
        assert int.from_bytes(_all_ones_product(a, b).astype("<u4").tobytes(), "little") == v


def test_ntt_cosets_beyond_2_28(ctx):
    """Products past the reference's 2^28-limb ceiling: M = 9 (one long
    operand folded over nine blocks, exact Python check) and M = 20, the
    largest shape, on all-ones operands (the largest coefficients; coset
    exponents up to 19 * 2^25, above 2^28 and 2^29 through constant factors),
    checked against the closed form."""
    rng = np.random.default_rng(30)
    La, Lb = (1 << 28) + (1 << 24), 3                          # M = 9
    A = rng.integers(0, 1 << 32, size=La, dtype=np.uint64).astype(np.uint32)
    B = np.array([0xFFFFFFFF, 0x12345678, 0x9ABCDEF1], dtype=np.uint32)
    dA, dB = to_dev(A), to_dev(B)
    dC = to_dev(np.full(La + Lb, 0xA5A5A5A5, dtype=np.uint32))
    ctx.mul_ntt(1, dA.ptr, La, La, dB.ptr, Lb, Lb, dC.ptr, La + Lb)
    a = int.from_bytes(A.astype("<u4").tobytes(), "little")
    b = int.from_bytes(B.astype("<u4").tobytes(), "little")
    assert int.from_bytes(dC.numpy().astype("<u4").tobytes(), "little") == a * b
    del A, dA, dC, a
    La, Lb = 1 << 28, (20 << 25) - (1 << 28)                   # M = 20
    dA = to_dev(np.full(La, 0xFFFFFFFF, dtype=np.uint32))
    dB = to_dev(np.full(Lb, 0xFFFFFFFF, dtype=np.uint32))
    dC = to_dev(np.zeros(La + Lb, dtype=np.uint32))
    ctx.mul_ntt(1, dB.ptr, Lb, Lb, dA.ptr, La, La, dC.ptr, La + Lb)
    assert np.array_equal(dC.numpy(), _all_ones_product(Lb, La))


def test_ntt_cosets_broadcast_and_square(ctx):
    """Coset products with a stride-0 B (transformed once for all rows) and a squaring."""
    rng = np.random.default_rng(29)
    N, La, Lb = 2, (1 << 25) - 100, 3000                       # need > 2^25: M = 2
    A, B, C = rand_buf(rng, N, La, La), rand_buf(rng, 1, Lb, Lb), rand_buf(rng, N, La + Lb, 0)
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C)
    ctx.mul_ntt(N, dA.ptr, La, La, dB.ptr, Lb, 0, dC.ptr, La + Lb)
    assert ref.mul_check(N, A, La, La, B, Lb, 0, dC.numpy(), La + Lb)
    L = (1 << 24) + 3                                          # squaring, M = 2
    S = rand_buf(rng, 1, 2 * L, 0)
    dS = to_dev(S)
    ctx.mul_ntt(1, dA.ptr, L, L, dA.ptr, L, L, dS.ptr, 2 * L)
    assert ref.mul_check(1, A, L, L, A, L, L, dS.numpy(), 2 * L)


def _ragged_case(ctx, La, Lb, rng):
    La, Lb = list(La), list(Lb)
    offA = np.concatenate([[0], np.cumsum(La)[:-1]]).astype(np.uint64)
    offB = np.concatenate([[0], np.cumsum(Lb)[:-1]]).astype(np.uint64)
    Lc = [a + b for a, b in zip(La, Lb)]
    offC = np.concatenate([[0], np.cumsum(Lc)[:-1]]).astype(np.uint64)
    A = rng.integers(0, 1 << 32, size=max(1, sum(La)), dtype=np.uint64).astype(np.uint32)
    B = rng.integers(0, 1 << 32, size=max(1, sum(Lb)), dtype=np.uint64).astype(np.uint32)
    C = np.full(max(1, sum(Lc)), 0xA5A5A5A5, dtype=np.uint32)
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C)
    ctx.mul_ragged(dA.ptr, offA, La, dB.ptr, offB, Lb, dC.ptr, offC)
    got = dC.numpy()
    for i in range(len(La)):
        a = ref.row_int(A[int(offA[i]):], 0, La[i], La[i])
        b = ref.row_int(B[int(offB[i]):], 0, Lb[i], Lb[i])
        c = ref.row_int(got[int(offC[i]):], 0, Lc[i], Lc[i])
        assert c == a * b, (i, La[i], Lb[i])


def test_ragged_uneven_pairs(ctx):
    """One call for pairs of independent, uneven lengths (log-uniform in
    [1, 4096], a few empty operands, either operand the longer): schoolbook,
    NTT buckets and zero products mixed."""
    rng = np.random.default_rng(0xC2)
    n = 300
    La = [int(2 ** rng.uniform(0, 12)) for _ in range(n)]
    Lb = [int(2 ** rng.uniform(0, 12)) for _ in range(n)]
    La[5], Lb[9] = 0, 0
    _ragged_case(ctx, La, Lb, rng)


def test_ragged_large_and_single(ctx):
    rng = np.random.default_rng(7)
    _ragged_case(ctx, [70000, 3, 130000], [50000, 90000, 1], rng)
    _ragged_case(ctx, [1], [1], rng)


def _int_rows(buf, N, L):
    out = []
    for r in range(N):
        out.append(int.from_bytes(buf[r * L:(r + 1) * L].astype("<u4").tobytes(), "little"))
    return out


@pytest.mark.parametrize("N,La,Lb,Ld,Le", [(3, 5000, 4000, 4500, 4499), (1, 40000, 50000, 60000, 30000),
                                           (2, 100000, 1, 3, 100000)])
def test_spectra_products_and_sums(ctx, N, La, Lb, Ld, Le):
    """Shared-transform spectra: A B and A B + D E (one inverse transform for
    the sum) equal the exact integers."""
    rng = np.random.default_rng(N * 7 + La + Le)
    A, B = rand_buf(rng, N, La, La), rand_buf(rng, N, Lb, Lb)
    D, E = rand_buf(rng, N, Ld, Ld), rand_buf(rng, N, Le, Le)
    Lc1 = La + Lb
    Lc2 = max(La + Lb, Ld + Le + 1)
    dA, dB, dD, dE = to_dev(A), to_dev(B), to_dev(D), to_dev(E)
    C1 = to_dev(np.zeros(N * Lc1, dtype=np.uint32))
    C2 = to_dev(np.zeros(N * Lc2, dtype=np.uint32))
    ctx.mul_spectra(N, dA.ptr, La, dB.ptr, Lb, C1.ptr, Lc1)
    ctx.mul_spectra(N, dA.ptr, La, dB.ptr, Lb, C2.ptr, Lc2, dD.ptr, Ld, dE.ptr, Le)
    a, b, d, e = _int_rows(A, N, La), _int_rows(B, N, Lb), _int_rows(D, N, Ld), _int_rows(E, N, Le)
    c1, c2 = _int_rows(C1.numpy(), N, Lc1), _int_rows(C2.numpy(), N, Lc2)
    for r in range(N):
        assert c1[r] == a[r] * b[r]
        assert c2[r] == a[r] * b[r] + d[r] * e[r]


def test_spectra_rejects_small_and_overflowing(ctx):
    """Below 8192 transform points the shared-transform path does not apply."""
    import gpupi_b200 as g
    rng = np.random.default_rng(5)
    A = to_dev(rand_buf(rng, 1, 100, 100))
    C = to_dev(np.zeros(200, dtype=np.uint32))
    with pytest.raises(g.GpupiError):
        ctx.mul_spectra(1, A.ptr, 100, A.ptr, 100, C.ptr, 200)
