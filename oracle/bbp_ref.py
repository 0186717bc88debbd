"""CPU restatement of the BBP fixed-point spot check (test infrastructure only).

Computes the same integer as the GPU kernel (gpupi_b200/csrc/bbp.cu):
floor(2^64 * frac(.)) of every term of
    frac(16^n pi) = frac(4 S1 - 2 S4 - S5 - S6),
summed modulo 2^64 with weights 4, -2, -1, -1.  Terms k <= n are
floor(2^64 frac(2^E / m)) with the even denominators rewritten over odd
moduli (16^e/(8k+4) = 4 16^(e-1)/(2k+1), 16^e/(8k+6) = 8 16^(e-1)/(4k+3));
k = n for j = 4, 6 is floor(2^64 / (8n+j)); the tail k = n+1 .. n+15 is
floor(2^(64-4d) / (8k+j)).  Every step is exact integer arithmetic and
addition mod 2^64 is associative, so the GPU's sum, in any order, equals this
one bit for bit.  Pure Python: for positions up to a few thousand.
"""

M64 = (1 << 64) - 1


def frac_pow2(E: int, m: int) -> int:
    """floor(2^64 * frac(2^E / m)) for odd m >= 1."""
    return (pow(2, E, m) << 64) // m


def bbp_fraction(n: int) -> int:
    s = 0
    for k in range(n + 1):
        e = n - k
        s += frac_pow2(4 * e, 8 * k + 1) << 2
        s -= (frac_pow2(4 * e - 2, 2 * k + 1) if e else ((1 << 64) // (8 * n + 4))) << 1
        s -= frac_pow2(4 * e, 8 * k + 5)
        s -= frac_pow2(4 * e - 1, 4 * k + 3) if e else ((1 << 64) // (8 * n + 6))
    for d in range(1, 16):
        k = n + d
        num = 1 << (64 - 4 * d)
        s += (num // (8 * k + 1)) << 2
        s -= (num // (8 * k + 4)) << 1
        s -= num // (8 * k + 5)
        s -= num // (8 * k + 6)
    return s & M64
