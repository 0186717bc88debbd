"""Pure-Python restatement of gpupi's ``pi_bs_gpu`` pipeline.

TEST INFRASTRUCTURE ONLY.  This module is the small-size oracle: tests,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may use
it as a checker.  Nothing on the product path imports it.

Every step follows the reference's arithmetic exactly, including the places
where the reference's buffer lengths decide a truncation (``compact``-derived
limb counts, modular subtraction widths and the top-limb sign probe of the
recursive inverse).  Python integers are exact, so the only thing this module
has to get right is *which* integer the reference computes at each step.

References are ``file:line`` inside the gpupi project.
"""
from __future__ import annotations

import sys
from dataclasses import dataclass

sys.set_int_max_str_digits(0)   # decimal strings of very long integers

MASK32 = (1 << 32) - 1
VALIDATION_MOD = 1_000_000_007          # pi_bs_gpu.cu:149
BLOCK_DIV_LO = 830297                    # pi_bs_gpu.cu:147
BLOCK_DIV_HI = 156590819                 # pi_bs_gpu.cu:148
INVERSE_CPU_LIMIT = 32 * 1024            # pi_bs_gpu.cu:1143
LOG2_10 = 3.32192809488736234787         # convert_decimal.cu:15
PRECISION_MARGIN_BITS = 34               # convert_decimal.cu:16


def nlimbs(x: int) -> int:
    """Number of 32-bit limbs ``compact()`` reports for a non-negative int
    (batch_arith.cu:415-424 via batch_bitlength.cu limb mode): 0 for 0."""
    return (x.bit_length() + 31) // 32


def mod_limbs(x: int, length: int) -> int:
    """Value of a ``length``-limb buffer holding x (two's complement wrap)."""
    return x & ((1 << (32 * length)) - 1)


def to_limbs(x: int, length: int | None = None) -> list[int]:
    n = nlimbs(x) if length is None else length
    return [(x >> (32 * i)) & MASK32 for i in range(n)]


def from_limbs(limbs) -> int:
    v = 0
    for i, w in enumerate(limbs):
        v |= int(w) << (32 * i)
    return v


# ---------------------------------------------------------------------------
# Leaves (pi_bs_gpu.cu:17-131)
# ---------------------------------------------------------------------------

def _reduce_gcd_quotient(a: int, b: int) -> tuple[int, int]:
    """pi_bs_gpu.cu:17-34: divide both by 3, 5, 23, 29 once each if both divisible."""
    for d in (3, 5, 23, 29):
        if a % d == 0 and b % d == 0:
            a //= d
            b //= d
    return a, b


def leaf_term(i: int) -> tuple[int, int, int]:
    """P, Q, R of one Chudnovsky term i, after the gcd pre-reduction
    (construct_leaf_17 body, pi_bs_gpu.cu:48-95)."""
    p1, p2, p3 = 6 * i + 1, 2 * i + 1, 6 * i + 5
    q1 = q2 = q3 = i + 1
    q4, q5, q6 = 640320 >> 6, 40020 >> 2, 426880 >> 7
    r1 = 545140134 * i + 13591409
    if p1 % 5 == 0 and q1 % 5 == 0:
        p1 //= 5
        q1 //= 5
    if p1 % 5 == 0 and q2 % 5 == 0:
        p1 //= 5
        q2 //= 5
    if p1 % 5 == 0 and q3 % 5 == 0:
        p1 //= 5
        q3 //= 5
    p1, q4 = _reduce_gcd_quotient(p1, q4)
    p1, q5 = _reduce_gcd_quotient(p1, q5)
    p2, q4 = _reduce_gcd_quotient(p2, q4)
    p2, q5 = _reduce_gcd_quotient(p2, q5)
    p3, q4 = _reduce_gcd_quotient(p3, q4)
    p3, q5 = _reduce_gcd_quotient(p3, q5)
    P = p1 * p2 * p3
    Q = q1 * q2 * q3 * q4 * q5 * q6
    R = r1 * q1 * q2 * q3 * q4 * q5
    assert P < 1 << 96 and Q < 1 << 128 and R < 1 << 192
    return P, Q, R


def leaf_index(i2: int, is_head: bool) -> int:
    """Term index of leaf row i2 (pi_bs_gpu.cu:40-45)."""
    return i2 * 17 + 16 if is_head else i2 + (i2 >> 4)


# ---------------------------------------------------------------------------
# Binary splitting (pi_bs_gpu.cu:504-792)
# ---------------------------------------------------------------------------

def binary_split(N: int) -> tuple[int, int]:
    """Q and R of the whole 17N-term series, following the level loop of
    binary_split_batched (pi_bs_gpu.cu:625-785)."""
    assert N > 0 and N & (N - 1) == 0
    n = 16 * N
    heads = [leaf_term(leaf_index(j, True)) for j in range(N)]
    P0 = [h[0] for h in heads]
    Q0 = [h[1] for h in heads]
    R0 = [h[2] for h in heads]
    rows = [leaf_term(leaf_index(j, False)) for j in range(n)]
    P = [r[0] for r in rows]
    Q = [r[1] for r in rows]
    R = [r[2] for r in rows]
    n1 = n
    while n1 > 1:
        subtract = n1 == n or n1 == (n >> 4)
        ignore_last_p = 1 if n1 <= N else 0
        half = n1 // 2
        shift = 15 * ((n // n1) + ((n // n1) >> 4))
        newP = [P[2 * k] * P[2 * k + 1] for k in range(half - ignore_last_p)]
        newQ = [Q[2 * k] * Q[2 * k + 1] for k in range(half)]
        newR = []
        for k in range(half):
            a = (R[2 * k] * Q[2 * k + 1]) << shift
            b = P[2 * k] * R[2 * k + 1]
            v = a - b if subtract else a + b
            assert v >= 0, "shift_sub result would wrap"
            newR.append(v)
        P, Q, R = newP, newQ, newR
        if n1 == (n >> 3):
            # head merge, pi_bs_gpu.cu:725-784
            mP = [P[k] * P0[k] for k in range(half)]
            mQ = [Q[k] * Q0[k] for k in range(half)]
            mR = [((R[k] * Q0[k]) << 15) + P[k] * R0[k] for k in range(half)]
            for arr in (mP, mQ, mR):
                for k in range(half):
                    for d in (BLOCK_DIV_LO, BLOCK_DIV_HI):
                        assert arr[k] % d == 0
                        arr[k] //= d
            P, Q, R = mP, mQ, mR
        n1 >>= 1
    return Q[0], R[0]


# ---------------------------------------------------------------------------
# sqrt(10005) Pell iteration (pi_bs_gpu.cu:1346-1522)
# ---------------------------------------------------------------------------

def sqrt_10005(target_digits: int) -> tuple[int, int]:
    p, q = 4001, 40
    valid = 7.5
    while valid < target_digits:
        valid *= 2
        p, q = p * p + 10005 * q * q, 2 * p * q
    return p, q


# ---------------------------------------------------------------------------
# Recursive inverse (pi_bs_gpu.cu:1145-1344)
# ---------------------------------------------------------------------------

def inverse_levels(L: int) -> list[int]:
    """Level list of recursive_inverse (pi_bs_gpu.cu:1187-1192)."""
    levels = [L]
    while levels[-1] > INVERSE_CPU_LIMIT:
        m = ((levels[-1] - 2) // 4) & ~31
        levels.append(levels[-1] - 2 * m)
    return levels


def recursive_inverse(x: int, x_len: int, L: int) -> int:
    """y ~ 2^L / x exactly as recursive_inverse computes it, including the
    modular widths of its in-place subtractions and the top-limb sign test."""
    levels = inverse_levels(L)
    y_len = x_len                                   # y_out = create(1, x.length)
    L0 = levels[-1]
    start = (L - L0) >> 6
    x0 = x >> (32 * start)
    y, res = divmod(1 << L0, x0)                   # GMP base case, :1237-1253
    res_len = nlimbs(res)
    for i in range(len(levels) - 1, 0, -1):
        L1, L2 = levels[i], levels[i - 1]
        m = (L2 - L1) >> 1
        off2 = (L - L2) >> 6
        off1 = (L - L1) >> 6
        x2_len = min(m >> 5, x_len - off2)
        x2 = (x >> (32 * off2)) & ((1 << (32 * x2_len)) - 1)
        y1_len = y_len - off1
        x2y1 = x2 * y
        r1m_len = res_len + (m >> 5) + 1
        v = mod_limbs((res << m) - x2y1, r1m_len)
        neg = (v >> (32 * (r1m_len - 1))) >= 0x80000000
        if neg:
            v = mod_limbs(-v, r1m_len)
        res2 = v * y
        res2_len = r1m_len + y1_len
        sh = L2 - 2 * m
        y2_len = res2_len - (sh >> 5)
        y2 = mod_limbs(res2 >> sh, y2_len)
        if neg:
            y2 = mod_limbs(y2 + 1, y2_len)
        ynew_len = y_len - off2
        y = mod_limbs((y << m) - y2 if neg else (y << m) + y2, ynew_len)
        if L2 != L:
            xn = x >> (32 * off2)
            res_full_len = r1m_len + (m >> 5)
            resv = v << m
            y2x = y2 * xn
            res = mod_limbs(y2x - resv if neg else resv - y2x, res_full_len)
            res_len = nlimbs(res)
        del x2y1
    return y


# ---------------------------------------------------------------------------
# pi_fractional (pi_bs_gpu.cu:1524-1685)
# ---------------------------------------------------------------------------

def series_blocks(target_digits: int) -> int:
    """N of pi_fractional (pi_bs_gpu.cu:1537-1541)."""
    N = 1
    while N * 17 * 14.3 < target_digits:
        N *= 2
    return N


def prec_limbs_for(target_digits: int) -> int:
    """pi_bs_gpu.cu:1542 and compute_prec_limbs_for_digits :941-944."""
    return (int(target_digits * 3.322) + 31) // 32 + 1


@dataclass
class PiResult:
    ret: int            # RET value
    ret_len: int        # RET.length after compact
    digits: str         # convert_digits decimal digits after the point
    convert_digits: int
    leaf_digits: int


def pi_fractional(target_digits: int) -> tuple[int, int]:
    """RET value and RET limb length."""
    N = series_blocks(target_digits)
    prec = prec_limbs_for(target_digits)
    Q, R = binary_split(N)
    rshift = 15 * N * 17 - 8
    Rs = R >> rshift
    extra = max(0, min(nlimbs(Q), nlimbs(Rs)) - prec)
    Qt = Q >> (32 * extra)
    Rt = Rs >> (32 * extra)
    P15, Q15 = sqrt_10005(target_digits)
    Pf = P15 * Qt
    Qf = Rt * Q15
    extra = max(0, min(nlimbs(Pf), nlimbs(Qf)) - prec)
    Pt = Pf >> (32 * extra)
    Qtt = Qf >> (32 * extra)
    qbits = Qtt.bit_length()
    L = 2 * qbits - 1
    inv = recursive_inverse(Qtt, nlimbs(Qtt), L)
    ret = Pt * inv
    final_shift = L - 32 * prec
    ret = ret >> final_shift
    return ret, nlimbs(ret)


# ---------------------------------------------------------------------------
# Decimal conversion (convert_decimal.cu, batch_decimal_naive.cu)
# ---------------------------------------------------------------------------

def round_up_decimal_digits(requested: int) -> tuple[int, int]:
    """(leaf_digits, convert_digits) of pi_bs_gpu.cu:924-939."""
    if requested == 0:
        return 0, 0
    digits, levels = requested, 0
    while digits >= 32 * 18:
        digits >>= 1
        levels += 1
    if (digits << levels) < requested:
        digits += 1
    return digits, digits << levels


def bits_for_digits(d: int) -> int:
    """convert_decimal.cu:36-39 (host double arithmetic, same IEEE result)."""
    import math
    return int(math.ceil(d * LOG2_10) + PRECISION_MARGIN_BITS)


def leaf_decimal(x: int, l_limb: int, l_dec: int) -> str:
    """Truncated decimal digits of x / 2^(32 l_limb), most significant first
    (batch_decimal_naive.cu:16-176 followed by assemble_decimal_output_kernel,
    convert_decimal.cu:119-136)."""
    v = (x * 10 ** l_dec) >> (32 * l_limb)
    s = str(v)
    return s.rjust(l_dec, "0")[-l_dec:]


def convert_decimal(value: int, value_len: int, input_bits: int,
                    total_digits: int, leaf_digits: int) -> str:
    """convert_decimal_equal_split (convert_decimal.cu:285-474) on one row."""
    ratio = total_digits // leaf_digits
    levels = ratio.bit_length() - 1
    assert leaf_digits << levels == total_digits
    bits = [input_bits] + [0] * levels
    digs = [total_digits] + [0] * levels
    limbs = [value_len] + [0] * levels
    for lv in range(1, levels + 1):
        digs[lv] = digs[lv - 1] >> 1
        bits[lv] = bits_for_digits(digs[lv])
        limbs[lv] = (bits[lv] + 31) // 32
    if levels == 0:
        need = bits_for_digits(total_digits)
        nl = (need + 31) // 32
        cur = [mod_limbs(value >> (input_bits - need), nl)]
        cur_len = nl
        leaf_bits = need
    else:
        cur = [value]
        cur_len = value_len
        for lv in range(levels):
            d = digs[lv + 1]
            cb = bits[lv + 1]
            nl = limbs[lv + 1]
            B = bits[lv]
            mant_bits = B - d
            mant_len = (mant_bits + 31) // 32
            power = 5 ** d
            nxt = []
            for x in cur:
                x = mod_limbs(x, cur_len)
                hi = mod_limbs(x >> (B - cb), nl)
                mant = x & ((1 << mant_bits) - 1)
                assert nlimbs(mant) <= mant_len
                prod = mant * power
                lo = mod_limbs(prod >> (mant_bits - cb), nl)
                nxt.append(hi)
                nxt.append(lo)
            cur = nxt
            cur_len = nl
        leaf_bits = bits[levels]
    align = cur_len * 32 - leaf_bits
    out = []
    for x in cur:
        xa = mod_limbs(x << align, cur_len)
        out.append(leaf_decimal(xa, cur_len, leaf_digits))
    return "".join(out)


def pi_digits(target_digits: int) -> PiResult:
    """Full pipeline of main_fractional (pi_bs_gpu.cu:2073-2431)."""
    leaf, conv = round_up_decimal_digits(target_digits)
    prec = prec_limbs_for(target_digits)
    ret, ret_len = pi_fractional(target_digits)
    if target_digits == 0:
        return PiResult(ret, ret_len, "", 0, 0)
    frac_len = min(prec, ret_len)
    frac = mod_limbs(ret, frac_len)
    digits = convert_decimal(frac, frac_len, prec * 32, conv, leaf)
    return PiResult(ret, ret_len, digits, conv, leaf)


# ---------------------------------------------------------------------------
# Output helpers (pi_bs_gpu.cu:852-896)
# ---------------------------------------------------------------------------

def mod_hash(limbs) -> int:
    """compute_mod_hash, pi_bs_gpu.cu:852-858."""
    base = (1 << 32) % VALIDATION_MOD
    v = 0
    for w in reversed(list(limbs)):
        v = (v * base + int(w)) % VALIDATION_MOD
    return v


def decimal_hash(digits: str) -> int:
    """compute_decimal_hash, pi_bs_gpu.cu:860-866."""
    v = 3
    for ch in digits:
        v = (v * 10 + (ord(ch) - 48)) % VALIDATION_MOD
    return v


def hex_preview(label: str, limbs) -> str:
    """print_hex_preview_with_hash, pi_bs_gpu.cu:868-896."""
    limbs = list(limbs)
    length = len(limbs)
    h = mod_hash(limbs)
    if length == 0:
        return f"{label} = 0 hash = {h}"
    first_count = min(length, 2)
    last_count = min(length, 2)
    s = f"{label} = "
    for i in range(last_count):
        idx = length - 1 - i
        s += f"{limbs[idx]:x}" if i == 0 else f"{limbs[idx]:08x}"
    if length > first_count + last_count:
        s += "..."
    for i in range(first_count, 0, -1):
        idx = i - 1
        if length <= first_count + last_count and idx >= length - last_count:
            continue
        s += f"{limbs[idx]:08x}"
    return s + f" hash = {h}"


if __name__ == "__main__":
    import sys
    d = int(sys.argv[1]) if len(sys.argv) > 1 else 1000
    r = pi_digits(d)
    limbs = to_limbs(r.ret, r.ret_len)
    print(hex_preview("RET", limbs))
    print("3" + r.digits[:d])
