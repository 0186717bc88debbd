"""CPU tests of the oracle itself (no GPU): the restatement is pinned against
mpmath's pi, the committed golden fixtures, the reference's conversion test
cases (exact digits for generic inputs) and its own batch-op semantics."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

import batch_ref as ref
import pi_ref

GOLDEN = json.loads((Path(__file__).parent / "golden" / "pi_golden.json").read_text())


def _true_pi(n):
    import mpmath
    mpmath.mp.dps = n + 40
    return mpmath.nstr(mpmath.pi, n + 30, strip_zeros=False).replace(".", "")[1:n + 1]


@pytest.mark.parametrize("d", [1, 2, 9, 10, 99, 575, 576, 577, 1151, 2000, 12345])
def test_restatement_gives_pi(d):
    assert pi_ref.pi_digits(d).digits[:d] == _true_pi(d)


@pytest.mark.parametrize("entry", [e for e in GOLDEN["runs"] if e["digits"] <= 100000], ids=lambda e: str(e["digits"]))
def test_golden_fixture(entry):
    r = pi_ref.pi_digits(entry["digits"])
    limbs = pi_ref.to_limbs(r.ret, r.ret_len)
    assert r.ret_len == entry["ret_len"]
    assert pi_ref.mod_hash(limbs) == entry["ret_hash"]
    assert pi_ref.hex_preview("RET", limbs) == entry["ret_preview"]
    dec = r.digits[:entry["digits"]]
    assert hashlib.sha256(dec.encode()).hexdigest() == entry["dec_sha256"]


def test_sizes_of_the_1e9_configuration():
    """Shapes quoted for 1e9 digits: N = 2^22 blocks, leaf 477 x 2^21 and
    prec_limbs 103,812,501 (the conversion benchmark of
    convert_decimal_test.cu:33 uses prec_limbs + 1 = 103,812,502 limbs)."""
    assert pi_ref.series_blocks(10 ** 9) == 1 << 22
    assert pi_ref.round_up_decimal_digits(10 ** 9) == (477, 477 << 21)
    assert pi_ref.prec_limbs_for(10 ** 9) + 1 == 103812502
    assert pi_ref.series_blocks(10 ** 6) == 8192
    assert pi_ref.round_up_decimal_digits(10 ** 6) == (489, 489 << 11)


def test_inverse_spec_small():
    """recursive_inverse yields floor(2^L/x) or one below it for random x
    above the host base-case limit."""
    import random
    rnd = random.Random(5)
    for bits in (40000, 70000, 140000):
        x = rnd.getrandbits(bits) | (1 << (bits - 1))
        L = 2 * bits - 1
        y = pi_ref.recursive_inverse(x, pi_ref.nlimbs(x), L)
        assert 0 <= (1 << L) // x - y <= 2


def _xorshift_words(n, seed, bits):
    state = seed or 1
    M = (1 << 64) - 1
    words = []
    for _ in range(n):
        state ^= state >> 12
        state ^= (state << 25) & M
        state ^= state >> 27
        words.append(((state * 2685821657736338717) & M) >> 32)
    extra = bits & 31
    if extra:
        words[-1] &= (1 << extra) - 1
    return words


@pytest.mark.parametrize("digits,seed", [(477, 0x1234), (954, 0x2345), (1908, 0x3456), (3816, 0x4567)])
def test_convert_matches_exact_digits(digits, seed):
    """convert_decimal_test.cu:301-304: for these seeded fractions the
    equal-split conversion equals the exact truncated expansion."""
    bits = pi_ref.bits_for_digits(digits) + 64
    limbs = (bits + 31) // 32
    words = _xorshift_words(limbs, seed, bits)
    x = pi_ref.from_limbs(words)
    exact = str((x * 10 ** digits) >> bits).rjust(digits, "0")
    assert pi_ref.convert_decimal(x, limbs, bits, digits, 477) == exact


def test_batch_ref_semantics():
    rng = np.random.default_rng(1)
    A = rng.integers(0, 1 << 32, 20, dtype=np.uint64).astype(np.uint32)
    B = rng.integers(0, 1 << 32, 20, dtype=np.uint64).astype(np.uint32)
    C = np.zeros(30, dtype=np.uint32)
    s = ref.add(2, A, 10, 10, B, 10, 10, C, 11, 15)
    for r in range(2):
        assert ref.row_int(s, r, 11, 15) == ref.row_int(A, r, 10, 10) + ref.row_int(B, r, 10, 10)
    d = ref.sub(1, A, 3, 3, B, 5, 5, C, 4, 4)
    assert ref.row_int(d, 0, 4, 4) == (ref.row_int(A, 0, 3, 3) - ref.row_int(B, 0, 5, 5)) % (1 << 128)
    q = ref.exactdiv_small(1, np.array([15, 0], dtype=np.uint32), 2, 2, 5)
    assert list(q) == [3, 0]
    out = ref.decimal_naive(1, np.array([1 << 31], dtype=np.uint32), 1, 1, 6, 6, bytearray(6))
    assert bytes(out) == b"000005"   # 1/2 -> "500000" written least significant first


def test_cpp_restatement_matches_python():
    """The host C++ restatement (oracle/pi_cpu.cpp, GMP, threads) prints the
    same RET preview, hash and digits as the Python restatement."""
    import subprocess
    import build_cpu
    exe = build_cpu.build()
    for d in (0, 100, 20000):
        out = subprocess.run([str(exe), str(d)], capture_output=True, text=True, check=True).stdout.splitlines()
        r = pi_ref.pi_digits(d)
        limbs = pi_ref.to_limbs(r.ret, r.ret_len)
        assert f"RET_len={r.ret_len}" in out[0]
        assert out[1] == pi_ref.hex_preview("RET", limbs)
        if d:
            assert out[2] == "DEC = 3" + r.digits[:min(63, d)] + "..." + r.digits[d - min(64, d):d]
