"""The BBP fixed-point restatement (oracle/bbp_ref.py) against pi's hex digits
from the pipeline restatement's RET, and the host-side bit extraction and
comparison helpers of the BBP spot check."""
import numpy as np

import bbp_ref
import pi_ref


def _ret_limbs(digits):
    r = pi_ref.pi_digits(digits)
    return np.array(pi_ref.to_limbs(r.ret, r.ret_len), dtype=np.uint32)


def test_bbp_restatement_matches_ret():
    import gpupi_b200 as g
    ret = _ret_limbs(3000)          # ~311 limbs: hex digits up to ~2490
    assert g.ret_hex_bits(ret, 0, 32) == 0x243F6A88
    for n in list(range(0, 40)) + [97, 500, 1234, 2000]:
        f = bbp_ref.bbp_fraction(n)
        err = 8 * (n + 17)
        lo, hi = ((f - err) % (1 << 64)) >> 40, ((f + err) % (1 << 64)) >> 40
        if lo == hi:
            assert g.ret_hex_bits(ret, n, 24) == f >> 40, n


def test_ret_hex_bits_window():
    import gpupi_b200 as g
    ret = np.array([0x89ABCDEF, 0x01234567, 3], dtype=np.uint32)   # 3.0123456789ABCDEF (hex)
    assert g.ret_hex_bits(ret, 0, 8) == 0x01
    assert g.ret_hex_bits(ret, 1, 12) == 0x123
    assert g.ret_hex_bits(ret, 7, 8) == 0x78      # straddles the limb boundary
    assert g.ret_hex_bits(ret, 10, 24) == 0xABCDEF
