"""Generate tests/golden/pi_golden.json from the CPU restatement.

Each run records what pi_bs_gpu prints or can be checked against: RET limb
count and its mod-(1e9+7) hash (pi_bs_gpu.cu:852-858), convert_digits, the
DEC preview hash over the first 4096 digits (:860-866), the --benchmark
prefix/suffix and a SHA-256 of all requested digits.  The digits themselves
are also checked against mpmath's pi here, independently of the reference
algorithm (the restatement must produce true pi digits).

    python tests/golden/make_golden.py
"""
import hashlib
import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent / "oracle"))
import pi_ref  # noqa: E402

DIGITS = [1, 10, 100, 575, 576, 1000, 10000, 100000, 1000000]


def true_pi_digits(n: int) -> str:
    import mpmath
    mpmath.mp.dps = n + 40
    return mpmath.nstr(mpmath.pi, n + 30, strip_zeros=False).replace(".", "")[1:n + 1]


def main() -> None:
    runs = []
    for d in DIGITS:
        r = pi_ref.pi_digits(d)
        dec = r.digits[:d]
        assert dec == true_pi_digits(d), f"restatement disagrees with pi at {d} digits"
        runs.append({
            "digits": d,
            "convert_digits": r.convert_digits,
            "leaf_digits": r.leaf_digits,
            "ret_len": r.ret_len,
            "ret_hash": pi_ref.mod_hash(pi_ref.to_limbs(r.ret, r.ret_len)),
            "ret_preview": pi_ref.hex_preview("RET", pi_ref.to_limbs(r.ret, r.ret_len)),
            "dec_prefix": "3" + dec[:63],
            "dec_suffix": dec[-64:],
            "dec_preview_hash": pi_ref.decimal_hash(dec[:4096]),
            "dec_sha256": hashlib.sha256(dec.encode()).hexdigest(),
        })
        print(runs[-1]["ret_preview"], d, flush=True)
    out = {"generator": "tests/golden/make_golden.py (oracle/pi_ref.py, checked against mpmath)",
           "runs": runs}
    (HERE / "pi_golden.json").write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    main()
