"""End-to-end parity of the pi pipeline (pi_bs_gpu main_fractional) against
the CPU restatement (RET limbs and every digit) and the committed golden
fixtures (RET hash / length, digit hashes) up to 1e6 digits."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

import pi_ref

pytestmark = pytest.mark.gpu

GOLDEN = json.loads((Path(__file__).parent / "golden" / "pi_golden.json").read_text())


@pytest.mark.parametrize("digits", [0, 1, 10, 100, 575, 576, 1000, 5000, 20000, 100000])
def test_pi_matches_oracle(ctx, digits):
    import gpupi_b200 as g
    r = g.pi_compute(digits, ctx)
    want = pi_ref.pi_digits(digits)
    assert r.ret_len == want.ret_len
    assert np.array_equal(r.ret, np.array(pi_ref.to_limbs(want.ret, want.ret_len), dtype=np.uint32))
    assert r.convert_digits == want.convert_digits
    assert r.dec == want.digits[:digits]


@pytest.mark.parametrize("entry", GOLDEN["runs"], ids=lambda e: str(e["digits"]))
def test_pi_golden(ctx, entry):
    import gpupi_b200 as g
    d = entry["digits"]
    r = g.pi_compute(d, ctx)
    assert r.ret_len == entry["ret_len"]
    assert pi_ref.mod_hash(r.ret) == entry["ret_hash"]
    assert r.convert_digits == entry["convert_digits"]
    assert hashlib.sha256(r.dec.encode()).hexdigest() == entry["dec_sha256"]
    assert pi_ref.decimal_hash(r.dec[:4096]) == entry["dec_preview_hash"]


@pytest.mark.parametrize("digits", [1000, 1000000])
def test_pi_into_pinned_buffers(ctx, digits):
    """RET and the digits copied straight into caller-owned pinned buffers
    (RET on a side stream while the digits are converted) match the default path."""
    import torch
    import gpupi_b200 as g
    want = g.pi_compute(digits, ctx)
    hd = torch.zeros(digits, dtype=torch.uint8, pin_memory=True)
    hr = torch.zeros(g.ret_limbs_bound(digits), dtype=torch.int32, pin_memory=True)
    r = g.pi_compute(digits, ctx, host_digits=hd, host_ret=hr)
    assert r.ret_len == want.ret_len
    assert np.array_equal(r.ret, want.ret)
    assert bytes(hd.numpy()).decode() == want.dec


def test_pi_1e7_matches_cpp_restatement(ctx):
    """10^7 digits: RET and every digit equal the host C++ restatement
    (oracle/pi_cpu.cpp, GMP), built on the spot with g++."""
    import subprocess
    import build_cpu
    import gpupi_b200 as g
    d = 10_000_000
    out = subprocess.run([str(build_cpu.build()), str(d)], capture_output=True, text=True,
                         check=True).stdout.splitlines()
    r = g.pi_compute(d, ctx)
    assert f"RET_len={r.ret_len}" in out[0]
    assert out[1] == pi_ref.hex_preview("RET", r.ret)
    assert out[3] == f"DEC_hash = {pi_ref.decimal_hash(r.dec)}"


def test_scratch_arena_reaches_steady_state(ctx):
    """Repeating one computation settles the scratch arena: after the first
    calls the temporaries fit its block (no request served outside it), and
    every repeat gives the same RET and digits."""
    import gpupi_b200 as g
    d = 300_000
    first = g.pi_compute(d, ctx)
    g.pi_compute(d, ctx)
    s0 = g.scratch_stats()
    r = g.pi_compute(d, ctx)
    s1 = g.scratch_stats()
    assert s1["spills"] == s0["spills"]
    assert s1["block_bytes"] > 0 and s1["high_water"] > 0
    assert np.array_equal(r.ret, first.ret)
    assert r.dec == first.dec


@pytest.mark.parametrize("digits", [20000, 300000, 3000000])
def test_plain_and_tuned_forms_agree(ctx, digits):
    """The plain form (the reference's op sequence) and the default tuned form
    (forward transforms shared within each merge level) produce the same RET
    and digits."""
    import gpupi_b200 as g
    tuned = g.pi_compute(digits, ctx)
    plain = g.pi_compute(digits, ctx, plain=True)
    assert tuned.ret_len == plain.ret_len
    assert np.array_equal(tuned.ret, plain.ret)
    assert tuned.dec == plain.dec


def test_pi_beyond_the_reference_ceiling(ctx):
    """1.2e9 digits: the splitting tree for 2^23 x 17 terms, whose top
    products (about 5.5e8 limbs) exceed the reference's 2^28-limb NTT ceiling
    and run on 17 cosets.  Its digits must agree with the 1e9-digit run on the
    first 1e9 - 64 digits, and RET with BBP at seeded positions."""
    import random
    import gpupi_b200 as g
    small = g.pi_compute(1_000_000_000, ctx)
    big = g.pi_compute(1_200_000_000, ctx)
    n = 1_000_000_000 - 64
    assert big.dec[:n] == small.dec[:n]
    assert big.ret_len > small.ret_len
    rng = random.Random(0x12E9)
    top = 8 * (big.ret_len - 1) - 64
    positions = sorted(rng.randrange(0, min(top, 1 << 30)) for _ in range(8))
    bad, unsure = g.bbp_spot_check(big.ret, positions)
    assert not bad and not unsure


def test_streamed_digits(ctx, tmp_path):
    """Streamed output (chunked device-to-host copies overlapping the writes):
    the chunks concatenate to the digits, a False return stops, and the file
    helper writes the CLI's "3<digits>\\n"."""
    import gpupi_b200 as g
    d = 100000
    want = g.pi_compute(d, ctx).dec
    chunks = []
    g.pi_stream(d, chunks.append, ctx, chunk=4096)
    assert len(chunks) == (d + 4095) // 4096
    assert b"".join(chunks).decode() == want
    first = []
    g.pi_stream(d, lambda b: (first.append(b), False)[1], ctx, chunk=4096)
    assert first == [want[:4096].encode()]
    path = tmp_path / "pi.txt"
    g.pi_to_file(d, path, ctx, chunk=10000)
    assert path.read_text() == "3" + want + "\n"


def test_cli_output_modes(tmp_path):
    """The CLI streams its digits: default mode prints the result line on
    stderr before "3<digits>" on stdout (as the reference orders them),
    --output FILE writes the same bytes to a file, --full-print is unchanged."""
    import subprocess
    cli = str(Path(__file__).resolve().parents[1] / "gpupi_b200" / "pi_bs_gpu")
    d = 100000
    want = "3" + pi_ref.pi_digits(d).digits[:d] + "\n"
    r = subprocess.run([cli, str(d)], capture_output=True, text=True, check=True)
    assert r.stdout == want
    assert r.stderr.startswith(f"target_digits={d} convert_digits=")
    merged = subprocess.run([cli, str(d)], stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True,
                            check=True).stdout
    assert merged.startswith(f"target_digits={d} ") and merged.endswith(want)
    path = tmp_path / "pi.txt"
    r = subprocess.run([cli, str(d), "--output", str(path)], capture_output=True, text=True, check=True)
    assert r.stdout == "" and path.read_text() == want
    assert f"output={path} bytes={d + 2}" in r.stderr
    r = subprocess.run([cli, "1000", "--full-print"], capture_output=True, text=True, check=True)
    # the DEC line, then the reference's closing newline (pi_bs_gpu.cu:2401-2423)
    assert r.stdout.endswith("DEC = 3" + pi_ref.pi_digits(1000).digits[:1000] + "\n\n")


def test_checkpoint_of_the_tree(ctx, tmp_path):
    """The splitting tree's result saved to a checkpoint and loaded back gives
    the same RET and digits; a corrupted, truncated or other-size checkpoint
    is not used (the tree runs and the file is rewritten)."""
    import gpupi_b200 as g
    d = 300_000
    want = g.pi_compute(d, ctx)
    ck = tmp_path / "tree.ckpt"
    a = g.pi_compute(d, ctx, checkpoint=ck)
    assert a.checkpoint_state == 2 and ck.exists()
    b = g.pi_compute(d, ctx, checkpoint=ck)
    assert b.checkpoint_state == 1
    for r in (a, b):
        assert np.array_equal(r.ret, want.ret) and r.dec == want.dec
    raw = bytearray(ck.read_bytes())
    raw[len(raw) // 2] ^= 1
    ck.write_bytes(bytes(raw))
    c = g.pi_compute(d, ctx, checkpoint=ck)
    assert c.checkpoint_state == 2 and c.dec == want.dec
    assert g.pi_compute(d, ctx, checkpoint=ck).checkpoint_state == 1
    ck.write_bytes(ck.read_bytes()[:-4])
    assert g.pi_compute(d, ctx, checkpoint=ck).checkpoint_state == 2
    small = g.pi_compute(20_000, ctx, checkpoint=ck)   # another tree size
    assert small.checkpoint_state == 2 and small.dec == g.pi_compute(20_000, ctx).dec
    # a checkpoint that cannot be written does not fail the computation
    nowhere = tmp_path / "missing-dir" / "tree.ckpt"
    e = g.pi_compute(d, ctx, checkpoint=nowhere)
    assert e.checkpoint_state == 3 and not nowhere.exists()
    assert np.array_equal(e.ret, want.ret) and e.dec == want.dec


def test_cli_checkpoint(tmp_path):
    import subprocess
    cli = str(Path(__file__).resolve().parents[1] / "gpupi_b200" / "pi_bs_gpu")
    ck = tmp_path / "tree.ckpt"
    r1 = subprocess.run([cli, "100000", "--checkpoint", str(ck)], capture_output=True, text=True, check=True)
    r2 = subprocess.run([cli, "100000", "--checkpoint", str(ck)], capture_output=True, text=True, check=True)
    assert f"checkpoint={ck} written" in r1.stderr and f"checkpoint={ck} loaded" in r2.stderr
    assert r1.stdout == r2.stdout == "3" + pi_ref.pi_digits(100000).digits[:100000] + "\n"
