"""Parity with gpupi's own CUDA build (the reference), pinned by fixtures the
reference itself produced on a B200 (tests/golden/ref_fixtures.json, made by
oracle/make_ref_fixtures.py from oracle/_ref, built from the reference's
sources by oracle/build_ref.py).

* pi at 1e6 ... 1e9 digits through this library's CLI: the whole stdout
  ("3" + every digit + newline) has the reference's SHA-256, and the
  `--benchmark` lines (RET length, RET preview with its mod-1e9+7 hash, DEC
  preview) are the reference's, byte for byte;
* the benchmark configurations on the same seeded inputs (oracle/ref_inputs.py):
  C2, 4096 uneven products, through the ragged call (the reference multiplied
  them one call per pair); C3, one 2^27 x 2^27-limb product; C4, a 2^25-limb
  fraction to 322,961,408 digits: results bit-identical (SHA-256);
* when the reference build is present, a live run of it at 1e6 and 1e7 digits
  against this library's CLI, and the reference's own 15 test programs
  compiled against this library's headers and linked with it.
"""
import hashlib
import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

import ref_inputs

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
FIX = json.loads((ROOT / "tests" / "golden" / "ref_fixtures.json").read_text())
CLI = ROOT / "gpupi_b200" / "pi_bs_gpu"
REF = ROOT / "oracle" / "_ref"


def _stdout_sha(cmd):
    p = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE)
    h = hashlib.sha256()
    n = 0
    while True:
        chunk = p.stdout.read(1 << 24)
        if not chunk:
            break
        h.update(chunk)
        n += len(chunk)
    err = p.stderr.read().decode()
    assert p.wait(timeout=900) == 0, err
    return h.hexdigest(), n, err


@pytest.mark.parametrize("entry", FIX["pi"], ids=lambda e: str(e["digits"]))
def test_cli_matches_reference_build(entry):
    d = entry["digits"]
    sha, n, err = _stdout_sha([str(CLI), str(d)])
    assert n == entry["stdout_bytes"]
    assert sha == entry["stdout_sha256"]
    assert f"RET_len={entry['ret_len']}" in err and f"convert_digits={entry['convert_digits']}" in err
    bench = subprocess.run([str(CLI), str(d), "--benchmark"], capture_output=True, text=True, check=True)
    lines = bench.stdout.splitlines()
    assert lines[1] == entry["ret_line"]
    assert lines[2] == entry["dec_line"]


@pytest.mark.parametrize("plain", [False, True], ids=["tuned", "plain"])
def test_api_matches_reference_build(ctx, plain):
    """Both forms of the pipeline through the Python API at 1e7 digits."""
    import gpupi_b200 as g
    import pi_ref
    entry = next(e for e in FIX["pi"] if e["digits"] == 10_000_000)
    r = g.pi_compute(entry["digits"], ctx, plain=plain)
    assert r.ret_len == entry["ret_len"]
    assert pi_ref.mod_hash(r.ret) == entry["ret_hash"]
    assert hashlib.sha256(("3" + r.dec + "\n").encode()).hexdigest() == entry["stdout_sha256"]


def _device_u32(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def test_c2_uneven_products_match_reference_build(ctx):
    import torch
    fx = FIX["configs"]["c2"]
    La, Lb, A, B = ref_inputs.c2_inputs()
    Lc = La.astype(np.uint64) + Lb
    offA = np.concatenate([[0], np.cumsum(La.astype(np.uint64))[:-1]]).astype(np.uint64)
    offB = np.concatenate([[0], np.cumsum(Lb.astype(np.uint64))[:-1]]).astype(np.uint64)
    offC = np.concatenate([[0], np.cumsum(Lc)[:-1]]).astype(np.uint64)
    dA, dB = _device_u32(A), _device_u32(B)
    dC = torch.zeros(int(Lc.sum()), dtype=torch.int32, device="cuda")
    ctx.mul_ragged(dA.data_ptr(), offA, La, dB.data_ptr(), offB, Lb, dC.data_ptr(), offC)
    C = dC.cpu().numpy().view(np.uint32)
    assert ref_inputs.digest(C)["sha256"] == fx["sha256"]


def test_c3_large_product_matches_reference_build(ctx):
    import torch
    fx = FIX["configs"]["c3"]
    A, B = ref_inputs.c3_inputs(int(fx["args"][0]))
    L = A.size
    dA, dB = _device_u32(A), _device_u32(B)
    del A, B
    dC = torch.zeros(2 * L, dtype=torch.int32, device="cuda")
    ctx.mul(1, dA.data_ptr(), L, L, dB.data_ptr(), L, L, dC.data_ptr(), 2 * L, 2 * L)
    del dA, dB
    C = dC.cpu().numpy().view(np.uint32)
    assert ref_inputs.digest(C)["sha256"] == fx["sha256"]


def test_c4_conversion_matches_reference_build(ctx):
    import torch
    fx = FIX["configs"]["c4"]
    X = ref_inputs.c4_input()
    L = X.size
    leaf, levels = 308, 20
    total = leaf << levels
    dX = _device_u32(X)
    out = torch.zeros(total, dtype=torch.uint8, device="cuda")
    ctx.convert_decimal(dX.data_ptr(), L, 32 * L, total, leaf, out.data_ptr())
    digits = bytes(out.cpu().numpy())
    assert ref_inputs.digest(digits)["sha256"] == fx["sha256"]


@pytest.mark.skipif(not (REF / "pi_bs_gpu_ref").exists(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("digits", [1_000_000, 10_000_000])
def test_live_reference_build(digits):
    """The reference binary run here, now, against this library's CLI."""
    ours = _stdout_sha([str(CLI), str(digits)])
    ref = _stdout_sha([str(REF / "pi_bs_gpu_ref"), str(digits)])
    assert ours[:2] == ref[:2]
    b1 = subprocess.run([str(CLI), str(digits), "--benchmark"], capture_output=True, text=True, check=True)
    b2 = subprocess.run([str(REF / "pi_bs_gpu_ref"), str(digits), "--benchmark"], capture_output=True, text=True,
                        check=True)
    assert b1.stdout.splitlines()[1:] == b2.stdout.splitlines()[1:]


REF_TESTS = sorted(p.name[: -len("_on_gpupi_b200")] for p in REF.glob("*_test_on_gpupi_b200"))


@pytest.mark.skipif(not REF_TESTS, reason="reference tests not built (oracle/build_ref.py --tests)")
@pytest.mark.parametrize("name", REF_TESTS or ["none"])
def test_reference_test_program_on_this_library(name):
    """gpupi's own test program, compiled against include/ and linked with
    libgpupi_b200.so: it must exit 0 and report no failure."""
    r = subprocess.run([str(REF / f"{name}_on_gpupi_b200")], capture_output=True, text=True, timeout=900)
    out = r.stdout + r.stderr
    assert r.returncode == 0, out[-3000:]
    assert "FAILED" not in out and "FAIL:" not in out, out[-3000:]
    assert "PASS" in out, out[-3000:]
