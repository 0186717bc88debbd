"""The tune table honoured on the GPU: whatever kernel or transform shape
it names, the products are bit-identical; the kernel families that ran show
the table was followed (per-launch timers).  gpupi_autotune measures,
checks and writes a table that then drives a bit-exact pi run."""
import json
from pathlib import Path

import numpy as np
import pytest

import batch_ref as ref
from helpers import to_dev

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(autouse=True)
def _restore_table():
    import gpupi_b200 as g
    yield
    g.tune_reset()
    if g.TUNE_TABLE_PATH.exists():
        g.tune_load(g.TUNE_TABLE_PATH)


def _families(fn):
    import gpupi_b200 as g
    g.timer_reset()
    g.timer_enable(True)
    fn()
    g.timer_enable(False)
    fams = set(g.timer_report())
    g.timer_reset()
    return fams


def _offsets(L):
    return np.concatenate([[0], np.cumsum(L.astype(np.uint64))[:-1]]).astype(np.uint64)


def _ragged_case(rng, n=300):
    La = rng.integers(17, 700, size=n).astype(np.uint32)
    Lb = rng.integers(17, 700, size=n).astype(np.uint32)
    A = rng.integers(0, 1 << 32, size=int(La.sum()), dtype=np.uint64).astype(np.uint32)
    B = rng.integers(0, 1 << 32, size=int(Lb.sum()), dtype=np.uint64).astype(np.uint32)
    return La, Lb, A, B


@pytest.mark.parametrize("kind,family", [("school", "schoolbook"), ("tc", "schoolbook_tc"), ("ntt", "ntt_local")])
def test_table_kernel_is_honoured_and_exact(ctx, kind, family):
    import gpupi_b200 as g
    rng = np.random.default_rng(42)
    La, Lb, A, B = _ragged_case(rng)
    Lc = La.astype(np.uint64) + Lb
    offA, offB, offC = _offsets(La), _offsets(Lb), _offsets(Lc)
    g.tune_load(text=f"mul 1024 {kind}\n")
    dA, dB, dC = to_dev(A), to_dev(B), g.DeviceLimbs(int(Lc.sum()))
    fams = _families(lambda: ctx.mul_ragged(dA.ptr, offA, La, dB.ptr, offB, Lb, dC.ptr, offC))
    assert family in fams
    got = dC.numpy()
    for i in range(0, len(La), 37):
        oa, ob, oc = int(offA[i]), int(offB[i]), int(offC[i])
        a = int.from_bytes(A[oa:oa + int(La[i])].tobytes(), "little")
        b = int.from_bytes(B[ob:ob + int(Lb[i])].tobytes(), "little")
        c = int.from_bytes(got[oc:oc + int(Lc[i])].tobytes(), "little")
        assert c == a * b


def test_all_tables_give_identical_products(ctx):
    import gpupi_b200 as g
    rng = np.random.default_rng(7)
    La, Lb, A, B = _ragged_case(rng, 500)
    Lc = La.astype(np.uint64) + Lb
    offA, offB, offC = _offsets(La), _offsets(Lb), _offsets(Lc)
    dA, dB = to_dev(A), to_dev(B)
    outs = []
    for text in ["mul 1024 school\n", "mul 1024 tc\n", "mul 1024 ntt\n", "mul 300 school\nmul 700 tc\n"]:
        g.tune_load(text=text)
        dC = g.DeviceLimbs(int(Lc.sum()))
        ctx.mul_ragged(dA.ptr, offA, La, dB.ptr, offB, Lb, dC.ptr, offC)
        outs.append(dC.numpy())
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])


def test_table_ntt_shape_is_honoured(ctx):
    """A product of 2 x 5000 limbs: the built-in 2^14-point transform, or two
    cosets of 2^13 points as the table says (the coset-combination kernel
    runs); same words either way."""
    import gpupi_b200 as g
    rng = np.random.default_rng(3)
    N, La, Lb = 3, 5000, 5000
    A = rng.integers(0, 1 << 32, size=N * La, dtype=np.uint64).astype(np.uint32)
    B = rng.integers(0, 1 << 32, size=N * Lb, dtype=np.uint64).astype(np.uint32)
    dA, dB = to_dev(A), to_dev(B)
    res = []
    for text, coset in [("", False), ("ntt 9000 10000 13 2\n", True)]:
        g.tune_reset()
        if text:
            g.tune_load(text=text)
        assert g.ntt_shape(La, Lb) == ((13, 2) if coset else (14, 1))
        dC = g.DeviceLimbs(N * (La + Lb))
        fams = _families(lambda: ctx.mul(N, dA.ptr, La, La, dB.ptr, Lb, Lb, dC.ptr, La + Lb, La + Lb))
        assert ("ntt_coset_combine" in fams) == coset
        res.append(dC.numpy())
    assert np.array_equal(res[0], res[1])
    C = np.zeros(N * (La + Lb), dtype=np.uint32)
    assert np.array_equal(res[0], ref.mul(N, A, La, La, B, Lb, Lb, C, La + Lb))


def test_autotune_writes_a_table_that_keeps_pi_exact(ctx, tmp_path):
    import gpupi_b200 as g
    path = tmp_path / "tune.txt"
    text = g.autotune(ctx, path, budget_limbs=1 << 20)
    assert text.count("\nmul ") >= 10 and "\nntt " in text
    assert "school=-2" not in text and "tc=-2" not in text   # no candidate disagreed
    fx = json.loads((ROOT / "tests" / "golden" / "ref_fixtures.json").read_text())["pi"][0]
    import pi_ref
    r = g.pi_compute(fx["digits"], ctx)
    assert r.ret_len == fx["ret_len"] and pi_ref.mod_hash(r.ret) == fx["ret_hash"]
