"""The tensor-core schoolbook (tcgen05 kind::i8 split-integer products,
csrc/mul_tc.cu) against exact Python integers and against the CUDA-core
schoolbook (gpupi batch_mul_naive's operation): bit for bit, over the
shapes the kernel handles (min(L_a, L_b) <= 2048, L_a + L_b <= 8192),
uneven and broadcast operands, padded strides, all-ones operands (largest
byte sums in the INT32 accumulators and the longest carry chains) and
repeated calls (the kernel's completion waits never ran out)."""
import numpy as np
import pytest

import batch_ref as ref
from helpers import rand_buf, to_dev

pytestmark = pytest.mark.gpu


def _run(N, La, Lb, sA, sB, sC, rng, fill="random", path="tc"):
    import gpupi_b200 as g
    A = rand_buf(rng, N, sA, La) if sA else rand_buf(rng, 1, La, La)
    B = rand_buf(rng, N, sB, Lb) if sB else rand_buf(rng, 1, Lb, Lb)
    C = rand_buf(rng, N, sC, 0)
    if fill == "ones":
        for r in range(N):
            A[r * sA: r * sA + La] = 0xFFFFFFFF
            B[r * sB: r * sB + Lb] = 0xFFFFFFFF
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C)
    if path == "tc":
        g.mul_tc(N, dA.ptr, La, sA, dB.ptr, Lb, sB, dC.ptr, sC)
    else:
        g.mul_naive(N, dA.ptr, La, sA, dB.ptr, Lb, sB, dC.ptr, sC)
    got = dC.numpy()
    assert g.tc_error() == 0
    return A, B, C, got


SHAPES = [(1, 1), (1, 7), (3, 4), (8, 8), (16, 16), (17, 33), (31, 32), (32, 32), (33, 95), (64, 64),
          (100, 300), (128, 128), (224, 224), (255, 257), (447, 1), (512, 512), (1000, 24), (24, 1000),
          (1024, 1024), (2048, 2048), (2048, 6144), (1, 8191), (3000, 1500)]


@pytest.mark.parametrize("La,Lb", SHAPES)
def test_tc_matches_exact_product(La, Lb):
    rng = np.random.default_rng(La * 7919 + Lb)
    N = 37 if La + Lb <= 256 else 5
    sA, sB, sC = La + 3, Lb + 1, La + Lb + 2
    A, B, C, got = _run(N, La, Lb, sA, sB, sC, rng)
    assert np.array_equal(got, ref.mul(N, A, La, sA, B, Lb, sB, C, sC))
    A, B, C, got = _run(2, La, Lb, La, Lb, La + Lb, rng, fill="ones")
    assert np.array_equal(got, ref.mul(2, A, La, La, B, Lb, Lb, C, La + Lb))


@pytest.mark.parametrize("La,Lb", [(5, 9), (64, 64), (300, 200), (511, 513)])
def test_tc_equals_cuda_core_schoolbook(La, Lb):
    """Same inputs through both schoolbook paths: identical words, padding included."""
    rng = np.random.default_rng(La + 31 * Lb)
    N, sA, sB, sC = 64, La + 1, Lb + 5, La + Lb + 4
    r1 = _run(N, La, Lb, sA, sB, sC, np.random.default_rng(1 + La), path="tc")[3]
    r2 = _run(N, La, Lb, sA, sB, sC, np.random.default_rng(1 + La), path="naive")[3]
    assert np.array_equal(r1, r2)
    del rng


def test_tc_broadcast_operand():
    """stride 0: one B row multiplies every A row (the conversion's 5^d)."""
    rng = np.random.default_rng(9)
    N, La, Lb = 40, 200, 77
    A, B, C, got = _run(N, La, Lb, La, 0, La + Lb, rng)
    assert np.array_equal(got, ref.mul(N, A, La, La, B, Lb, 0, C, La + Lb))


def test_tc_rejects_out_of_range_shapes():
    import gpupi_b200 as g
    import torch
    buf = torch.zeros(1 << 15, dtype=torch.int32, device="cuda")
    p = buf.data_ptr()
    for La, Lb in [(0, 5), (5, 0), (2049, 2049), (4096, 4097)]:
        with pytest.raises(g.GpupiError):
            g.mul_tc(1, p, La, La, p, Lb, Lb, p, La + Lb)
