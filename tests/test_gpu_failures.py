"""Failure detection and error paths, with no GPU fault involved.

* The tensor-core kernel's bounded waits: a self-test CTA waits on a barrier
  that never completes; the wait runs out, the kernel records it in the
  library's device error word and returns, and the next product is exact
  (the context and the GPU stay usable).
* Allocation failures injected on the host (gpupi_fail_alloc): the n-th
  scratch-arena request of a pi computation, a decimal conversion or a ragged
  batch, or a context's workspace growth, fails with cudaErrorMemoryAllocation
  (2); the error reaches the caller, every scratch byte handed out is
  returned (no leak), and the same call then succeeds with the exact result.
  The reference returns cudaError_t the same way (pi_bs_gpu.cu:493-501) but
  leaves some allocations unchecked (:1199-1203).
"""
import hashlib

import numpy as np
import pytest

import batch_ref as ref
from helpers import to_dev

pytestmark = pytest.mark.gpu


def test_tc_wait_timeout_is_reported_and_the_gpu_stays_usable():
    import gpupi_b200 as g
    seen, after = g.tc_selftest_timeout()
    assert seen == 2 and after == 0
    rng = np.random.default_rng(5)
    La = Lb = 300
    A = rng.integers(0, 1 << 32, size=4 * La, dtype=np.uint64).astype(np.uint32)
    B = rng.integers(0, 1 << 32, size=4 * Lb, dtype=np.uint64).astype(np.uint32)
    dA, dB, dC = to_dev(A), to_dev(B), g.DeviceLimbs(4 * (La + Lb))
    g.mul_tc(4, dA.ptr, La, La, dB.ptr, Lb, Lb, dC.ptr, La + Lb)
    C = np.zeros(4 * (La + Lb), dtype=np.uint32)
    assert np.array_equal(dC.numpy(), ref.mul(4, A, La, La, B, Lb, Lb, C, La + Lb))
    assert g.tc_error() == 0


@pytest.mark.parametrize("nth", [1, 2, 7, 25])
def test_scratch_failure_in_pi_propagates_without_leak(ctx, nth):
    import gpupi_b200 as g
    d = 100_000
    want = g.pi_compute(d, ctx)
    base = g.scratch_live_bytes()
    g.fail_alloc(g.ALLOC_SCRATCH, nth)
    with pytest.raises(g.GpupiError, match="cudaError 2"):
        g.pi_compute(d, ctx)
    g.fail_alloc(0, 0)
    assert g.scratch_live_bytes() == base
    again = g.pi_compute(d, ctx)
    assert np.array_equal(again.ret, want.ret) and again.dec == want.dec


@pytest.mark.parametrize("nth", [1, 3])
def test_scratch_failure_in_conversion_propagates_without_leak(ctx, nth):
    import gpupi_b200 as g
    rng = np.random.default_rng(11)
    L, leaf, levels = 4096, 308, 6
    X = to_dev(rng.integers(0, 1 << 32, size=L, dtype=np.uint64).astype(np.uint32))
    out = g.DeviceBytes(leaf << levels)
    ctx.convert_decimal(X.ptr, L, 32 * L, leaf << levels, leaf, out.ptr)
    want = out.text()
    base = g.scratch_live_bytes()
    g.fail_alloc(g.ALLOC_SCRATCH, nth)
    with pytest.raises(g.GpupiError, match="cudaError 2"):
        ctx.convert_decimal(X.ptr, L, 32 * L, leaf << levels, leaf, out.ptr)
    g.fail_alloc(0, 0)
    assert g.scratch_live_bytes() == base
    ctx.convert_decimal(X.ptr, L, 32 * L, leaf << levels, leaf, out.ptr)
    assert hashlib.sha256(out.text().encode()).digest() == hashlib.sha256(want.encode()).digest()


def test_workspace_growth_failure_leaves_the_context_usable():
    import gpupi_b200 as g
    c = g.Context()
    try:
        rng = np.random.default_rng(12)
        N, La, Lb = 2, 5000, 3000
        A = rng.integers(0, 1 << 32, size=N * La, dtype=np.uint64).astype(np.uint32)
        B = rng.integers(0, 1 << 32, size=N * Lb, dtype=np.uint64).astype(np.uint32)
        dA, dB, dC = to_dev(A), to_dev(B), g.DeviceLimbs(N * (La + Lb))
        g.fail_alloc(g.ALLOC_WORKSPACE, 1)
        with pytest.raises(g.GpupiError, match="cudaError 2"):
            c.mul(N, dA.ptr, La, La, dB.ptr, Lb, Lb, dC.ptr, La + Lb, La + Lb)
        g.fail_alloc(0, 0)
        assert c.workspace_size == 0
        c.mul(N, dA.ptr, La, La, dB.ptr, Lb, Lb, dC.ptr, La + Lb, La + Lb)
        C = np.zeros(N * (La + Lb), dtype=np.uint32)
        assert np.array_equal(dC.numpy(), ref.mul(N, A, La, La, B, Lb, Lb, C, La + Lb))
        assert c.workspace_size > 0
    finally:
        c.close()


def test_scratch_failure_in_ragged_batch(ctx):
    import gpupi_b200 as g
    rng = np.random.default_rng(13)
    n = 64
    La = rng.integers(1, 3000, size=n).astype(np.uint32)
    Lb = rng.integers(1, 3000, size=n).astype(np.uint32)
    Lc = La.astype(np.uint64) + Lb

    def offs(L):
        return np.concatenate([[0], np.cumsum(L.astype(np.uint64))[:-1]]).astype(np.uint64)

    A = rng.integers(0, 1 << 32, size=int(La.sum()), dtype=np.uint64).astype(np.uint32)
    B = rng.integers(0, 1 << 32, size=int(Lb.sum()), dtype=np.uint64).astype(np.uint32)
    dA, dB, dC = to_dev(A), to_dev(B), g.DeviceLimbs(int(Lc.sum()))
    base = g.scratch_live_bytes()
    g.fail_alloc(g.ALLOC_SCRATCH, 2)
    with pytest.raises(g.GpupiError, match="cudaError 2"):
        ctx.mul_ragged(dA.ptr, offs(La), La, dB.ptr, offs(Lb), Lb, dC.ptr, offs(Lc))
    g.fail_alloc(0, 0)
    assert g.scratch_live_bytes() == base
    ctx.mul_ragged(dA.ptr, offs(La), La, dB.ptr, offs(Lb), Lb, dC.ptr, offs(Lc))
    got = dC.numpy()
    oa, ob, oc = offs(La), offs(Lb), offs(Lc)
    for i in range(0, n, 7):
        a = int.from_bytes(A[int(oa[i]):int(oa[i]) + int(La[i])].tobytes(), "little")
        b = int.from_bytes(B[int(ob[i]):int(ob[i]) + int(Lb[i])].tobytes(), "little")
        c = int.from_bytes(got[int(oc[i]):int(oc[i]) + int(Lc[i])].tobytes(), "little")
        assert c == a * b
