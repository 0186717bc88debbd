"""The allocation-free add (gpupi_mp_add_noalloc) against the regular one.

Callers that cannot allocate device memory when they need an add (all memory
already given to another allocator, or loops that must not call cudaMalloc /
cudaFree because those can synchronise the device) use gpupi_mp_add_noalloc:
its carry flags live in a fixed 256 KiB array inside the library.  This file
is collected last on purpose; it must pass both alone in a fresh process and
after the other tests.  The check is bit-exact, two calls in a row (the
second call finds the first call's flags still in the array).
"""
import numpy as np
import pytest

from helpers import rand_buf, to_dev

pytestmark = pytest.mark.gpu


def _add_both_ways(ctx, N, L, seed):
    import gpupi_b200 as g
    rng = np.random.default_rng(seed)
    A, B = rand_buf(rng, N, L, L), rand_buf(rng, N, L, L)
    # long all-ones runs so carries cross tiles and the fix-up reads the flags
    for r in range(N):
        s = int(rng.integers(0, L // 2))
        A[r * L + s: r * L + s + L // 3] = 0xFFFFFFFF
    dA, dB = to_dev(A), to_dev(B)
    want, got = to_dev(np.zeros(N * (L + 1), dtype=np.uint32)), to_dev(np.zeros(N * (L + 1), dtype=np.uint32))
    ctx.add(N, dA.ptr, L, L, dB.ptr, L, L, want.ptr, L + 1, L + 1)
    g.add_noalloc(N, dA.ptr, L, L, dB.ptr, L, L, got.ptr, L + 1, L + 1)
    return want.numpy(), got.numpy()


def test_noalloc_add_matches_add_twice(ctx):
    # multi-tile rows (uses the fixed flag array), then a different shape
    for (N, L, seed) in [(3, 50000, 1), (5, 20000, 2)]:
        want, got = _add_both_ways(ctx, N, L, seed)
        assert np.array_equal(got, want)
    # warp-per-row shapes need no flags at all
    want, got = _add_both_ways(ctx, 700, 300, 3)
    assert np.array_equal(got, want)


def test_noalloc_add_rejects_beyond_limit():
    import gpupi_b200 as g
    # 20 rows x 3300 tiles of 4096 limbs = 66000 flags > 65536: rejected before any launch
    N, L = 20, 4096 * 3300
    d = g.DeviceLimbs(N * L)
    with pytest.raises(g.GpupiError):
        g.add_noalloc(N, d.ptr, L, L, d.ptr, L, L, d.ptr, L, L)
