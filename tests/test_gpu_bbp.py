"""BBP hex-digit spot check on the GPU: the kernel's fixed-point sums equal the
CPU restatement bit for bit, and the pipeline's RET agrees with BBP at seeded
positions (an independent check of pi's digits, integer arithmetic only)."""
import numpy as np
import pytest

import bbp_ref

pytestmark = pytest.mark.gpu


def test_bbp_kernel_equals_restatement():
    import gpupi_b200 as g
    pos = list(range(0, 33)) + [97, 500, 1234, 2000, 4095]
    got = g.bbp_fractions(pos)
    for n, f in zip(pos, got):
        assert int(f) == bbp_ref.bbp_fraction(n), n


def test_ret_agrees_with_bbp(ctx):
    import gpupi_b200 as g
    r = g.pi_compute(1000000, ctx, copy_digits=0)
    rng = np.random.default_rng(0xBB9)
    top = 8 * (r.ret_len - 1) - 64            # keep clear of the truncated tail
    pos = sorted(int(x) for x in rng.integers(0, top, size=16))
    bad, unsure = g.bbp_spot_check(r.ret, pos)
    assert bad == []
    assert len(unsure) <= 2
