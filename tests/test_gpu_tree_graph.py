"""The splitting tree as a CUDA graph (pi_engine.cu tree_run): the first run
of a size records the compact() length schedule, the second captures the
tree with it, later runs launch the graph and check the device's lengths
against the schedule.  Every run's RET and digits equal the reference
build's; an altered schedule is caught by that check and the tree runs
directly; the stage profiler and the kernel timers keep the direct path."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

import pi_ref

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
FIX = {e["digits"]: e for e in json.loads((ROOT / "tests" / "golden" / "ref_fixtures.json").read_text())["pi"]}


def _delta(a, b):
    return {k: b[k] - a[k] for k in a}


def _check_ref(r, d):
    e = FIX[d]
    assert r.ret_len == e["ret_len"] and pi_ref.mod_hash(r.ret) == e["ret_hash"]
    assert hashlib.sha256(("3" + r.dec + "\n").encode()).hexdigest() == e["stdout_sha256"]


@pytest.mark.parametrize("plain", [False, True], ids=["tuned", "plain"])
def test_graph_replays_are_exact(plain):
    import gpupi_b200 as g
    ctx = g.Context()
    try:
        d = 1_000_000
        s0 = g.tree_graph_stats()
        launches = []
        for _ in range(4):
            l0 = g.launch_count()
            r = g.pi_compute(d, ctx, plain=plain)
            launches.append(g.launch_count() - l0)
            _check_ref(r, d)
        dd = _delta(s0, g.tree_graph_stats())
        assert dd == {"recorded": 1, "captured": 1, "replayed": 3, "fallbacks": 0, "disabled": 0}
        # a graph run counts the kernels its graph holds, the same every time
        assert launches[3] == launches[2] > 0
    finally:
        ctx.close()


def test_altered_schedule_falls_back_to_the_direct_tree(ctx):
    import gpupi_b200 as g
    d = 300_000
    want = g.pi_compute(d, ctx)
    g.pi_compute(d, ctx)
    g.pi_compute(d, ctx)
    s0 = g.tree_graph_stats()
    g.tree_graph_perturb()
    r = g.pi_compute(d, ctx)
    assert _delta(s0, g.tree_graph_stats())["fallbacks"] == 1
    assert np.array_equal(r.ret, want.ret) and r.dec == want.dec
    # and the size records, captures and replays again
    for _ in range(3):
        r = g.pi_compute(d, ctx)
        assert np.array_equal(r.ret, want.ret) and r.dec == want.dec
    dd = _delta(s0, g.tree_graph_stats())
    assert dd["recorded"] == 1 and dd["captured"] == 1 and dd["replayed"] >= 1


def test_timers_and_profiler_keep_the_direct_tree(ctx):
    import gpupi_b200 as g
    d = 200_000
    for _ in range(3):
        g.pi_compute(d, ctx)
    s0 = g.tree_graph_stats()
    g.timer_reset()
    g.timer_enable(True)
    try:
        r = g.pi_compute(d, ctx)
    finally:
        g.timer_enable(False)
        g.timer_reset()
    p = g.pi_compute(d, ctx, profile=True)
    assert _delta(s0, g.tree_graph_stats())["replayed"] == 0
    assert r.dec == p.dec == g.pi_compute(d, ctx).dec
