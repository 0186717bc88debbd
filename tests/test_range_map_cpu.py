"""The scratch arena's host bookkeeping (gpupi_b200/csrc/range_map.h), built
with g++ and exercised by a randomised invariant check (no GPU)."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not installed")
def test_range_map_invariants(tmp_path):
    exe = tmp_path / "range_map_check"
    subprocess.run(["g++", "-std=c++17", "-O2", f"-I{ROOT / 'gpupi_b200' / 'csrc'}",
                    str(ROOT / "tests" / "range_map_check.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert "range_map ok" in r.stdout
