"""The tree checkpoint's file format (gpupi_b200/csrc/checkpoint_file.h),
built with g++: round trip, atomic rename, and rejection of another tree
size, flipped bits, truncation, trailing bytes, damaged length fields and
lengths above the caller's bound; a write to an unwritable location fails
cleanly (no GPU)."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not installed")
def test_checkpoint_file_format(tmp_path):
    exe = tmp_path / "checkpoint_check"
    subprocess.run(["g++", "-std=c++17", "-O2", f"-I{ROOT / 'gpupi_b200' / 'csrc'}",
                    str(ROOT / "tests" / "checkpoint_check.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    assert "checkpoint ok" in r.stdout
