"""Build the host C++ restatement (oracle/pi_cpu.cpp) into oracle/_build/pi_cpu.

Test infrastructure and CPU baseline only.  g++ -O2, std::thread, GMP linked
by path through the prototype header in oracle/shim (the image has
libgmp.so.10 but no gmp.h).

    python oracle/build_cpu.py
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_build" / "pi_cpu"
GMP = "/usr/lib/x86_64-linux-gnu/libgmp.so.10"


def build() -> Path:
    src = HERE / "pi_cpu.cpp"
    OUT.parent.mkdir(exist_ok=True)
    deps = [src, HERE / "shim" / "gmp.h"]
    if OUT.exists() and all(OUT.stat().st_mtime > d.stat().st_mtime for d in deps):
        return OUT
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", str(HERE / "shim"), str(src), GMP,
                    "-o", str(OUT)], check=True)
    return OUT


if __name__ == "__main__":
    print(build())
    sys.exit(0)
