"""Build the gpupi_b200 native library and CLI for sm_100a.

Outputs (in-tree, git-ignored):
  gpupi_b200/libgpupi_b200.so   batched-MP API + C ABI + pi pipeline
  gpupi_b200/pi_bs_gpu          command-line driver (same interface as gpupi's)

Each .cu file is compiled to an object under gpupi_b200/_build/ (rebuilt when
the source or any header is newer), then linked.  nvcc cross-compiles, so this
runs on machines without a GPU.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
INCLUDE = ROOT / "include"
BUILD = HERE / "_build"
LIB = HERE / "libgpupi_b200.so"
CLI = HERE / "pi_bs_gpu"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         f"-I{INCLUDE}", f"-I{CSRC}"]

LIB_SOURCES = [
    "batch_arith.cu", "carry_ops.cu", "shift.cu", "bitlength.cu", "exactdiv.cu",
    "mul_naive.cu", "mul_tc.cu", "mul_ntt.cu", "decimal.cu", "pi_engine.cu", "bbp.cu", "mul_ragged.cu", "scratch.cu", "tune.cu", "int_peak.cu", "capi.cu",
]
CLI_SOURCES = ["pi_main.cu"]


def _headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h")))


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: Path, obj: Path, extra: list[str]) -> None:
    cmd = [NVCC, *ARCH, *FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stderr}")
    if r.stderr.strip():
        sys.stderr.write(r.stderr)


def build(verbose: bool = False, jobs: int | None = None, extra: list[str] | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    extra = extra or []
    hdrs = _headers()
    work = []
    for name in LIB_SOURCES + CLI_SOURCES:
        src = CSRC / name
        obj = BUILD / (name + ".o")
        if _stale(obj, [src, *hdrs, Path(__file__)]):
            work.append((src, obj))
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        futs = {ex.submit(_compile, s, o, extra): s for s, o in work}
        for f in cf.as_completed(futs):
            f.result()
            if verbose:
                print("compiled", futs[f].name)
    lib_objs = [BUILD / (n + ".o") for n in LIB_SOURCES]
    if _stale(LIB, lib_objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, lib_objs), "-lcudart"]
        subprocess.run(cmd, check=True)
    cli_objs = [BUILD / (n + ".o") for n in CLI_SOURCES]
    if _stale(CLI, cli_objs + [LIB]):
        cmd = [NVCC, *ARCH, "-o", str(CLI), *map(str, cli_objs), f"-L{HERE}", "-lgpupi_b200",
               "-Xlinker", "-rpath=$ORIGIN", "-lcudart"]
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True)
    print(LIB)
