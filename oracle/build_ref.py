"""Build the reference (gpupi) from its own sources into oracle/_ref/.

Test infrastructure only.  Compiles the unmodified reference sources where
they lie (``--reference DIR``, else ``$GPUPI_REFERENCE_DIR``, else
``../reference`` beside this repository) with nvcc for sm_100a, adding two shim headers
written for this project (oracle/shim: a <cuda/warp> stand-in, since CUDA 12.9
lacks that CUDA 13 header, and GMP's public prototypes, since the image has
libgmp.so.10 but no gmp.h).  GMP is linked by path.  Outputs:

  oracle/_ref/pi_bs_gpu_ref          the reference pi_bs_gpu (parity oracle + GPU timing)
  oracle/_ref/<name>_ref             reference tests linked with the reference library
  oracle/_ref/<name>_on_gpupi_b200   the same tests linked with libgpupi_b200.so
                                     through include/ (drop-in check)
  oracle/_ref/ref_configs_ref        oracle/ref_configs.cu (benchmark configurations
                                     through the public API) linked with the
                                     reference's objects (fixture generator)
  oracle/_ref/ref_configs_on_gpupi_b200  the same program linked with libgpupi_b200.so

    python oracle/build_ref.py [--tests] [--reference DIR]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
REF = Path(os.environ.get("GPUPI_REFERENCE_DIR", str(ROOT.parent / "reference")))
OUT = HERE / "_ref"
SHIM = HERE / "shim"
NVCC = "/usr/local/cuda/bin/nvcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
GMP = "-Xlinker=/usr/lib/x86_64-linux-gnu/libgmp.so.10"

LIB_SRCS = ["batch_arith.cu", "batch_mul_ntt.cu", "batch_add.cu", "batch_sub.cu", "batch_shift_add.cu",
            "batch_shift_sub.cu", "batch_mul_small.cu", "batch_exactdiv_small.cu", "batch_add_small.cu",
            "batch_sub_small.cu", "batch_mul_naive.cu", "batch_bitlength.cu", "batch_shift.cu",
            "convert_decimal.cu", "batch_decimal_naive.cu"]

# reference test -> sources it links besides itself (from its *_compile.sh)
TESTS = {
    "batch_add_test": ["batch_add.cu"],
    "batch_sub_test": ["batch_sub.cu"],
    "batch_add_small_test": ["batch_add_small.cu"],
    "batch_sub_small_test": ["batch_sub_small.cu"],
    "batch_mul_small_test": ["batch_mul_small.cu"],
    "batch_shift_add_test": ["batch_shift_add.cu"],
    "batch_shift_sub_test": ["batch_shift_sub.cu"],
    "batch_shift_test": ["batch_shift.cu"],
    "batch_exactdiv_small_test": ["batch_exactdiv_small.cu"],
    "batch_bitlength_test": ["batch_bitlength.cu"],
    "batch_mul_naive_test": ["batch_mul_naive.cu"],
    "batch_mul_ntt_test": ["batch_mul_ntt.cu"],
    "batch_decimal_naive_test": ["batch_decimal_naive.cu"],
    "convert_decimal_test": LIB_SRCS,
    "batch_arith_test": [s for s in LIB_SRCS if s not in ("convert_decimal.cu", "batch_decimal_naive.cu")],
}


def nvcc_obj(src: Path, obj: Path, includes: list[Path]) -> None:
    if obj.exists() and obj.stat().st_mtime > src.stat().st_mtime:
        return
    cmd = [NVCC, *ARCH, "-O3", "-std=c++17", "-w", *[f"-I{p}" for p in includes], "-c", str(src), "-o", str(obj)]
    subprocess.run(cmd, check=True)


def build_pi() -> Path:
    objdir = OUT / "obj"
    objdir.mkdir(parents=True, exist_ok=True)
    srcs = ["pi_bs_gpu.cu"] + LIB_SRCS
    with cf.ThreadPoolExecutor() as ex:
        list(ex.map(lambda s: nvcc_obj(REF / s, objdir / (s + ".o"), [SHIM, REF]), srcs))
    exe = OUT / "pi_bs_gpu_ref"
    subprocess.run([NVCC, *ARCH, "-o", str(exe), *[str(objdir / (s + ".o")) for s in srcs], GMP], check=True)
    return exe


def build_configs() -> None:
    """oracle/ref_configs.cu linked both ways (reference objects; this library)."""
    objdir = OUT / "obj"
    objdir.mkdir(parents=True, exist_ok=True)
    src = HERE / "ref_configs.cu"
    deps = [s for s in LIB_SRCS]
    with cf.ThreadPoolExecutor() as ex:
        list(ex.map(lambda s: nvcc_obj(REF / s, objdir / (s + ".o"), [SHIM, REF]), deps))
    robj = objdir / "ref_configs.o"
    nvcc_obj(src, robj, [SHIM, REF])
    subprocess.run([NVCC, *ARCH, "-o", str(OUT / "ref_configs_ref"), str(robj),
                    *[str(objdir / (d + ".o")) for d in deps], GMP], check=True)
    mine = ROOT / "gpupi_b200"
    mobj = objdir / "ref_configs.mine.o"
    nvcc_obj(src, mobj, [ROOT / "include"])
    subprocess.run([NVCC, *ARCH, "-o", str(OUT / "ref_configs_on_gpupi_b200"), str(mobj), f"-L{mine}",
                    "-lgpupi_b200", "-Xlinker", f"-rpath={mine}"], check=True)


def build_tests() -> None:
    objdir = OUT / "obj"
    objdir.mkdir(parents=True, exist_ok=True)
    mine = ROOT / "gpupi_b200"
    jobs = []
    for name, deps in TESTS.items():
        jobs.append((name, deps))

    def one(job):
        name, deps = job
        src = REF / (name + ".cu")
        # reference test linked with the reference sources
        for d in deps:
            nvcc_obj(REF / d, objdir / (d + ".o"), [SHIM, REF])
        tobj = objdir / (name + ".o")
        nvcc_obj(src, tobj, [SHIM, REF])
        subprocess.run([NVCC, *ARCH, "-o", str(OUT / (name + "_ref")), str(tobj),
                        *[str(objdir / (d + ".o")) for d in deps], GMP, "-lcurand"], check=True)
        # the same test source compiled against include/ and linked with libgpupi_b200.so
        mobj = objdir / (name + ".mine.o")
        nvcc_obj(src, mobj, [SHIM, ROOT / "include"])
        subprocess.run([NVCC, *ARCH, "-o", str(OUT / (name + "_on_gpupi_b200")), str(mobj), f"-L{mine}",
                        "-lgpupi_b200", "-Xlinker", f"-rpath={mine}", GMP, "-lcurand"], check=True)
        return name

    with cf.ThreadPoolExecutor() as ex:
        for n in ex.map(one, jobs):
            print("built", n)


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--tests", action="store_true", help="also build the reference tests both ways")
    ap.add_argument("--reference", help="reference source directory")
    a = ap.parse_args()
    global REF
    if a.reference:
        REF = Path(a.reference)
    if not REF.exists():
        print("reference sources not present; nothing to build", file=sys.stderr)
        return 0
    print("built", build_pi())
    build_configs()
    print("built ref_configs")
    if a.tests:
        build_tests()
    return 0


if __name__ == "__main__":
    sys.exit(main())
