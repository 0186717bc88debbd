"""CPU checks of the native boundary: the library builds for sm_100a, loads,
and exports every symbol include/gpupi_c.h declares plus the reference's C++
API (mangled names) so gpupi's own callers link unchanged.  No compute calls."""
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def built():
    from gpupi_b200.build import build
    return build()


def _exports(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib)], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


def test_c_abi_symbols(built):
    import gpupi_b200 as g
    header = (ROOT / "include" / "gpupi_c.h").read_text()
    declared = set(re.findall(r"\b(gpupi_[a-z0-9_]+)\(", header))
    exported = _exports(built)
    assert declared, "no declarations parsed"
    assert declared <= exported, declared - exported
    assert declared == set(g.C_ABI_SYMBOLS)
    lib = g.lib()
    assert lib.gpupi_version().startswith(b"gpupi_b200")


CPP_API = ["batch_mp_array_create", "batch_mp_array_release", "batch_mp_init", "batch_mp_destroy",
           "batch_mp_workspace_size", "batch_mp_ensure_workspace", "batch_mp_mul", "batch_mp_mul_small",
           "batch_mp_exactdiv_small", "batch_mp_add", "batch_mp_add_small", "batch_mp_shift_add",
           "batch_mp_shift_sub", "batch_mp_sub", "batch_mp_sub_small", "batch_mp_shift_bits",
           "batch_mp_bitlength_max", "batch_mp_limblength_max", "batch_add_simple", "batch_sub_simple",
           "batch_add_small", "batch_sub_small", "batch_mul_small", "batch_shift_bits", "batch_shift_add_simple",
           "batch_shift_sub_simple", "batch_mul_naive", "batch_mul_ntt", "init_ntt_precomputed_tables",
           "batch_mul_ntt_workspace_size", "batch_exactdiv_small", "batch_bitlength_max", "batch_limblength_max",
           "batch_bitlength_workspace_size", "batch_decimal_naive", "convert_decimal_precompute_powers",
           "convert_decimal_release_powers", "convert_decimal_equal_split",
           "batch_add_simple_workspace_size", "batch_sub_simple_workspace_size", "batch_add_small_workspace_size",
           "batch_sub_small_workspace_size", "batch_mul_small_workspace_size",
           "batch_shift_add_simple_workspace_size", "batch_shift_sub_simple_workspace_size"]


def test_reference_cpp_api_exported(built):
    out = subprocess.run(["nm", "-DC", "--defined-only", str(built)], capture_output=True, text=True, check=True).stdout
    names = {re.sub(r"\(.*", "", line.split(" ", 2)[-1]) for line in out.splitlines() if line.strip()}
    missing = [n for n in CPP_API if n not in names]
    assert not missing, missing
    assert "BatchMPArray::compact" in names


def test_cli_exists(built):
    assert (ROOT / "gpupi_b200" / "pi_bs_gpu").exists()
    r = subprocess.run([str(ROOT / "gpupi_b200" / "pi_bs_gpu")], capture_output=True, text=True)
    assert r.returncode == 1 and "Usage" in r.stderr


@pytest.mark.parametrize("args", [["100", "--bogus"], ["100", "--benchmark", "--full-print"],
                                  ["100", "--output"], ["100", "--full-print", "--output", "x.txt"],
                                  ["100", "--plain", "--plain"], ["-5"], ["100", "--checkpoint"]])
def test_cli_rejects_bad_arguments(built, args):
    """Usage errors exit 1 before any device work, as the reference's CLI does."""
    r = subprocess.run([str(ROOT / "gpupi_b200" / "pi_bs_gpu"), *args], capture_output=True, text=True)
    assert r.returncode == 1 and "Usage" in r.stderr


def test_no_cpu_fallback_without_gpu():
    """Compute entry points refuse to run without a CUDA device."""
    import torch
    import gpupi_b200 as g
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(g.GpupiError):
        g.Context()
