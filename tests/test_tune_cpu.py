"""The tune table (gpupi_b200/csrc/tune.cu) on the host, no GPU: parsing,
rejection of malformed lines (the table in effect stays), the kernel each
length bucket gets (gpupi's public batch_mp_mul rule kept: the NTT never at
or below 1024 limbs, always above), and NTT shapes by need range."""
import pytest

import gpupi_b200 as g


@pytest.fixture(autouse=True)
def _fresh_table():
    g.tune_reset()
    yield
    g.tune_reset()


def test_builtin_rule():
    assert g.mul_kind(16, 16) == "school"          # register kernel
    assert g.mul_kind(200, 248) == "school"        # built-in crossover: 448
    assert g.mul_kind(200, 249) == "ntt"
    assert g.mul_kind(600, 424, public_api=True) == "school"   # the reference's 1024 rule
    assert g.mul_kind(600, 425, public_api=True) == "ntt"
    assert g.ntt_shape(3000, 3000) == (13, 1)
    assert g.ntt_shape(1 << 24, (1 << 24) + 1) == (25, 1)


def test_table_buckets_and_constraints():
    n = g.tune_load(text="""# comment line
mul 64 school
mul 1024 tc      # tensor cores up to 1024
mul 6000 tc
ntt 8193 10240 13 2
""")
    assert n == 4
    assert g.mul_kind(20, 20) == "school"
    assert g.mul_kind(40, 40) == "tc"
    assert g.mul_kind(512, 512) == "tc"
    assert g.mul_kind(2000, 2000) == "tc"
    assert g.mul_kind(3000, 2999) == "ntt"          # above every entry
    assert g.mul_kind(2049, 2049) == "ntt"          # tc limit: shorter operand <= 2048
    assert g.mul_kind(512, 512, public_api=True) == "tc"
    assert g.mul_kind(2000, 2000, public_api=True) == "ntt"
    assert g.ntt_shape(5000, 5000) == (13, 2)       # need 9999 in [8193, 10240]
    assert g.ntt_shape(3000, 3000) == (13, 1)       # below the entry: built-in rule
    assert g.ntt_shape(6000, 6000) == (14, 1)       # above it: built-in rule
    assert "mul 1024 tc" in g.tune_describe()


def test_public_rule_never_uses_ntt_at_or_below_1024():
    g.tune_load(text="mul 2000 ntt\n")
    assert g.mul_kind(100, 100) == "ntt"
    assert g.mul_kind(100, 100, public_api=True) == "school"


@pytest.mark.parametrize("bad", ["mul 0 tc", "mul 100 fft", "ntt 10 5 13 1", "ntt 8193 20000 13 1",
                                 "ntt 100 200 12 2", "frobnicate 1", "mul"])
def test_malformed_lines_are_rejected(bad):
    g.tune_load(text="mul 512 tc\n")
    with pytest.raises(g.GpupiError):
        g.tune_load(text="mul 64 school\n" + bad + "\n")
    assert g.mul_kind(100, 100) == "tc"             # the previous table stays in effect


def test_table_file_round_trip(tmp_path):
    p = tmp_path / "t.txt"
    p.write_text("mul 256 school\nmul 4096 tc\nntt 16385 20480 14 2\n")
    assert g.tune_load(p) == 3
    assert g.mul_kind(1000, 1000) == "tc" and g.ntt_shape(9000, 9000) == (14, 2)
    with pytest.raises(g.GpupiError):
        g.tune_load(tmp_path / "missing.txt")
