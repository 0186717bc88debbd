#!/usr/bin/env python
"""Benchmark: milliseconds to compute pi to 1,000,000,000 decimal digits on a
B200 with gpupi_b200 (the pi_bs_gpu pipeline: Chudnovsky binary splitting,
Pell sqrt(10005), recursive reciprocal, final product, decimal conversion).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--digits D]

One JSON line on stdout (rank 0).  A step is one full pipeline run.  The
pipeline does not shard (it is one dependent chain of products), so N > 1
runs N independent replicas, one per GPU, timed as the max over ranks.

Our arm (``--impl ours``):
  value      device time per step (CUDA events on the library's stream), RET
             and digits left in HBM (no host copies inside the step);
  e2e        the same computation through the C ABI call with the digits and
             RET copied into pinned host memory every step (wall clock);
  roofline   the kernel family with the largest share of device time, its
             algorithmic bytes / its event-timed duration, against the
             measured HBM copy bandwidth;
  cpu_baseline  the CPU restatement (oracle) on a bounded sample, rank 0.
  reference_gpu_build  gpupi's own CUDA build (oracle/_ref/pi_bs_gpu_ref,
             compiled from the reference's sources) and this library's CLI
             run alternately as cold processes, `--benchmark`, same digits:
             each program's own elapsed_ms and RET hash (rank 0, after the
             timed regions).
The reference arm (``--impl reference``) runs gpupi's own CUDA build,
``pi_bs_gpu_ref <digits> --benchmark``, one cold process per step on rank 0's
GPU, and reports its own elapsed_ms (CUDA events around the same pipeline,
digits left on the device, like ``value``).  Where that build is absent it
times the host C++ restatement instead (the reference has no CPU
implementation) and says so.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import random
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent

# DRAM traffic of the dominant kernel family relative to its algorithmic
# bytes, from one ncu capture (dram__bytes_read.sum + dram__bytes_write.sum of
# k_rows_r<12> on a 2^22 x 2^22-limb product: 264.0 MB against 302.0 MB of
# algorithmic bytes; part of the output is still in L2 at kernel end).  The
# pi run's launches are scaled by their algorithmic bytes.
BBP_POSITIONS = 64
# DRAM bytes (read + write) over algorithmic bytes of one launch, from ncu
# captures (profiles/ntt_rows_cols_4Mi.md, profiles/ntt_split_rows_4Mi.md,
# profiles/ntt_rows_level_pi1e8.md); applied to each launch of the family
NCU_TRAFFIC_RATIO = {"ntt_rows_fused": 264.006 / 301.990,
                     "ntt_cols_fwd_first": 229.642496 / 234.881024,
                     "ntt_rows_level": (2630.51 + 1619.05) / 4026.531840}
NCU_TRAFFIC_SOURCE = {"ntt_rows_fused": "ncu capture of k_rows_r<12> on a 2^22 x 2^22-limb product, "
                                        "scaled to each launch by its algorithmic bytes",
                      "ntt_cols_fwd_first": "ncu capture of k_cols_r<6, first, fwd, pair> on a 2^22 x 2^22-limb "
                                            "product, scaled to each launch by its algorithmic bytes",
                      "ntt_rows_level": "ncu capture of k_rows_level in pi to 1e8 digits (2^25 points x 3 primes "
                                        "per launch), scaled to each launch by its algorithmic bytes"}
# Warp instructions per algorithmic byte of each kernel family, by pipe
# (FMA-heavy = IMAD, ALU, all), from one ncu capture of every launch of pi to
# 1e8 digits with the library's kernel-timer bytes of the same computation
# (profiles/int_pipes_pi1e8.md).  Scaled to this run's bytes and divided by
# the live integer-pipe peaks they give each family's integer roofline.
INT_WINST_PER_BYTE = {
    "ntt_rows_level": (0.20437, 0.205252, 0.487605), "ntt_cols_fwd_first": (0.187598, 0.211507, 0.477682),
    "ntt_cols_inv": (0.100109, 0.11195, 0.246731), "schoolbook_tc": (0.143044, 0.265617, 0.763927),
    "ntt_crt_carry": (0.075663, 0.095934, 0.230741), "ntt_rows_fused": (0.223057, 0.220512, 0.527792),
    "schoolbook": (0.212093, 0.176371, 0.49994), "ntt_cols_fwd": (0.080255, 0.096138, 0.204625),
    "carry_chain": (0.077046, 0.098004, 0.245578), "ntt_local": (0.55531, 0.538007, 1.292256),
    "ntt_rows_inv": (0.078142, 0.077174, 0.193306), "ntt_rows_fwd": (0.10064, 0.094374, 0.250671),
    "ntt_coset_combine": (0.103479, 0.100658, 0.265951), "decimal_extract": (0.075693, 0.08626, 0.224201),
    "decimal_leaf": (0.596097, 0.168555, 0.837855), "shift": (0.035647, 0.045182, 0.115069)}
INT_SOURCE = ("ncu sm__inst_executed_pipe_{fmaheavy,alu}.sum and sm__inst_executed.sum over every launch of "
              "pi_bs_gpu 100000000 (profiles/int_pipes_pi1e8.md), per algorithmic byte, scaled to this run")
sys.path.insert(0, str(ROOT))

METRIC = "ms to 1e9 digits of pi (bit-exact), tuned vs plain form on B200; NTT HBM GB/s"
CPU_SAMPLE_DIGITS = 20_000_000         # host C++ restatement, all cores: ~9 s on 8 cores
REF_SAMPLE_DIGITS = 10_000_000         # per reference-arm step, ~4 s on 8 cores
PY_SAMPLE_DIGITS = 1_000_000           # CPython fallback when the C++ restatement is not built


def _peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text())
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "fallback": True}


class Clocks:
    """nvidia-smi sampler over the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = Path(f"/tmp/gpupi_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        # nvidia-smi's own start-up (NVML initialisation) must not fall inside
        # the timed region: wait for its first sample before timing starts
        t0 = time.time()
        while time.time() - t0 < 10.0 and self.proc.poll() is None:
            self.f.flush()
            if self.path.exists() and self.path.stat().st_size > 0:
                break
            time.sleep(0.05)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        self.path.unlink(missing_ok=True)
        loaded = [s for s in sm if s > 0.5 * max(smax or [1])] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _max_over_ranks(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(ws: int):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def _pi_cpu(digits: int) -> dict | None:
    """Run the host C++ restatement (oracle/_build/pi_cpu, GMP, all host
    threads) once; None when it is not built."""
    exe = ROOT / "oracle" / "_build" / "pi_cpu"
    if not exe.exists():
        return None
    out = subprocess.run([str(exe), str(digits)], capture_output=True, text=True, check=True).stdout
    first = out.splitlines()[0]
    fields = dict(kv.split("=", 1) for kv in first.split() if "=" in kv)
    ret_hash = int(out.splitlines()[1].rsplit("=", 1)[1])
    return {"ms": float(fields["elapsed_ms"]), "threads": int(fields["threads"]), "ret_hash": ret_hash}


def _cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline_sample(digits: int) -> dict:
    r = _pi_cpu(digits)
    if r is not None:
        ms = r["ms"]
        return {"value": ms * (1e9 / digits), "unit": "ms (linear extrapolation to 1e9 digits)",
                "cores": r["threads"], "kind": "port",
                "sample": f"pi to {digits} digits with the host C++ restatement of the pipeline "
                          f"(oracle/pi_cpu.cpp, GMP integers, {r['threads']} threads on {_cpu_model()}): "
                          f"{ms:.1f} ms, RET hash {r['ret_hash']}, scaled by 1e9/{digits} "
                          f"(a lower bound: binary splitting grows faster than linearly)",
                "sample_ms": ms}
    sys.path.insert(0, str(ROOT / "oracle"))
    import pi_ref
    d = PY_SAMPLE_DIGITS
    t0 = time.perf_counter()
    pi_ref.pi_digits(d)
    ms = (time.perf_counter() - t0) * 1e3
    return {"value": ms * (1e9 / d), "unit": "ms (linear extrapolation to 1e9 digits)", "cores": 1,
            "kind": "port",
            "sample": f"pi to {d} digits with the CPU restatement of the pipeline (oracle/pi_ref.py, "
                      f"CPython big integers, one core): {ms:.1f} ms, scaled by 1e9/{d} "
                      f"(a lower bound: binary splitting grows faster than linearly)",
            "sample_ms": ms}


REF_CLI = ROOT / "oracle" / "_ref" / "pi_bs_gpu_ref"
OUR_CLI = ROOT / "gpupi_b200" / "pi_bs_gpu"
REF_FIXTURES = ROOT / "tests" / "golden" / "ref_fixtures.json"


def _cli_benchmark(exe: Path, digits: int, device: int) -> dict:
    """One cold `<exe> <digits> --benchmark` process: its own elapsed_ms, RET
    length and RET hash (pi_bs_gpu.cu:2216-2224 format), and the wall time."""
    env = dict(os.environ, CUDA_VISIBLE_DEVICES=str(device))
    t0 = time.perf_counter()
    r = subprocess.run([str(exe), str(digits), "--benchmark"], capture_output=True, text=True, env=env,
                       timeout=900)
    wall = (time.perf_counter() - t0) * 1e3
    if r.returncode != 0:
        raise RuntimeError(f"{exe.name} {digits} --benchmark exited {r.returncode}: {r.stderr[-500:]}")
    lines = r.stdout.splitlines()
    f = dict(kv.split("=", 1) for kv in lines[0].split() if "=" in kv)
    ret_line = next(l for l in lines if l.startswith("RET = "))
    return {"elapsed_ms": float(f["elapsed_ms"]), "ret_len": int(f["RET_len"]),
            "ret_hash": int(ret_line.rsplit("=", 1)[1]), "wall_ms": wall}


def _ref_fixture(digits: int) -> dict | None:
    """The reference build's recorded result for this digit count, if any."""
    if not REF_FIXTURES.exists():
        return None
    for e in json.loads(REF_FIXTURES.read_text()).get("pi", []):
        if e["digits"] == digits:
            return e
    return None


def _gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def run_reference_arm(args, ws, rank, local):
    """gpupi's own CUDA build, one cold `pi_bs_gpu_ref <digits> --benchmark`
    process per step on this rank's GPU (rank 0 only), timed by its own
    device events; its RET is checked against the recorded fixture.  Without
    that build (or a GPU) the arm times the host C++ restatement instead."""
    if rank != 0:
        return
    if REF_CLI.exists() and _gpu_available():
        for _ in range(args.warmup):
            _cli_benchmark(REF_CLI, args.digits, local)
        runs = [_cli_benchmark(REF_CLI, args.digits, local) for _ in range(args.steps)]
        ms = statistics.mean(r["elapsed_ms"] for r in runs)
        fx = _ref_fixture(args.digits)
        line = {
            "impl": "reference", "metric": METRIC, "value": ms, "unit": "ms", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (pi has no input data)",
            "config": {"workload": f"pi to {args.digits} decimal digits (pi_bs_gpu {args.digits})",
                       "digits": args.digits, "program": "gpupi's pi_bs_gpu built unmodified from its sources "
                                                          "for sm_100a (oracle/build_ref.py)",
                       "l2": "working set larger than L2; no flush needed"},
            "step_ms": [round(r["elapsed_ms"], 3) for r in runs],
            "process_wall_ms": [round(r["wall_ms"], 1) for r in runs],
            "ret_len": runs[-1]["ret_len"], "ret_hash": runs[-1]["ret_hash"],
            "ret_matches_fixture": (None if fx is None else
                                    all(r["ret_hash"] == fx["ret_hash"] and r["ret_len"] == fx["ret_len"]
                                        for r in runs)),
            "cpu_baseline": {"value": ms, "unit": "ms", "cores": 1, "kind": "reference",
                             "sample": f"gpupi's own CUDA build (one host thread driving the GPU), "
                                       f"pi_bs_gpu_ref {args.digits} --benchmark, one cold process per step, "
                                       f"mean of its own elapsed_ms over {args.steps} steps"},
            "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return
    d = REF_SAMPLE_DIGITS
    use_cpp = _pi_cpu(1000) is not None
    if not use_cpp:
        sys.path.insert(0, str(ROOT / "oracle"))
        import pi_ref
        d = PY_SAMPLE_DIGITS // 5

    def one():
        if use_cpp:
            return _pi_cpu(d)
        t0 = time.perf_counter()
        pi_ref.pi_digits(d)
        return {"ms": (time.perf_counter() - t0) * 1e3, "threads": 1}

    for _ in range(args.warmup):
        one()
    runs = [one() for _ in range(args.steps)]
    ms = statistics.mean(r["ms"] for r in runs) * (args.digits / d)
    cores = runs[0]["threads"]
    what = (f"oracle/pi_cpu.cpp (GMP, {cores} threads on {_cpu_model()})" if use_cpp
            else "oracle/pi_ref.py (CPython, one core)")
    line = {
        "impl": "reference", "metric": METRIC, "value": ms, "unit": "ms", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (pi has no input data)",
        "config": {"workload": f"pi to {args.digits} decimal digits (pi_bs_gpu {args.digits})",
                   "digits": args.digits, "sample_digits_per_step": d,
                   "l2": "working set larger than L2; no flush needed"},
        "cpu_baseline": {"value": ms, "unit": "ms", "cores": cores, "kind": "port",
                         "sample": f"pi to {d} digits per step with {what} (gpupi's own build "
                                   f"oracle/_ref/pi_bs_gpu_ref is not present or there is no GPU; the "
                                   f"reference has no CPU implementation), mean of {args.steps} steps scaled "
                                   f"linearly to {args.digits} (a lower bound)"},
        "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, ws, rank, local):
    import torch
    import gpupi_b200 as g

    torch.cuda.set_device(local)
    ctx = g.Context()
    digits = args.digits
    # warm-up: sizes the workspace and the stream-ordered pool, and takes the
    # splitting tree's graph through its one-time steps (the first run records
    # the length schedule, the second captures the graph into its own device
    # block, later runs replay it); then one run with the kernel timers on
    # sizes their event pool (the timers run the tree directly)
    for _ in range(max(3, args.warmup)):
        g.pi_compute(digits, ctx, device_only=True)
    g.timer_reset()
    g.timer_enable(True)
    g.pi_compute(digits, ctx, device_only=True)
    g.timer_enable(False)
    g.timer_reset()
    torch.cuda.synchronize()

    # device-timed steps, results stay in HBM
    clocks = Clocks(local)
    clocks.start()
    _barrier(ws)
    torch.cuda.synchronize()
    launches0 = g.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    inner = []
    for _ in range(args.steps):
        r = g.pi_compute(digits, ctx, device_only=True)
        inner.append(r.elapsed_ms)
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    _barrier(ws)
    launches = g.launch_count() - launches0
    ms_local = e0.elapsed_time(e1) / args.steps
    ms = _max_over_ranks(ms_local, ws)

    # the plain form (the reference's op sequence; same RET and digits),
    # device-timed the same way
    for _ in range(max(1, args.warmup - 1)):
        g.pi_compute(digits, ctx, device_only=True, plain=True)
    _barrier(ws)
    torch.cuda.synchronize()
    e4 = torch.cuda.Event(enable_timing=True)
    e5 = torch.cuda.Event(enable_timing=True)
    e4.record()
    for _ in range(args.steps):
        rp = g.pi_compute(digits, ctx, device_only=True, plain=True)
    e5.record()
    torch.cuda.synchronize()
    ms_plain = _max_over_ranks(e4.elapsed_time(e5) / args.steps, ws)

    # the same steps again with per-launch CUDA events around every kernel
    # (kernel families and the roofline of the dominant one)
    g.timer_reset()
    g.timer_enable(True)
    _barrier(ws)
    torch.cuda.synchronize()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record()
    for _ in range(args.steps):
        g.pi_compute(digits, ctx, device_only=True)
    e3.record()
    torch.cuda.synchronize()
    g.timer_enable(False)
    ktimes = g.timer_report()
    kgaps = g.timer_gaps()
    ms_timed_local = e2.elapsed_time(e3) / args.steps

    # end to end through the C ABI, digits + RET copied to pinned host memory
    pinned = torch.empty(digits, dtype=torch.uint8, pin_memory=True)
    pinned_ret = torch.empty(g.ret_limbs_bound(digits), dtype=torch.int32, pin_memory=True)
    # one untimed call first: the first use of freshly pinned pages is slow
    g.pi_compute(digits, ctx, host_digits=pinned, host_ret=pinned_ret)
    h0, d0 = g.transfer_bytes()
    e2e_times = []
    ret_hash = None
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = g.pi_compute(digits, ctx, host_digits=pinned, host_ret=pinned_ret)
        torch.cuda.synchronize()
        e2e_times.append((time.perf_counter() - t0) * 1e3)
    h1, d1 = g.transfer_bytes()
    sys.path.insert(0, str(ROOT / "oracle"))
    head = bytes(pinned[:50].numpy()).decode()
    if head != "14159265358979323846264338327950288419716939937510"[:min(50, digits)]:
        raise SystemExit(f"bench: digits do not start like pi: {head}")
    from pi_ref import mod_hash
    ret_hash = mod_hash(r.ret)
    # RET must be the reference build's, recorded on a B200 by
    # oracle/make_ref_fixtures.py (pi_bs_gpu.cu:2216-2224 hash)
    fx = _ref_fixture(digits)
    if fx is not None and (fx["ret_hash"] != ret_hash or fx["ret_len"] != r.ret_len):
        raise SystemExit(f"bench: RET (len {r.ret_len}, hash {ret_hash}) differs from the reference build's "
                         f"(len {fx['ret_len']}, hash {fx['ret_hash']})")
    e2e = _max_over_ranks(statistics.mean(e2e_times), ws)

    # independent check of RET: BBP hex digits at 64 seeded positions
    # (integer fixed point on the GPU), outside the timed regions
    bbp = None
    if rank == 0:
        rng = random.Random(0xBB964)
        top = 8 * (r.ret_len - 1) - 64
        positions = sorted(rng.randrange(0, top) for _ in range(BBP_POSITIONS))
        t0 = time.perf_counter()
        bad, unsure = g.bbp_spot_check(r.ret, positions)
        bbp = {"positions": len(positions), "hex_digits_each": 6, "mismatches": len(bad),
               "inconclusive": len(unsure), "seconds": round(time.perf_counter() - t0, 2),
               "max_position": positions[-1]}

    # roofline of the dominant kernel family
    peaks = _peaks()
    dom = max(ktimes.items(), key=lambda kv: kv[1][1]) if ktimes else None
    total_kernel_ms = sum(v[1] for v in ktimes.values())
    roof = None
    if dom:
        name, (n, kms, kbytes) = dom
        achieved = kbytes / (kms * 1e-3) / 1e9
        ratio = NCU_TRAFFIC_RATIO.get(name)
        roof = {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"],
                "traffic": (ratio * kbytes / n) if ratio else None,
                "traffic_unit": "bytes per launch (DRAM read + write)",
                "traffic_source": NCU_TRAFFIC_SOURCE.get(name),
                "launches_per_step": n / args.steps, "share_of_kernel_time": kms / total_kernel_ms,
                "peak_source": "measured" if not peaks.get("fallback") else "fallback"}
    families = {k: {"launches_per_step": v[0] / args.steps, "ms_per_step": v[1] / args.steps,
                    "GBps": (v[2] / (v[1] * 1e-3) / 1e9) if v[1] > 0 else None} for k, v in ktimes.items()}
    # integer roofline of each family: t_min = max(IMAD / IMAD peak, ALU /
    # ALU peak, all / issue peak) from the instruction counts per byte
    ipk = g.int_peak()
    pim, pal = ipk["imad_winst_per_s"], ipk["alu_winst_per_s"]
    for k, f in families.items():
        ir = INT_WINST_PER_BYTE.get(k)
        n, kms, kbytes = ktimes[k]
        if ir and kms > 0:
            tmin = max(ir[0] * kbytes / pim, ir[1] * kbytes / pal, ir[2] * kbytes / (pim + pal))
            f["int_roofline_frac"] = tmin / (kms * 1e-3)
    roof_int = None
    if dom and dom[0] in INT_WINST_PER_BYTE:
        name, (n, kms, kbytes) = dom
        ir = INT_WINST_PER_BYTE[name]
        achieved = ir[2] * kbytes / (kms * 1e-3)
        roof_int = {"bound": "integer issue", "kernel": name, "achieved": achieved, "peak": pim + pal,
                    "unit": "warp instructions/s", "frac": families[name]["int_roofline_frac"],
                    "imad_pipe_frac": ir[0] * kbytes / (kms * 1e-3) / pim,
                    "alu_pipe_frac": ir[1] * kbytes / (kms * 1e-3) / pal,
                    "peaks_measured": {"imad_winst_per_s": pim, "alu_winst_per_s": pal,
                                       "how": "gpupi_int_peak (csrc/int_peak.cu) in this run"},
                    "source": INT_SOURCE,
                    "note": "the binding roofline of the NTT passes; roofline (HBM) above is the contract's"}

    if rank != 0:
        return
    cpu = cpu_baseline_sample(CPU_SAMPLE_DIGITS) if (ws == 1 and not args.no_cpu) else None
    # gpupi's own CUDA build beside this library's CLI: cold processes,
    # alternating, same digits, each program's own elapsed_ms
    refcli = None
    if ws == 1 and args.ref_cli_runs > 0 and REF_CLI.exists() and OUR_CLI.exists():
        theirs, ours = [], []
        for _ in range(args.ref_cli_runs):
            theirs.append(_cli_benchmark(REF_CLI, digits, local))
            ours.append(_cli_benchmark(OUR_CLI, digits, local))
        tm = statistics.median(x["elapsed_ms"] for x in theirs)
        om = statistics.median(x["elapsed_ms"] for x in ours)
        refcli = {"reference_elapsed_ms": [round(x["elapsed_ms"], 3) for x in theirs],
                  "ours_elapsed_ms": [round(x["elapsed_ms"], 3) for x in ours],
                  "reference_median_ms": tm, "ours_median_ms": om, "reference_over_ours": tm / om,
                  "ret_hash_equal": all(a["ret_hash"] == b["ret_hash"] == ret_hash and a["ret_len"] == b["ret_len"]
                                        for a, b in zip(theirs, ours)),
                  "how": f"pi_bs_gpu_ref {digits} --benchmark (gpupi built from its sources, oracle/build_ref.py) "
                         f"and gpupi_b200/pi_bs_gpu {digits} --benchmark, alternating cold processes"}
    line = {
        "metric": METRIC, "value": ms, "unit": "ms", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (pi has no input data)",
        "config": {"workload": f"pi to {digits} decimal digits (pi_bs_gpu {digits})", "digits": digits,
                   "form": "tuned (forward transforms shared within each merge level of the splitting tree; "
                           "otherwise the reference's op sequence, one op per launch, compact after every op)",
                   "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
                   "l2": "working set (tens of GB) larger than L2; no flush needed"},
        "whole_job": {"digits_per_s": ws * digits / (ms * 1e-3), "pi_runs_per_s": ws / (ms * 1e-3),
                      "note": "each GPU computes its own 1e9-digit pi per step (replicas); value is the "
                              "max-over-ranks time of one step, so ideal weak scaling keeps it constant"},
        "forms": {"tuned_ms": ms, "plain_ms": ms_plain, "plain_over_tuned": ms_plain / ms,
                  "plain_ret_len": rp.ret_len},
        "pipeline_elapsed_ms": statistics.mean(inner),
        "step_ms": [round(x, 3) for x in inner],
        "ms_per_step_with_kernel_timers": ms_timed_local,
        "ret_len": r.ret_len, "ret_hash": ret_hash, "convert_digits": r.convert_digits,
        "e2e": {"value": e2e, "unit": "ms", "h2d_bytes_per_step": (h1 - h0) // args.steps,
                "d2h_bytes_per_step": (d1 - d0) // args.steps},
        "gpu_launches": launches,
        "tree_graph": dict(g.tree_graph_stats(), note="splitting tree as a CUDA graph: recorded and captured in the "
                                                       "warm-up, replayed in the timed steps"),
        "roofline": roof,
        "roofline_int": roof_int,
        "kernel_families": families,
        "launch_gaps": {
            "device_ms_per_step": sum(v[1] for v in kgaps.values()) / args.steps,
            "top": {k: {"per_step": v[0] / args.steps, "device_ms": v[1] / args.steps,
                        "host_ms": v[2] / args.steps}
                    for k, v in sorted(kgaps.items(), key=lambda kv: -kv[1][1])[:8]}},
        "clocks": clk,
        "cpu_baseline": cpu,
        "bbp_check": bbp,
        "ref_fixture": (None if fx is None else {"ret_hash": fx["ret_hash"], "ret_len": fx["ret_len"],
                                                   "match": True, "source": "tests/golden/ref_fixtures.json"}),
        "reference_gpu_build": refcli,
    }
    print(json.dumps(line), flush=True)
    ctx.close()


def run_ntt(args, ws, rank, local):
    """One batched NTT product of two ntt_limbs-limb operands per step (the
    2^27 x 2^27-limb configuration by default), operands resident in HBM."""
    import torch
    import gpupi_b200 as g

    torch.cuda.set_device(local)
    ctx = g.Context()
    L = args.ntt_limbs
    gen = torch.Generator(device="cuda")
    gen.manual_seed(0x4D595DF4)
    A = torch.randint(-2 ** 31, 2 ** 31 - 1, (L,), dtype=torch.int32, device="cuda", generator=gen)
    B = torch.randint(-2 ** 31, 2 ** 31 - 1, (L,), dtype=torch.int32, device="cuda", generator=gen)
    C = torch.zeros(2 * L, dtype=torch.int32, device="cuda")

    def step():
        if args.ntt_path == "spectra":   # split row passes (the tuned form's building block)
            ctx.mul_spectra(1, A.data_ptr(), L, B.data_ptr(), L, C.data_ptr(), 2 * L)
        else:
            ctx.mul(1, A.data_ptr(), L, L, B.data_ptr(), L, L, C.data_ptr(), 2 * L, 2 * L)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    g.timer_reset()
    g.timer_enable(True)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    g.timer_enable(False)
    ms = _max_over_ranks(e0.elapsed_time(e1) / args.steps, ws)
    fam = {k: {"launches_per_step": v[0] / args.steps, "ms_per_step": v[1] / args.steps,
               "GBps": v[2] / (v[1] * 1e-3) / 1e9 if v[1] > 0 else None} for k, v in g.timer_report().items()}
    if rank == 0:
        print(json.dumps({"metric": f"ms per {L}x{L}-limb NTT product ({args.ntt_path})", "value": ms, "unit": "ms",
                          "steps": args.steps, "warmup": args.warmup, "dtype": "u32",
                          "a_b_ret_GBps": 16.0 * L / (ms * 1e-3) / 1e9, "kernel_families": fam}), flush=True)
    ctx.close()


def run_convert(args, ws, rank, local):
    """Decimal conversion of a seeded 2^25-limb binary fraction (2^30 input
    bits) to 308 * 2^20 = 322,961,408 digits (leaf 308, 20 levels), input
    and digits resident in HBM."""
    import torch
    import gpupi_b200 as g

    torch.cuda.set_device(local)
    ctx = g.Context()
    L = 1 << 25
    leaf, levels = 308, 20
    total = leaf << levels
    gen = torch.Generator(device="cuda")
    gen.manual_seed(0xC4)
    X = torch.randint(-2 ** 31, 2 ** 31 - 1, (L,), dtype=torch.int32, device="cuda", generator=gen)
    out = torch.empty(total, dtype=torch.uint8, device="cuda")
    for _ in range(args.warmup):
        ctx.convert_decimal(X.data_ptr(), L, 32 * L, total, leaf, out.data_ptr())
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        ctx.convert_decimal(X.data_ptr(), L, 32 * L, total, leaf, out.data_ptr())
    e1.record()
    torch.cuda.synchronize()
    ms = _max_over_ranks(e0.elapsed_time(e1) / args.steps, ws)
    head = bytes(out[:16].cpu().numpy())
    if rank == 0:
        print(json.dumps({"metric": f"ms to convert a {L}-limb fraction to {total} decimal digits", "value": ms,
                          "unit": "ms", "steps": args.steps, "warmup": args.warmup, "dtype": "u32",
                          "digits_per_s": total / (ms * 1e-3), "first_digits": head.decode("ascii", "replace")}),
              flush=True)
    ctx.close()


def run_intpeak(args, ws, rank, local):
    """The integer-pipe peaks every limb kernel is measured against."""
    import torch
    import gpupi_b200 as g
    torch.cuda.set_device(local)
    runs = [g.int_peak() for _ in range(max(1, args.steps))]
    best = {k: max(r[k] for r in runs) for k in runs[0]}
    if rank == 0:
        print(json.dumps({"metric": "integer-pipe peak (warp instructions per second)", "value": best["imad_winst_per_s"],
                          "unit": "warp IMAD/s", "alu_winst_per_s": best["alu_winst_per_s"], "steps": len(runs),
                          "how": "eight independent mad.lo.u32 (lop3.b32) chains per thread, 2 x 1024 threads "
                                 "per SM, CUDA events (csrc/int_peak.cu)"}), flush=True)


def run_mulsmall(args, ws, rank, local):
    """One batch of equal products through each product kernel: the
    CUDA-core schoolbook, the tensor-core schoolbook (tcgen05 int8) and the
    NTT, operands resident in HBM, results compared word for word."""
    import torch
    import gpupi_b200 as g
    torch.cuda.set_device(local)
    ctx = g.Context()
    L, N = args.mul_limbs, args.mul_batch
    La, Lb = L // 2, L - L // 2
    gen = torch.Generator(device="cuda")
    gen.manual_seed(0xB5)
    A = torch.randint(-2 ** 31, 2 ** 31 - 1, (N * La,), dtype=torch.int32, device="cuda", generator=gen)
    B = torch.randint(-2 ** 31, 2 ** 31 - 1, (N * Lb,), dtype=torch.int32, device="cuda", generator=gen)
    outs, times = {}, {}
    kernels = {"ntt": lambda C: ctx.mul_ntt(N, A.data_ptr(), La, La, B.data_ptr(), Lb, Lb, C.data_ptr(), L)}
    if L <= 1024:
        kernels["school"] = lambda C: g.mul_naive(N, A.data_ptr(), La, La, B.data_ptr(), Lb, Lb, C.data_ptr(), L)
    if min(La, Lb) <= 2048 and L <= 8192:
        kernels["tc"] = lambda C: g.mul_tc(N, A.data_ptr(), La, La, B.data_ptr(), Lb, Lb, C.data_ptr(), L)
    for name, f in kernels.items():
        C = torch.zeros(N * L, dtype=torch.int32, device="cuda")
        for _ in range(args.warmup):
            f(C)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            f(C)
        e1.record()
        torch.cuda.synchronize()
        times[name] = _max_over_ranks(e0.elapsed_time(e1) / args.steps, ws)
        outs[name] = C
    same = all(torch.equal(outs[k], outs["ntt"]) for k in outs)
    macs = 16.0 * La * Lb * N   # byte products of the split-integer form
    if rank == 0:
        print(json.dumps({"metric": f"ms for {N} products of {La} x {Lb} limbs", "value": times.get("tc"),
                          "unit": "ms", "steps": args.steps, "warmup": args.warmup, "dtype": "u32",
                          "ms": times, "results_equal": same, "tc_error": g.tc_error(),
                          "tc_useful_int8_macs_per_s": macs / (times["tc"] * 1e-3) if "tc" in times else None}),
              flush=True)
    ctx.close()


def run_uneven(args, ws, rank, local):
    """4096 independent products with lengths log-uniform in [8, 4096] limbs
    per operand (seeded), operands resident in HBM: one ragged call
    (bucketed: schoolbook launch + NTT per transform size) against one
    batch_mp_mul call per pair, the form gpupi's API allows."""
    import numpy as np
    import torch
    import gpupi_b200 as g

    torch.cuda.set_device(local)
    ctx = g.Context()
    rng = np.random.default_rng(0xC2)
    n = 4096
    La = np.floor(2 ** rng.uniform(3, 12, size=n)).astype(np.uint32)
    Lb = np.floor(2 ** rng.uniform(3, 12, size=n)).astype(np.uint32)
    offA = np.concatenate([[0], np.cumsum(La.astype(np.uint64))[:-1]]).astype(np.uint64)
    offB = np.concatenate([[0], np.cumsum(Lb.astype(np.uint64))[:-1]]).astype(np.uint64)
    Lc = La.astype(np.uint64) + Lb
    offC = np.concatenate([[0], np.cumsum(Lc)[:-1]]).astype(np.uint64)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(0xC2)
    A = torch.randint(-2 ** 31, 2 ** 31 - 1, (int(La.sum()),), dtype=torch.int32, device="cuda", generator=gen)
    B = torch.randint(-2 ** 31, 2 ** 31 - 1, (int(Lb.sum()),), dtype=torch.int32, device="cuda", generator=gen)
    C = torch.zeros(int(Lc.sum()), dtype=torch.int32, device="cuda")
    C2 = torch.zeros_like(C)

    def ragged():
        ctx.mul_ragged(A.data_ptr(), offA, La, B.data_ptr(), offB, Lb, C.data_ptr(), offC)

    def per_pair():
        for i in range(n):
            ctx.mul(1, A.data_ptr() + 4 * int(offA[i]), int(La[i]), int(La[i]),
                    B.data_ptr() + 4 * int(offB[i]), int(Lb[i]), int(Lb[i]),
                    C2.data_ptr() + 4 * int(offC[i]), int(Lc[i]), int(Lc[i]))

    def timed(f):
        for _ in range(args.warmup):
            f()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            f()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps

    ms_r = _max_over_ranks(timed(ragged), ws)
    ms_p = _max_over_ranks(timed(per_pair), ws)
    same = bool(torch.equal(C, C2))
    if rank == 0:
        print(json.dumps({"metric": "ms for 4096 uneven products (log-uniform 8..4096 limbs per operand)",
                          "value": ms_r, "unit": "ms", "steps": args.steps, "warmup": args.warmup, "dtype": "u32",
                          "plain_per_pair_ms": ms_p, "speedup_vs_per_pair": ms_p / ms_r,
                          "limb_products": int((La.astype(np.uint64) * Lb).sum()), "results_equal": same}),
              flush=True)
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--digits", type=int, default=1_000_000_000)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--workload", choices=["pi", "ntt", "convert", "uneven", "intpeak", "mulsmall"], default="pi",
                    help="pi: the pi_bs_gpu pipeline (default); ntt: one large product per step; "
                         "convert: one 2^25-limb decimal conversion per step; uneven: 4096 uneven products; "
                         "intpeak: the integer-pipe peaks; mulsmall: one batch of equal products through "
                         "each product kernel")
    ap.add_argument("--mul-limbs", type=int, default=1024, help="mulsmall: L_a + L_b")
    ap.add_argument("--mul-batch", type=int, default=16384, help="mulsmall: products per batch")
    ap.add_argument("--ntt-limbs", type=int, default=1 << 27)
    ap.add_argument("--ntt-path", choices=["fused", "spectra"], default="fused",
                    help="ntt workload: fused row pass, or forward / inverse spectra")
    ap.add_argument("--ref-cli-runs", type=int, default=3,
                    help="pi workload: cold runs each of gpupi's own build and this library's CLI (0: skip)")
    args = ap.parse_args()
    ws, rank, local = _dist()
    if args.impl == "reference":
        # rank 0 alone runs the reference; the other ranks exit without work
        # (no process group: nothing is exchanged)
        run_reference_arm(args, ws, rank, local)
        return
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        # NCCL between the GPUs; gloo when there is no GPU (the reference arm
        # and the multi-rank plumbing run on host cores)
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    ok = False
    try:
        if args.workload == "ntt":
            run_ntt(args, ws, rank, local)
        elif args.workload == "convert":
            run_convert(args, ws, rank, local)
        elif args.workload == "uneven":
            run_uneven(args, ws, rank, local)
        elif args.workload == "intpeak":
            run_intpeak(args, ws, rank, local)
        elif args.workload == "mulsmall":
            run_mulsmall(args, ws, rank, local)
        else:
            run_ours(args, ws, rank, local)
        ok = True
    finally:
        if ws > 1:
            import torch.distributed as dist
            # the closing barrier only on success: a rank that failed must
            # not wait in it while its peers sit in a different collective
            if ok:
                dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
