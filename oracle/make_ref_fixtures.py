"""Generate tests/golden/ref_fixtures.json by running the reference build
(test infrastructure only; needs a GPU and oracle/_ref built by
oracle/build_ref.py from the reference's own sources).

For each pi size it runs the reference's CLI, ``pi_bs_gpu_ref <digits>
--benchmark`` (pi_bs_gpu.cu:2073-2431), and records its result line fields
(RET_len, convert_digits), the RET preview line with its mod-1e9+7 hash, the
DEC preview line, and the SHA-256 and size of its whole stdout ("3" + digits
+ newline).  For the batched configurations it runs
``ref_configs_ref c2 | c3 27 | c4`` (oracle/ref_configs.cu linked with the
reference's objects; inputs from the splitmix64 streams of
oracle/ref_inputs.py) and records the digest of the raw result.

    python oracle/make_ref_fixtures.py [--out FILE] [--pi 1000000,...] [--configs c2,c3,c4]
"""
from __future__ import annotations

import argparse
import hashlib
import json
import subprocess
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
REF = HERE / "_ref"


def stream_digest(cmd: list[str], timeout: float = 1200.0) -> dict:
    """Run cmd, hashing its stdout as it streams; returns the digest, the
    first / last 16 bytes, stderr and the wall time."""
    t0 = time.time()
    p = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE)
    h = hashlib.sha256()
    n = 0
    head = b""
    tail = b""
    while True:
        chunk = p.stdout.read(1 << 24)
        if not chunk:
            break
        if len(head) < 16:
            head = (head + chunk)[:16]
        tail = (tail + chunk)[-16:]
        h.update(chunk)
        n += len(chunk)
    err = p.stderr.read().decode()
    rc = p.wait(timeout=timeout)
    if rc != 0:
        raise RuntimeError(f"{cmd} exited {rc}: {err[-2000:]}")
    return {"sha256": h.hexdigest(), "bytes": n, "head": head.hex(), "tail": tail.hex(), "stderr": err,
            "wall_s": round(time.time() - t0, 2)}


def parse_result_line(line: str) -> dict:
    out = {}
    for kv in line.split():
        if "=" in kv:
            k, v = kv.split("=", 1)
            out[k] = v
    return out


def pi_fixture(digits: int) -> dict:
    exe = str(REF / "pi_bs_gpu_ref")
    # --benchmark prints three stdout lines: the result line (with
    # workspace_max), "RET = <preview> hash = h" and "DEC = 3<63>...<64>"
    bench = subprocess.run([exe, str(digits), "--benchmark"], capture_output=True, text=True, check=True)
    lines = [l for l in bench.stdout.splitlines() if l.strip()]
    f = parse_result_line(next(l for l in lines if l.startswith("target_digits=")))
    ret_line = next(l for l in lines if l.startswith("RET = "))
    dec_line = next((l for l in lines if l.startswith("DEC = ")), None)
    # default mode: "3" + every digit + newline on stdout, result line on stderr
    d = stream_digest([exe, str(digits)])
    f2 = parse_result_line(next(l for l in d["stderr"].splitlines() if l.startswith("target_digits=")))
    return {"digits": digits, "ret_len": int(f["RET_len"]), "convert_digits": int(f["convert_digits"]),
            "ret_line": ret_line, "ret_hash": int(ret_line.rsplit("=", 1)[1]), "dec_line": dec_line,
            "stdout_sha256": d["sha256"], "stdout_bytes": d["bytes"],
            "ref_elapsed_ms": [float(f["elapsed_ms"]), float(f2["elapsed_ms"])],
            "workspace_max": f.get("workspace_max")}


def config_fixture(name: str, args: list[str]) -> dict:
    d = stream_digest([str(REF / "ref_configs_ref"), name, *args])
    ms = None
    for l in d["stderr"].splitlines():
        if l.startswith("elapsed_ms="):
            ms = float(l.split("=", 1)[1])
    return {"config": name, "args": args, "sha256": d["sha256"], "bytes": d["bytes"], "head": d["head"],
            "tail": d["tail"], "ref_elapsed_ms": ms}


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(ROOT / "tests" / "golden" / "ref_fixtures.json"))
    ap.add_argument("--pi", default="1000000,10000000,100000000,1000000000")
    ap.add_argument("--configs", default="c2,c3,c4")
    a = ap.parse_args()
    out = {"generator": "oracle/make_ref_fixtures.py (reference build: oracle/build_ref.py)", "pi": [],
           "configs": {}}
    for d in [int(x) for x in a.pi.split(",") if x]:
        fx = pi_fixture(d)
        print(json.dumps(fx), flush=True)
        out["pi"].append(fx)
    for c in [x for x in a.configs.split(",") if x]:
        fx = config_fixture(c, ["27"] if c == "c3" else [])
        print(json.dumps(fx), flush=True)
        out["configs"][c] = fx
    Path(a.out).write_text(json.dumps(out, indent=1) + "\n")
    print("wrote", a.out)
    return 0


if __name__ == "__main__":
    sys.exit(main())
