"""Records what the drop-in executables print when MGXBench's benchmark.py drives them.

benchmark.py builds one MPMD command per repetition (benchmark.py:127-130),
    <launcher> -np 1 EXE auto N LIB : -np 1 EXE auto N LIB : ...
with MGXBENCH_INNER_LOOPS and MGXBENCH_INTERNAL_WARMUP in the environment, and for 2D also
MGXBENCH_GRID_ROWS/COLS and MGXBENCH_SUMMA_BK (benchmark.py:113-119).  It accepts a run when
exactly one BENCHMARK_RESULT record is printed (45-50), the exit status is 0, valid=1, size,
ranks and library match, decomposition (case-insensitive) and loops match, and seconds is a
positive finite number (147-156).  `run_case` issues that command against build/mm_1d or
build/mm_2d through mgxbench_b200/mgx-onegpu-launch on the GPU; `accepts` restates the checks.

    python tests/golden/make_dropin_records.py tests/golden/dropin_records.json

writes the records (on a GPU box) that tests/test_dropin_contract.py replays through the
unmodified benchmark.py where MGXBench's sources are present.
"""
import json
import math
import os
import re
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
LAUNCHER = ROOT / "mgxbench_b200" / "mgx-onegpu-launch"
BUILD = ROOT / "build"

# (decomposition, size, ranks, library, grid rows, grid cols, SUMMA BK)
CASES = [("1d", 1024, 4, "MMM", None, None, None), ("1d", 1024, 4, "SSS", None, None, None),
         ("2d", 1024, 4, "MMM", 2, 2, 256), ("2d", 1024, 4, "NNN", 2, 2, 256)]


def benchmark_command(decomposition, size, ranks, lib):
    exe = BUILD / ("mm_1d" if decomposition == "1d" else "mm_2d")
    cmd = [sys.executable, str(LAUNCHER)]
    for r in range(ranks):
        if r:
            cmd.append(":")
        cmd += ["-np", "1", str(exe), "auto", str(size), lib]
    return cmd


def benchmark_env(decomposition, grid_rows=None, grid_cols=None, summa_bk=256, inner_loops=1):
    env = dict(os.environ)
    if decomposition == "2d":
        env["MGXBENCH_GRID_ROWS"] = str(grid_rows)
        env["MGXBENCH_GRID_COLS"] = str(grid_cols)
        env["MGXBENCH_SUMMA_BK"] = str(summa_bk)
    env["MGXBENCH_INNER_LOOPS"] = str(inner_loops)
    env["MGXBENCH_INTERNAL_WARMUP"] = "0"
    return env


def accepts(output, returncode, decomposition, size, ranks, lib, inner_loops=1):
    """benchmark.py's acceptance of one run: returns (ok, reason)."""
    found = re.findall(r"BENCHMARK_RESULT\s+([^\r\n]+)", output)
    if len(found) != 1:
        return False, f"{len(found)} BENCHMARK_RESULT records"
    rec = dict(x.split("=", 1) for x in found[0].split())
    if returncode != 0 or rec.get("valid") != "1":
        return False, f"exit {returncode}, valid={rec.get('valid')}"
    if int(rec["size"]) != size or int(rec["ranks"]) != ranks or rec["library"] != lib:
        return False, "metadata mismatch"
    if rec.get("decomposition", "").lower() != decomposition or int(rec.get("loops", 0)) != inner_loops:
        return False, "decomposition/inner-loop mismatch"
    t = float(rec["seconds"])
    if not math.isfinite(t) or t <= 0:
        return False, "invalid time"
    return True, "accepted"


def run_case(decomposition, size, ranks, lib, grid_rows=None, grid_cols=None, summa_bk=None, timeout=600):
    proc = subprocess.run(benchmark_command(decomposition, size, ranks, lib), capture_output=True, text=True,
                          timeout=timeout, env=benchmark_env(decomposition, grid_rows, grid_cols, summa_bk or 256))
    return {"decomposition": decomposition, "size": size, "ranks": ranks, "library": lib,
            "grid_rows": grid_rows, "grid_cols": grid_cols, "summa_bk": summa_bk,
            "returncode": proc.returncode, "stdout": proc.stdout, "stderr": proc.stderr}


def main(argv):
    out = Path(argv[1]) if len(argv) > 1 else ROOT / "tests" / "golden" / "dropin_records.json"
    records = [run_case(*c) for c in CASES]
    for r in records:
        ok, why = accepts(r["stdout"] + "\n" + r["stderr"], r["returncode"], r["decomposition"], r["size"],
                          r["ranks"], r["library"])
        if not ok:
            print(f"{r['decomposition']} {r['library']}: not accepted ({why})", file=sys.stderr)
            return 1
    out.write_text(json.dumps(records, indent=1) + "\n")
    print(f"wrote {len(records)} records to {out}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main(sys.argv))
