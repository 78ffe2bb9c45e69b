"""The drop-in boundary without a GPU: the one-GPU launcher, MGXBench's benchmark.py contract and
the executables' argument checks (1D-row-block/mmb.cu:185-236, 2D-block-matrix/mmb.cu:81-101)."""
import importlib.util
import json
import os
import re
import subprocess
import sys
from pathlib import Path

import pytest

from conftest import REFERENCE, ROOT

LAUNCHER = ROOT / "mgxbench_b200" / "mgx-onegpu-launch"
BUILD = ROOT / "build"
REFERENCE_BENCHMARK = REFERENCE / "benchmark.py"
RECORDS = ROOT / "tests" / "golden" / "dropin_records.json"
NO_REFERENCE = f"MGXBench sources not found at {REFERENCE} (set MGXBENCH_REFERENCE)"


def _load_launcher():
    spec = importlib.util.spec_from_loader("mgxlaunch", loader=None)
    mod = importlib.util.module_from_spec(spec)
    exec(LAUNCHER.read_text(), mod.__dict__)
    return mod


def test_launcher_counts_mpmd_segments():
    L = _load_launcher()
    argv = "-np 1 /x/mm_1d auto 64 MMM : -np 1 /x/mm_1d auto 64 MMM : -np 2 /x/mm_1d auto 64 MMM".split()
    ranks, cmd = L.parse(argv)
    assert ranks == 4 and cmd == ["/x/mm_1d", "auto", "64", "MMM"]
    ranks, cmd = L.parse("-np 1 /x/mm_2d 0 64 NNN : -np 1 /x/mm_2d 1 64 NNN".split())
    assert ranks == 2 and cmd[1] == "0"
    for bad in ("-np 1 /x/a auto 64 MMM : -np 1 /x/a auto 32 MMM", "-np 0 /x/a auto 64 MMM", "/x/a auto 64 MMM"):
        with pytest.raises((ValueError, IndexError)):
            L.parse(bad.split())


def _stub_exe(tmp_path):
    """An executable that reports the emulated rank count the way mm_1d does."""
    exe = tmp_path / "build" / "mm_1d"
    exe.parent.mkdir()
    exe.write_text("#!/usr/bin/env python3\nimport os,sys\nn=sys.argv[2];lib=sys.argv[3]\n"
                   "r=os.environ['MGXBENCH_EMULATED_RANKS']\nl=os.environ.get('MGXBENCH_INNER_LOOPS','10')\n"
                   "print(f'BENCHMARK_RESULT decomposition=1D library={lib} size={n} ranks={r} seconds=0.25 valid=1 "
                   "loops={l} form=fp64 tflops=1.0')\n")
    exe.chmod(0o755)
    return exe


def test_launcher_execs_one_process_with_rank_count(tmp_path):
    exe = _stub_exe(tmp_path)
    out = subprocess.run([sys.executable, str(LAUNCHER), "-np", "1", str(exe), "auto", "64", "SSS", ":",
                          "-np", "1", str(exe), "auto", "64", "SSS"], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    assert "ranks=2" in out.stdout and "library=SSS" in out.stdout


@pytest.mark.skipif(not REFERENCE_BENCHMARK.exists(), reason=NO_REFERENCE)
def test_reference_benchmark_drives_the_launcher(tmp_path):
    """MGXBench's unmodified benchmark.py accepts the one-GPU launcher and our result line."""
    exe = _stub_exe(tmp_path)
    cmd = [sys.executable, str(REFERENCE_BENCHMARK), "--decomposition", "1d", "--size", "64", "--ranks", "4",
           "--libraries", "MMM", "SSS", "--warmup", "0", "--repeats", "2", "--launcher", str(LAUNCHER),
           "--build-dir", str(exe.parent), "--output", str(tmp_path / "out")]
    out = subprocess.run(cmd, capture_output=True, text=True, cwd=str(REFERENCE_BENCHMARK.parent),
                         env=dict(os.environ, PYTHONDONTWRITEBYTECODE="1"))
    assert out.returncode == 0, out.stdout + out.stderr
    doc = json.loads(next((tmp_path / "out").rglob("benchmark.json")).read_text())
    assert [r["library"] for r in doc["results"]] == ["MMM", "SSS"]
    assert all(r["ranks"] == 4 and r["validated"] for r in doc["results"])


@pytest.mark.skipif(not (BUILD / "mm_1d").exists(), reason="executables not built")
def test_mm1d_argument_errors():
    r = subprocess.run([str(BUILD / "mm_1d")], capture_output=True, text=True)
    assert r.returncode == 1 and "Usage:" in r.stderr
    r = subprocess.run([str(BUILD / "mm_1d"), "0", "64", "MQZ"], capture_output=True, text=True)
    assert r.returncode == 1 and "Invalid communication string" in r.stderr


@pytest.mark.skipif(not (BUILD / "mm_2d").exists(), reason="executables not built")
def test_mm2d_argument_errors():
    r = subprocess.run([str(BUILD / "mm_2d"), "0", "64"], capture_output=True, text=True)
    assert r.returncode == 2 and "2D SUMMA: Usage: mm_2d" in r.stderr
    r = subprocess.run([str(BUILD / "mm_2d"), "0", "64", "MYC"], capture_output=True, text=True)
    assert r.returncode == 2 and "invalid matrix size or library" in r.stderr
    env = dict(os.environ, MGXBENCH_EMULATED_RANKS="3")
    r = subprocess.run([str(BUILD / "mm_2d"), "0", "64", "MMM"], capture_output=True, text=True, env=env)
    assert r.returncode == 2 and "N must be divisible" in r.stderr
    env = dict(os.environ, MGXBENCH_EMULATED_RANKS="4", MGXBENCH_GRID_ROWS="3")
    r = subprocess.run([str(BUILD / "mm_2d"), "0", "64", "MMM"], capture_output=True, text=True, env=env)
    assert r.returncode == 2 and "invalid process grid" in r.stderr


def _replay_exe(build_dir, decomposition, records):
    """An executable that prints what build/mm_1d or build/mm_2d printed on a GPU for the same
    size, emulated rank count and library (tests/golden/dropin_records.json), after checking the
    environment benchmark.py set."""
    exe = build_dir / ("mm_1d" if decomposition == "1d" else "mm_2d")
    table = {f"{r['size']}:{r['ranks']}:{r['library']}": r for r in records if r["decomposition"] == decomposition}
    exe.write_text("#!/usr/bin/env python3\nimport json,os,sys\n"
                   f"T=json.loads({json.dumps(json.dumps(table))})\n"
                   "r=T[f\"{sys.argv[2]}:{os.environ['MGXBENCH_EMULATED_RANKS']}:{sys.argv[3]}\"]\n"
                   "assert os.environ['MGXBENCH_INNER_LOOPS']=='1'\n"
                   "if r['grid_rows']:\n"
                   "    assert os.environ['MGXBENCH_GRID_ROWS']==str(r['grid_rows'])\n"
                   "    assert os.environ['MGXBENCH_GRID_COLS']==str(r['grid_cols'])\n"
                   "    assert os.environ['MGXBENCH_SUMMA_BK']==str(r['summa_bk'])\n"
                   "sys.stdout.write(r['stdout']);sys.stderr.write(r['stderr']);sys.exit(r['returncode'])\n")
    exe.chmod(0o755)
    return exe


@pytest.mark.skipif(not REFERENCE_BENCHMARK.exists(), reason=NO_REFERENCE)
@pytest.mark.skipif(not RECORDS.exists(), reason="no recorded executable output (tests/golden/make_dropin_records.py)")
@pytest.mark.parametrize("decomposition", ["1d", "2d"])
def test_reference_benchmark_accepts_the_executables_output(tmp_path, decomposition):
    """MGXBench's unmodified benchmark.py, through the one-GPU launcher, accepts what build/mm_1d
    and build/mm_2d printed on a B200 for the same command lines (recorded by
    tests/test_gpu_dropin.py / make_dropin_records.py)."""
    records = json.loads(RECORDS.read_text())
    mine = [r for r in records if r["decomposition"] == decomposition]
    assert mine
    build = tmp_path / "build"
    build.mkdir()
    _replay_exe(build, decomposition, records)
    libs = [r["library"] for r in mine]
    cmd = [sys.executable, str(REFERENCE_BENCHMARK), "--decomposition", decomposition, "--size", str(mine[0]["size"]),
           "--ranks", str(mine[0]["ranks"]), "--libraries", *libs, "--warmup", "1", "--repeats", "2",
           "--launcher", str(LAUNCHER), "--build-dir", str(build), "--output", str(tmp_path / "out")]
    if decomposition == "2d":
        cmd += ["--grid-rows", str(mine[0]["grid_rows"]), "--grid-cols", str(mine[0]["grid_cols"]),
                "--summa-bk", str(mine[0]["summa_bk"])]
    out = subprocess.run(cmd, capture_output=True, text=True, cwd=str(REFERENCE_BENCHMARK.parent),
                         env=dict(os.environ, PYTHONDONTWRITEBYTECODE="1"))
    assert out.returncode == 0, out.stdout + out.stderr
    doc = json.loads(next((tmp_path / "out").rglob("benchmark.json")).read_text())
    assert [r["library"] for r in doc["results"]] == libs
    assert all(r["validated"] and r["ranks"] == mine[0]["ranks"] for r in doc["results"])
    assert not doc["failures"]


@pytest.mark.skipif(not REFERENCE_BENCHMARK.exists(), reason=NO_REFERENCE)
def test_reference_benchmark_auto_through_the_forwarder(tmp_path):
    """`benchmark.py --libraries AUTO` imports autotuning.predictive.auto (benchmark.py:83-85).
    A copy of MGXBench's driver files, made here for the test only, with this library's
    mgxbench_b200/dropin/autotuning/ in place of its own, reaches the learned cost model's
    AUTO report (extrapolation model: no GPU needed)."""
    import shutil
    tree = tmp_path / "mgxbench"
    tree.mkdir()
    shutil.copy(REFERENCE_BENCHMARK, tree / "benchmark.py")
    shutil.copytree(REFERENCE / "configuration", tree / "configuration")
    shutil.copytree(ROOT / "mgxbench_b200" / "dropin" / "autotuning", tree / "autotuning")
    cmd = [sys.executable, str(tree / "benchmark.py"), "--decomposition", "2d", "--size", "8192", "--ranks", "4",
           "--libraries", "AUTO", "--prediction-model", "extrapolation", "--output", str(tmp_path / "auto")]
    out = subprocess.run(cmd, capture_output=True, text=True, cwd=str(tree),
                         env=dict(os.environ, PYTHONDONTWRITEBYTECODE="1", MGXBENCH_B200_ROOT=str(ROOT)))
    assert out.returncode == 0, out.stdout + out.stderr
    assert "AUTOTUNING REPORT" in out.stdout
    rep = json.loads((tmp_path / "auto" / "autotuning_prediction.json").read_text())
    assert rep["status"] == "PREDICTED" and rep["best"]["form"] in ("fp64", "ozaki", "crt")
    assert rep["decomposition"] == "2d" and rep["ranks"] == 4
