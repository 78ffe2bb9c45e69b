"""The AUTO front end (mgxbench_b200.predictive): report schema, ranking rule and grid choice,
on a synthetic sweep database with the regression model (no GPU needed).  The keys follow
MGXBench's autotuning_prediction.json (autotuning/predictive.py:627-631)."""
import json
import math
import types

import pytest

from mgxbench_b200 import autotune as at
from mgxbench_b200 import predictive as pr


def _synthetic_db(path):
    """Runtime ~ c * MNK with Ozaki cheaper per split at large sizes; error falls 100x per split."""
    db = at.SweepDB(path)
    rows = []
    for i, d in enumerate((256, 512, 1024, 2048, 4096, 8192, 16384)):
        for c in at.candidates():
            mnk = float(d) ** 3
            if c.is_fp64:
                t, e = 2 * mnk / 35e12 / min(c.ksplit or 4, 4) ** (0.5 if d < 1024 else 0.0) + 2e-5, 3e-16
            else:
                t, e = c.splits * (c.splits + 1) / 2 * 2 * mnk / 3e15 + 1e-4, 10.0 ** (-8 - 2 * (c.splits - 3)) * 3
            rows.append({"m": d, "n": d, "k": d, "exp_range": 10, "tile": c.tile, "splits": c.splits,
                         "seconds": t, "error": max(e, at.ERROR_FLOOR), "set": "train"})
    db.add(rows)
    return path


def _args(tmp_path, **kw):
    a = dict(decomposition="1d", ranks=4, size=16384, grid_rows=None, grid_cols=None,
             prediction_model="extrapolation", auto_model=None, db=str(tmp_path / "db.jsonl"), auto_validate=False,
             auto_feedback=False, build_dir="build", output=str(tmp_path / "out"), warmup=1, repeats=1,
             timeout=60, exp_range=10, target=1e-15, project_root=str(tmp_path))
    a.update(kw)
    return types.SimpleNamespace(**a)


def test_auto_report_schema_and_choice(tmp_path, capsys):
    _synthetic_db(tmp_path / "db.jsonl")
    assert pr.auto(_args(tmp_path)) == 0
    rep = json.loads((tmp_path / "out" / "autotuning_prediction.json").read_text())
    for key in ("size", "ranks", "decomposition", "architecture_id", "best", "ranking", "speedup_vs_MPI_predicted",
                "prediction_model", "calibration_file", "status", "measured"):
        assert key in rep
    assert rep["status"] == "PREDICTED" and rep["measured"] is False
    assert rep["prediction_model"] == "loglog-regression"
    best = rep["best"]
    # at 16384^3 the fastest candidate meeting 1e-15 is the Ozaki form with the fewest adequate splits
    assert best["meets_target"] and best["form"] == "ozaki"
    feas = [r for r in rep["ranking"] if r["meets_target"]]
    assert [r["predicted_s"] for r in feas] == sorted(r["predicted_s"] for r in feas)
    assert rep["ranking"][:len(feas)] == feas
    assert all(r["predicted_error"] <= 1e-15 for r in feas)
    assert rep["speedup_vs_fp64_predicted"] > 1.0
    out = capsys.readouterr().out
    assert "AUTOTUNING REPORT" in out and "Predicted Time" in out


def test_auto_small_problem_prefers_fp64(tmp_path):
    _synthetic_db(tmp_path / "db.jsonl")
    assert pr.auto(_args(tmp_path, size=256)) == 0
    rep = json.loads((tmp_path / "out" / "autotuning_prediction.json").read_text())
    assert rep["best"]["form"] == "fp64"


def test_auto_2d_grid_and_extrapolation(tmp_path):
    _synthetic_db(tmp_path / "db.jsonl")
    assert pr.auto(_args(tmp_path, decomposition="2d", ranks=6, size=65536)) == 0
    rep = json.loads((tmp_path / "out" / "autotuning_prediction.json").read_text())
    assert (rep["best"]["grid_rows"], rep["best"]["grid_cols"]) == (2, 3)
    assert rep["best"]["extrapolated"] is True


def test_grid_shape_matches_dims_create():
    assert pr.grid_shape(1) == (1, 1)
    assert pr.grid_shape(4) == (2, 2)
    assert pr.grid_shape(8) == (2, 4)
    assert pr.grid_shape(15) == (3, 5)
    assert pr.grid_shape(7) == (1, 7)
    assert pr.grid_shape(12, 4, 3) == (4, 3)


def test_auto_without_model_is_an_error(tmp_path, capsys):
    rc = pr.auto(_args(tmp_path, prediction_model="ml", auto_model=str(tmp_path / "none.json")))
    assert rc == 2
    assert "AUTO:" in capsys.readouterr().err


def test_cli_argument_checks(tmp_path):
    with pytest.raises(SystemExit):
        pr.main(["auto", "--decomposition", "2d", "--ranks", "4", "--size", "64", "--grid-rows", "3",
                 "--grid-cols", "2"])
    with pytest.raises(SystemExit):
        pr.main(["auto", "--decomposition", "1d", "--ranks", "4", "--size", "64", "--auto-feedback"])


def test_auto_accepts_benchmark_py_namespace(tmp_path):
    """benchmark.py --libraries AUTO passes its own parsed arguments (benchmark.py:52-80, 83-85)."""
    _synthetic_db(tmp_path / "db.jsonl")
    ns = types.SimpleNamespace(decomposition="2d", size=8192, ranks=4, libraries=["AUTO"], warmup=2,
                               warmup_mode="external", retries=0, repeats=5, launcher="mpirun", launcher_args="",
                               build_dir="build", output=str(tmp_path / "results"), timeout=600, plot=False,
                               inner_loops=1, environment=None, label="default", device_map="local",
                               grid_rows=None, grid_cols=None, summa_bk=512, prediction_model="extrapolation",
                               auto_model=None, auto_validate=False, auto_feedback=False, db=str(tmp_path / "db.jsonl"))
    assert pr.auto(ns) == 0
    rep = json.loads((tmp_path / "results" / "autotuning_prediction.json").read_text())
    assert rep["best"]["summa_bk"] == 512 and rep["best"]["grid_rows"] * rep["best"]["grid_cols"] == 4
