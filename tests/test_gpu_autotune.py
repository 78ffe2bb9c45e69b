"""The learned cost model on the GPU: the executables' MGXBENCH_FORM=auto choice (C++ host,
inference through mgx_mlp_forward) agrees with the Python rule, and the network trained by the
library's own kernels on the measured sweep chooses better than the regression baseline."""
import json
import os
import re
import subprocess
import sys
from pathlib import Path

import pytest

from conftest import ROOT
from test_autotune import synthetic_rows

pytestmark = pytest.mark.gpu

DATA = ROOT / "mgxbench_b200" / "data"


def _train_toy(tmp_path, epochs=150):
    from mgxbench_b200 import autotune as at
    shapes = at.random_shapes(300, seed=5)
    rows = synthetic_rows(shapes, seed=5)
    mdl = at.MlpModel().fit(rows, epochs=epochs, batch=256)
    path = tmp_path / "toy_mlp.json"
    mdl.save(path, "toy")
    return at.MlpModel.load(path), path


@pytest.mark.parametrize("exe,n,er", [("mm_1d", 512, 0), ("mm_1d", 4096, 30), ("mm_2d", 1536, 12)])
def test_executable_auto_form_matches_python_choice(tmp_path, exe, n, er):
    from mgxbench_b200 import autotune as at
    model, path = _train_toy(tmp_path)
    env = dict(os.environ, MGXBENCH_FORM="auto", MGXBENCH_AUTO_MODEL=str(path), MGXBENCH_INNER_LOOPS="1",
               MGXBENCH_INPUT="wide" if er else "uniform", MGXBENCH_EXP_RANGE=str(er))
    r = subprocess.run([str(ROOT / "build" / exe), "auto", str(n), "MMM"], capture_output=True, text=True,
                       env=env, timeout=300)
    # exit 2 = the toy model's choice missed the accuracy target (its error predictions are not
    # the GPU's); the choice itself is what is compared here
    assert r.returncode in (0, 2), r.stdout + r.stderr
    m = re.search(r"mmb autotune: .* choice=(\w+) splits=(\d+) ksplit=(\d+)", r.stdout)
    assert m, r.stdout
    cands = at.candidates(n, n, n)
    if exe == "mm_2d":
        cands = [c for c in cands if c.ksplit == 1]
    c = at.choose(model, n, n, n, er, 1e-15, cands)
    assert m.group(1) == c.form
    assert int(m.group(2)) == c.splits and int(m.group(3)) == c.ksplit
    rec = dict(x.split("=", 1) for x in re.findall(r"BENCHMARK_RESULT\s+([^\r\n]+)", r.stdout)[0].split())
    assert rec["form"] == m.group(1)


def test_executable_auto_without_model_fails_loudly(tmp_path):
    env = dict(os.environ, MGXBENCH_FORM="auto", MGXBENCH_AUTO_MODEL=str(tmp_path / "absent.json"))
    r = subprocess.run([str(ROOT / "build" / "mm_1d"), "auto", "256", "MMM"], capture_output=True, text=True,
                       env=env, timeout=120)
    assert r.returncode != 0 and "AUTO:" in r.stderr


def test_packaged_model_loads_and_predicts():
    from mgxbench_b200 import autotune as at
    path = DATA / "mlp_b200.json"
    if not path.is_file():
        pytest.skip("no packaged model")
    mdl = at.MlpModel.load(path)
    pred = mdl.predict(16384, 16384, 16384, 20, at.candidates())
    assert len(pred) == len(at.candidates())
    assert all(t > 0 and e > 0 for t, e in pred)


def test_trained_network_beats_regression_on_measured_sweep():
    """Trains the MLP on the GPU (the library's forward/backward/Adam kernels) from the 2000
    measured training runs and compares its choices on the 500 exhaustively measured held-out
    shapes with the regression baseline's: regret at each accuracy target, misses of the
    target, and how closely each predicts the measured runtimes."""
    from mgxbench_b200 import autotune as at
    db_path = DATA / "sweep_b200.jsonl"
    if not db_path.is_file():
        pytest.skip("no measured sweep packaged")
    db = at.SweepDB(db_path)
    train = [r for r in db.rows if r.get("set") == "train"]
    held = [r for r in db.rows if r.get("set") == "heldout"]
    assert len(train) >= 2000 and len({(r["m"], r["n"], r["k"], r["exp_range"]) for r in held}) >= 500
    mlp = at.MlpModel().fit(train)
    reg = at.RegressionModel().fit(train)
    em, er = at.evaluate(mlp, held), at.evaluate(reg, held)
    print(json.dumps({"mlp": em, "regression": er}))
    assert em["misses_over_targets"] <= er["misses_over_targets"]
    assert em["regret"]["1e-15"]["mean_regret"] < er["regret"]["1e-15"]["mean_regret"]
    assert em["mean_regret_over_targets"] < er["mean_regret_over_targets"]
    assert em["accuracy"]["runtime_abs_ln_median"] < er["accuracy"]["runtime_abs_ln_median"]


def test_predictive_auto_validates_through_the_executable(tmp_path):
    """MGXBench-shaped AUTO with --auto-validate --auto-feedback: the packaged model's choice is run
    by build/mm_1d and the measurement is appended to a sweep database."""
    import shutil
    import types

    from mgxbench_b200 import predictive as pr
    if not (DATA / "mlp_b200.json").is_file():
        pytest.skip("no packaged model")
    db = tmp_path / "db.jsonl"
    shutil.copy(DATA / "sweep_b200.jsonl", db)
    n_before = len(db.read_text().splitlines())
    args = types.SimpleNamespace(decomposition="1d", ranks=2, size=2048, grid_rows=None, grid_cols=None,
                                 prediction_model="ml", auto_model=None, db=str(db), auto_validate=True,
                                 auto_feedback=True, build_dir="build", output=str(tmp_path / "out"), warmup=1,
                                 repeats=2, timeout=300, exp_range=10, target=1e-15, project_root=str(ROOT))
    assert pr.auto(args) == 0
    rep = json.loads((tmp_path / "out" / "autotuning_prediction.json").read_text())
    assert rep["status"] == "VALIDATED" and rep["measured"] is True
    assert rep["validation"]["measured_s"] > 0 and rep["validation"]["valid"] is True
    assert rep["feedback"]["status"] == "SAVED"
    assert len(db.read_text().splitlines()) == n_before + 1
