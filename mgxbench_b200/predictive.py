"""AUTO front end of the learned cost model, shaped like MGXBench's autotuning/predictive.py.

MGXBench's `benchmark.py --libraries AUTO` calls `autotuning.predictive.auto(args)`
(benchmark.py:83-85), which ranks the calibrated communication configurations by predicted
time, writes `autotuning_prediction.json` and prints an AUTOTUNING REPORT
(autotuning/predictive.py:606-657).  In this library the communication codes are labels only;
what AUTO picks is the kernel configuration (native FP64, or Ozaki with s splits) for the
problem, subject to an accuracy target.  `auto(args)` accepts the same argument namespace
(decomposition, ranks, size, grid_rows, grid_cols, prediction_model, auto_model,
auto_validate, auto_feedback, build_dir, output, ...) and writes a report with the same keys
(autotuning/predictive.py:627-631) plus the predicted error of every candidate.

    python -m mgxbench_b200.predictive auto --decomposition 1d --ranks 4 --size 8192
    python -m mgxbench_b200.predictive calibrate --db sweep.jsonl --out mlp.json

`--prediction-model ml` uses the MLP (inference on the GPU through mgx_mlp_forward);
`extrapolation` uses the regression baseline fitted on the sweep database's training rows
(the method without the network); `auto` takes the MLP when its file exists.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import subprocess
import sys
from pathlib import Path

from mgxbench_b200 import autotune as at

PACKAGE = Path(__file__).resolve().parent
ROOT = PACKAGE.parent
DEFAULT_MODEL = PACKAGE / "data" / "mlp_b200.json"
DEFAULT_DB = PACKAGE / "data" / "sweep_b200.jsonl"
TRAIN_LO, TRAIN_HI = 256, 32768      # the sweep's log-uniform dimension range


def grid_shape(p, rows=None, cols=None):
    """The 2D process grid: explicit rows/cols, else the most square factorisation with
    rows <= cols (2D-block-matrix/mmb.cu:45-58, MPI_Dims_create)."""
    if rows and cols:
        return rows, cols
    r = int(math.isqrt(p))
    while p % r:
        r -= 1
    return r, p // r


def resolve_model(method, supplied=None, db=None):
    """(model object, algorithm name, file) for `method` in {ml, extrapolation, auto}."""
    path = Path(supplied) if supplied else DEFAULT_MODEL
    if method == "auto":
        method = "ml" if path.is_file() else "extrapolation"
    if method == "ml":
        if not path.is_file():
            raise ValueError(f"cost model {path} missing; run: python -m mgxbench_b200.predictive calibrate --help")
        return at.MlpModel.load(path), "mlp", str(path)
    dbp = Path(db) if db else DEFAULT_DB
    rows = [r for r in at.SweepDB(dbp).rows if r.get("set") == "train"]
    if not rows:
        raise ValueError(f"no training rows in {dbp}; run: python -m mgxbench_b200.predictive calibrate --help")
    return at.RegressionModel().fit(rows), "loglog-regression", str(dbp)


def rank_candidates(model, algorithm, m, n, k, exp_range, target, grid=(1, 1), bk=None, library="MMM"):
    """Every candidate with its predicted time and error; feasible ones (error <= target) first,
    fastest first -- the same rule as autotune.choose."""
    cands = at.candidates(m, n, k)
    if grid != (1, 1) or bk:
        # the 2D SUMMA plan runs whole-K tiles (its panels are the K split)
        cands = [c for c in cands if c.ksplit == 1]
    pred = model.predict(m, n, k, exp_range, cands)
    extrapolated = not all(TRAIN_LO <= d <= TRAIN_HI for d in (m, n, k))
    out = []
    for (t, e), c in zip(pred, cands):
        out.append({"library": library, "form": c.form, "tile": c.tile, "tile_m": c.tile_m,
                    "ksplit": c.ksplit, "splits": c.splits, "grid_rows": grid[0], "grid_cols": grid[1], "summa_bk": bk,
                    "predicted_s": float(t), "predicted_error": float(e), "meets_target": bool(e <= target),
                    "algorithm": algorithm, "extrapolated": extrapolated})
    feasible = sorted((r for r in out if r["meets_target"]), key=lambda r: r["predicted_s"])
    rest = sorted((r for r in out if not r["meets_target"]), key=lambda r: (-r["splits"], r["tile"]))
    return feasible + rest


def _measure(args, best, root):
    """Runs the chosen configuration through the drop-in executable once and parses its
    BENCHMARK_RESULT record."""
    exe = Path(root) / args.build_dir / ("mm_2d" if args.decomposition == "2d" else "mm_1d")
    if not exe.is_file():
        raise ValueError(f"executable not found: {exe}")
    env = dict(os.environ, MGXBENCH_EMULATED_RANKS=str(args.ranks), MGXBENCH_FORM=best["form"],
               MGXBENCH_SPLITS=str(max(best["splits"], 2)), MGXBENCH_MODULI=str(max(best["splits"], 8)),
               MGXBENCH_KSPLIT=str(best["ksplit"]), MGXBENCH_TILE_M=str(best.get("tile_m", 128)),
               MGXBENCH_INNER_LOOPS=str(args.repeats),
               MGXBENCH_INTERNAL_WARMUP=str(args.warmup))
    er = getattr(args, "exp_range", 0) or 0
    env["MGXBENCH_INPUT"] = "wide" if er > 0 else "uniform"
    env["MGXBENCH_EXP_RANGE"] = str(int(er))
    if args.decomposition == "2d":
        env["MGXBENCH_GRID_ROWS"], env["MGXBENCH_GRID_COLS"] = str(best["grid_rows"]), str(best["grid_cols"])
        if best["summa_bk"]:
            env["MGXBENCH_SUMMA_BK"] = str(best["summa_bk"])
    cp = subprocess.run([str(exe), "auto", str(args.size), best["library"]], env=env, capture_output=True,
                        text=True, timeout=args.timeout)
    line = next((l for l in cp.stdout.splitlines() if l.startswith("BENCHMARK_RESULT")), None)
    if cp.returncode != 0 or line is None:
        raise ValueError(f"validation run failed (rc={cp.returncode}): {cp.stderr.strip()[-300:]}")
    kv = dict(re.findall(r"(\w+)=(\S+)", line))
    return {"measured_s": float(kv["seconds"]), "valid": kv.get("valid") == "1",
            "norm_rel_err": float(kv["norm_rel_err"]) if "norm_rel_err" in kv else None}


def auto(args):
    """Predicts the fastest configuration that meets the accuracy target (same role and report
    keys as autotuning/predictive.py:606-657)."""
    root = Path(getattr(args, "project_root", None) or ROOT)
    target = getattr(args, "target", None) or 1e-15
    exp_range = getattr(args, "exp_range", 0) or 0
    try:
        model, algorithm, model_file = resolve_model(getattr(args, "prediction_model", "auto"),
                                                     getattr(args, "auto_model", None), getattr(args, "db", None))
    except (ValueError, ImportError, RuntimeError) as exc:
        print(f"AUTO: {exc}", file=sys.stderr)
        return 2
    grid, bk = (1, 1), None
    if args.decomposition == "2d":
        grid = grid_shape(args.ranks, getattr(args, "grid_rows", None), getattr(args, "grid_cols", None))
        bk = getattr(args, "summa_bk", None) or int(os.environ.get("MGXBENCH_SUMMA_BK", "256"))
    ranking = rank_candidates(model, algorithm, args.size, args.size, args.size, exp_range, target, grid, bk)
    best = ranking[0]
    fp64 = next(r for r in ranking if r["form"] == "fp64")
    speedup = fp64["predicted_s"] / best["predicted_s"]
    report = {"size": args.size, "ranks": args.ranks, "decomposition": args.decomposition,
              "architecture_id": _architecture_id(), "best": best, "ranking": ranking,
              "speedup_vs_MPI_predicted": None, "speedup_vs_fp64_predicted": speedup,
              "target_error": target, "exp_range": exp_range, "prediction_model": algorithm,
              "calibration_file": model_file, "status": "PREDICTED", "measured": False}
    status = 0
    if getattr(args, "auto_validate", False):
        try:
            meas = _measure(args, best, root)
            report["validation"] = dict(meas, status="VALIDATED" if meas["valid"] else "INVALID",
                                        predicted_s=best["predicted_s"],
                                        absolute_error_s=abs(meas["measured_s"] - best["predicted_s"]))
            report["measured"] = True
            status = 0 if meas["valid"] else 1
            if getattr(args, "auto_feedback", False) and meas["valid"]:
                db = at.SweepDB(getattr(args, "db", None) or DEFAULT_DB)
                db.add([{"m": args.size, "n": args.size, "k": args.size, "exp_range": exp_range,
                         "tile": best["tile"], "splits": best["splits"], "seconds": meas["measured_s"],
                         "tflops": 2.0 * args.size ** 3 / meas["measured_s"] / 1e12,
                         "error": max(meas["norm_rel_err"] or at.ERROR_FLOOR, at.ERROR_FLOOR), "set": "train",
                         "source": "auto-feedback"}])
                report["feedback"] = {"status": "SAVED", "database": str(db.path)}
        except (ValueError, subprocess.TimeoutExpired, OSError) as exc:
            report["validation"] = {"status": "FAILED", "reason": str(exc)}
            status = 1
        report["status"] = "VALIDATED" if status == 0 else "VALIDATION_FAILED"
    out = Path(getattr(args, "output", "results/auto_prediction")) / "autotuning_prediction.json"
    if not out.is_absolute():
        out = root / out
    out.parent.mkdir(parents=True, exist_ok=True)
    out.write_text(json.dumps(report, indent=2) + "\n")
    print("\n" + "=" * 48 + "\n         MGXBench - AUTOTUNING REPORT\n" + "=" * 48)
    print(f"Prediction Model  : {algorithm}\nConfiguration:\n  Matrix Size       : {args.size}"
          f"\n  GPUs              : {args.ranks} (emulated on one GPU)\n  Decomposition     : {args.decomposition.upper()}")
    if args.decomposition == "2d":
        print(f"  Grid              : {grid[0]} x {grid[1]}")
    print(f"\nBest Predicted Configuration:\n  Form              : {best['form']}"
          f"\n  Splits            : {best['splits'] if best['form'] != 'fp64' else 'N/A'}"
          f"{' (moduli)' if best['form'] == 'crt' else ''}"
          f"\n  K slices          : {best['ksplit']}"
          f"\n  Tile              : {best.get('tile_m', 128) if best['form'] == 'fp64' else (256 if best['form'] == 'crt' else 128)} x {256 if best['form'] == 'crt' else 128}"
          f"\n  SUMMA BK          : {bk if args.decomposition == '2d' else 'N/A'}"
          f"\n  Predicted Time    : {best['predicted_s']:.6f} s"
          f"\n  Predicted Error   : {best['predicted_error']:.3e} (target {target:.1e})"
          f"\n  Speedup vs FP64   : {speedup:.2f}x"
          f"\n  Extrapolation     : {'YES' if best['extrapolated'] else 'NO'}"
          f"\n\nStatus: {report['status']}{'' if report['measured'] else ' (not measured)'}\nReport: {out}\n"
          + "=" * 48)
    if getattr(args, "auto_validate", False):
        print("Validation status:", report.get("validation", {}).get("status", "UNKNOWN"))
        if report.get("feedback"):
            print("Feedback status:", report["feedback"]["status"])
    return status


def _architecture_id():
    try:
        import torch
        if torch.cuda.is_available():
            return torch.cuda.get_device_name(0)
    except ImportError:
        pass
    return "unknown"


def calibrate(args):
    """Measured sweep into the database, then the MLP trained on the GPU from its training rows."""
    db = at.run_sweep(args.db, args.train, args.heldout, args.seed, args.budget)
    rows = [r for r in db.rows if r.get("set") == "train"]
    mdl = at.MlpModel().fit(rows, epochs=args.epochs)
    mdl.save(args.out, db.digest())
    print(json.dumps({"rows": len(db.rows), "trained_on": len(rows), "model": str(args.out),
                      "loss": mdl.loss_history[-1]}))
    return 0


def main(argv=None):
    p = argparse.ArgumentParser(prog="mgxbench_b200.predictive",
                                description="AUTO selection of the FP64-accurate GEMM configuration")
    sub = p.add_subparsers(dest="command", required=True)
    c = sub.add_parser("calibrate", help="measure the sweep and train the cost model")
    c.add_argument("--db", default=str(DEFAULT_DB))
    c.add_argument("--out", default=str(DEFAULT_MODEL))
    c.add_argument("--train", type=int, default=2000)
    c.add_argument("--heldout", type=int, default=500)
    c.add_argument("--seed", type=int, default=0)
    c.add_argument("--budget", type=float, default=None)
    c.add_argument("--epochs", type=int, default=1000)
    a = sub.add_parser("auto", help="predict the fastest configuration meeting the error target")
    a.add_argument("--decomposition", choices=("1d", "2d"), required=True)
    a.add_argument("--ranks", type=int, required=True)
    a.add_argument("--size", type=int, required=True)
    a.add_argument("--grid-rows", type=int, default=None)
    a.add_argument("--grid-cols", type=int, default=None)
    a.add_argument("--summa-bk", type=int, default=256)
    a.add_argument("--prediction-model", choices=("extrapolation", "ml", "auto"), default="auto")
    a.add_argument("--build-dir", default="build")
    a.add_argument("--auto-model", default=None)
    a.add_argument("--db", default=None)
    a.add_argument("--auto-validate", action="store_true")
    a.add_argument("--auto-feedback", action="store_true")
    a.add_argument("--warmup", type=int, default=2)
    a.add_argument("--repeats", type=int, default=5)
    a.add_argument("--timeout", type=int, default=600)
    a.add_argument("--output", default="results/auto_prediction")
    a.add_argument("--exp-range", type=float, default=0.0, help="input exponent range (0: MGXBench's inputs)")
    a.add_argument("--target", type=float, default=1e-15, help="normwise error target")
    args = p.parse_args(argv)
    if args.command == "auto":
        if args.ranks <= 0 or args.size <= 0:
            p.error("--ranks and --size must be positive")
        if (args.grid_rows is None) != (args.grid_cols is None):
            p.error("--grid-rows and --grid-cols must be supplied together")
        if args.grid_rows is not None and args.grid_rows * args.grid_cols != args.ranks:
            p.error("--grid-rows * --grid-cols must equal --ranks")
        if args.auto_feedback and not args.auto_validate:
            p.error("--auto-feedback requires --auto-validate")
        return auto(args)
    return calibrate(args)


if __name__ == "__main__":
    raise SystemExit(main())
