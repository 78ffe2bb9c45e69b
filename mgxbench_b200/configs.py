"""Measurements of the five workload configurations this library is specified on, one JSON line
each (python -m mgxbench_b200.configs [cfg1 cfg2 cfg3 cfg4 cfg5]).

  cfg1  FP64 N = 1024, uniform [-1, 1), one 1D block
  cfg2  FP64 N = 8192, uniform, 1D row-block with 4 row panels of 2048 x 8192 run in sequence
  cfg3  Ozaki N = 16384, u * 2^e (e in [-20, 20]), split count swept 3..9, native FP64 beside
  cfg4  2D SUMMA M = 12288, N = 20480, K = 16384, 3 x 5 grid, panel width 512, FP64 and Ozaki
        forms, each one persistent plan replayed from a CUDA graph
  cfg5  learned cost model: regret against the exhaustive sweep and prediction accuracy, beside
        the regression baseline (the packaged sweep database and model, or the files given)

Times are CUDA events on the launching stream after warm-up; errors are against the GPU
double-double product (all rows for cfg1, sampled rows otherwise).  Inputs are seeded synthetic
matrices with the shapes and distributions of the configurations.
"""
from __future__ import annotations

import json
import sys

import torch

import mgxbench_b200 as mgx


def _events():
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _time(fn, reps=3, warm=1):
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    e0, e1 = _events()
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    e1.synchronize()
    return e0.elapsed_time(e1) / reps * 1e-3


def _mat(r, c, kind, seed, e_range=0):
    x = torch.empty((r, c), dtype=torch.float64, device="cuda")
    mgx.fill_matrix(x, kind, e_range=e_range, seed=seed)
    return x


def cfg1():
    """The drop-in call (mgx_ab_multiply: 128 x 128 tiles, whole K), then every FP64 tile shape and
    K-slice count measured (64 output tiles of 128 x 128 leave most of the 148 SMs idle), and the
    one the learned cost model picks."""
    n = 1024
    A, B, C = _mat(n, n, 1, 11), _mat(n, n, 1, 12), torch.empty((n, n), dtype=torch.float64, device="cuda")
    peak = max(mgx.peak_fp64(k, 20000) for k in (3, 4))
    # 20 warm-up calls: each product is about 0.1 ms, and the clock must ramp up first
    t = _time(lambda: mgx.ab_multiply(A, B, C), reps=20, warm=20)
    e = mgx.error_vs_dd(A, B, C)
    out = [{"config": "cfg1", "form": "fp64", "n": n, "tile": "128x128", "ksplit": 1, "tflops": 2 * n ** 3 / t / 1e12,
            "seconds": t, "fp64_peak_tflops": peak, "frac_of_fp64_peak": 2 * n ** 3 / t / 1e12 / peak,
            "normwise_err": e["normwise"], "max_rel_err": e["max_rel"], "rows_checked": e["rows_checked"]}]
    from mgxbench_b200 import autotune as at
    from mgxbench_b200 import predictive as pr_mod
    fp64 = [c for c in at.candidates(n, n, n) if c.is_fp64]
    ws = mgx.OzakiWorkspace()
    measured = {}
    for c in fp64:
        measured[c] = _time(lambda: mgx.gemm_fp64(A, B, C, ksplit=c.ksplit, workspace=ws, tile_m=c.tile_m), reps=20,
                            warm=20)
    best = min(measured, key=measured.get)
    out.append({"config": "cfg1", "form": "fp64", "n": n, "measured": {c.name: 2 * n ** 3 / v / 1e12
                                                                      for c, v in measured.items()},
                "best": best.name, "best_tflops": 2 * n ** 3 / measured[best] / 1e12,
                "best_frac_of_fp64_peak": 2 * n ** 3 / measured[best] / 1e12 / peak})
    if pr_mod.DEFAULT_MODEL.is_file():
        model = at.MlpModel.load(pr_mod.DEFAULT_MODEL)
        c = at.choose(model, n, n, n, 0, 1.0, fp64)  # the form is fixed; the model picks tile and K slices
        t2 = _time(lambda: mgx.gemm_fp64(A, B, C, ksplit=c.ksplit, workspace=ws, tile_m=c.tile_m), reps=20,
                   warm=20)
        e2 = mgx.error_vs_dd(A, B, C)
        tf2 = 2 * n ** 3 / t2 / 1e12
        out.append({"config": "cfg1", "form": "fp64", "n": n, "tile": f"{c.tile_m}x128", "ksplit": c.ksplit,
                    "choice_from": "learned cost model", "tflops": tf2, "seconds": t2, "frac_of_fp64_peak": tf2 / peak,
                    # regret: the pick's time in the same sweep as the best (0 when it is the best)
                    "regret_vs_best_measured": measured[c] / measured[best] - 1, "normwise_err": e2["normwise"],
                    "max_rel_err": e2["max_rel"], "rows_checked": e2["rows_checked"]})
    return out


def cfg2():
    n, panels = 8192, 4
    mi = n // panels
    A, B, C = _mat(n, n, 1, 21), _mat(n, n, 1, 22), torch.empty((n, n), dtype=torch.float64, device="cuda")

    def run():
        for r in range(panels):
            mgx.gemm_fp64(A[r * mi:(r + 1) * mi], B, C[r * mi:(r + 1) * mi])
    t = _time(run, reps=3)
    peak = max(mgx.peak_fp64(k, 20000) for k in (3, 4))
    e = mgx.error_vs_dd(A, B, C, row_start=n // 2 - 128, row_count=256)
    tf = 2 * n ** 3 / t / 1e12
    return {"config": "cfg2", "form": "fp64", "n": n, "row_panels": panels, "tflops": tf, "seconds": t,
            "fp64_peak_tflops": peak, "frac_of_fp64_peak": tf / peak, "normwise_err": e["normwise"],
            "max_rel_err": e["max_rel"], "rows_checked": e["rows_checked"]}


def cfg3(splits=range(3, 10), moduli=(12, 13, 14, 15, 16)):
    n, er = 16384, 20
    A, B, C = _mat(n, n, 2, 31, er), _mat(n, n, 2, 32, er), torch.empty((n, n), dtype=torch.float64, device="cuda")
    rows = (n // 2 - 128, 256)
    out = []
    tn = _time(lambda: mgx.gemm_fp64(A, B, C), reps=2)
    en = mgx.error_vs_dd(A, B, C, *rows)
    out.append({"config": "cfg3", "form": "fp64", "n": n, "tflops": 2 * n ** 3 / tn / 1e12, "seconds": tn,
                "normwise_err": en["normwise"], "max_rel_err": en["max_rel"]})
    for s in splits:
        ws = torch.empty(mgx.ozaki_workspace_size(n, n, n, s), dtype=torch.uint8, device="cuda")
        t = _time(lambda: mgx.gemm_ozaki(A, B, C, splits=s, workspace=_Fixed(ws)), reps=2)
        e = mgx.error_vs_dd(A, B, C, *rows)
        out.append({"config": "cfg3", "form": "ozaki", "splits": s, "n": n, "effective_tflops": 2 * n ** 3 / t / 1e12,
                    "seconds": t, "int8_tops": 2 * n ** 3 * s * (s + 1) / 2 / t / 1e12,
                    "normwise_err": e["normwise"], "max_rel_err": e["max_rel"],
                    "max_componentwise_err": e["max_componentwise"], "meets_1e-15": e["normwise"] <= 1e-15,
                    "speedup_vs_fp64": tn / t})
        del ws
    for q in moduli:
        ws = torch.empty(mgx.crt_workspace_size(n, n, n, q), dtype=torch.uint8, device="cuda")
        t = _time(lambda: mgx.gemm_ozaki_crt(A, B, C, moduli=q, workspace=_Fixed(ws)), reps=2)
        e = mgx.error_vs_dd(A, B, C, *rows)
        out.append({"config": "cfg3", "form": "crt", "moduli": q, "n": n, "effective_tflops": 2 * n ** 3 / t / 1e12,
                    "seconds": t, "int8_tops": 2 * n ** 3 * q / t / 1e12,
                    "normwise_err": e["normwise"], "max_rel_err": e["max_rel"],
                    "max_componentwise_err": e["max_componentwise"], "meets_1e-15": e["normwise"] <= 1e-15,
                    "speedup_vs_fp64": tn / t})
        del ws
    return out


class _Fixed:
    def __init__(self, t):
        self.t = t

    def get(self, nbytes):
        return self.t


def cfg4(splits=None, model="default"):
    """The Ozaki plan's split count comes from the packaged learned cost model (the autotuner)
    when it is present, else from the a-priori error model."""
    M, N, K, pr, pc, bk = 12288, 20480, 16384, 3, 5, 512
    A, B = _mat(M, K, 1, 41), _mat(K, N, 1, 42)
    C = torch.empty((M, N), dtype=torch.float64, device="cuda")
    chooser = "ozaki_choose_splits"
    if splits is None:
        splits = mgx.ozaki_choose_splits(K, 0.0, 1e-15)
        from mgxbench_b200 import autotune as at
        from mgxbench_b200 import predictive as pr_mod
        if model == "default":
            model = at.MlpModel.load(pr_mod.DEFAULT_MODEL) if pr_mod.DEFAULT_MODEL.is_file() else None
        if model is not None:
            plan_cands = [c for c in at.candidates() if c.ksplit == 1]  # SUMMA panels are the K split
            oz = [c for c in plan_cands if c.form == "ozaki"]  # the plan runs the slice form
            splits = at.choose(model, M, N, K, 0, 1e-15, oz).splits
            chooser = "learned cost model"
    out = []
    for form, s in ((mgx.FORM_FP64, 0), (mgx.FORM_OZAKI, splits)):
        plan = mgx.SummaPlan(M, N, K, pr, pc, bk, form=form, splits=max(s, 2))
        stream = torch.cuda.Stream()
        plan.run(A, B, C, stream=stream)
        stream.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            plan.run(A, B, C, stream=stream)
        t = _time(g.replay, reps=3)
        e = mgx.error_vs_dd(A, B, C, row_start=M // 2 - 128, row_count=256)
        info = plan.info()
        rec = {"config": "cfg4", "form": "fp64" if form == mgx.FORM_FP64 else "ozaki", "splits": s or None,
               "m": M, "n": N, "k": K, "grid": f"{pr}x{pc}", "panel_k": bk,
               "tflops": 2 * M * N * K / t / 1e12, "seconds": t,
               "normwise_err": e["normwise"], "max_rel_err": e["max_rel"], "graph": True,
               "kernel_launches_per_product": mgx.launches_per_product(form, K, s), "splits_from": chooser if s else None}
        if form == mgx.FORM_FP64:
            # every block and panel in one persistent kernel
            rec.update(panels=info["panels"], work_tiles=info["work_tiles"], persistent_launches_per_product=1)
        else:
            # the slice form's sums are exact: the plan runs one product of all of C, without the panel list
            rec.update(panel_list="not used (exact accumulation: one product of all of C)",
                       k_chunks=info["panels"], product_work_items=info["work_tiles"])
        out.append(rec)
        del g
        plan.close()
    # the CRT form on the same grid: one whole-K product per block (exact integer sums, so the
    # panel order does not matter; build/mm_2d with MGXBENCH_FORM=crt MGXBENCH_BATCH=0), and all
    # blocks as one product (its default), bit-identical
    q = mgx.crt_choose_moduli(K, 1e-15)
    rcut = [M * i // pr for i in range(pr + 1)]
    ccut = [N * j // pc for j in range(pc + 1)]
    ws = mgx.OzakiWorkspace()

    def blocks():
        for i in range(pr):
            for j in range(pc):
                mgx.gemm_ozaki_crt(A[rcut[i]:rcut[i + 1]], B[:, ccut[j]:ccut[j + 1]],
                                   C[rcut[i]:rcut[i + 1], ccut[j]:ccut[j + 1]], moduli=q, workspace=ws)
    t = _time(blocks, reps=2)
    e = mgx.error_vs_dd(A, B, C, row_start=M // 2 - 128, row_count=256)
    per_block = C.clone()
    out.append({"config": "cfg4", "form": "crt", "moduli": q, "m": M, "n": N, "k": K, "grid": f"{pr}x{pc}",
                "blocks": pr * pc, "launches": "one product per block", "tflops": 2 * M * N * K / t / 1e12,
                "seconds": t, "normwise_err": e["normwise"], "max_rel_err": e["max_rel"], "graph": False,
                "moduli_from": "crt_choose_moduli"})
    # all blocks as one product: the SUMMA plan with the CRT form, replayed from a CUDA graph
    plan = mgx.SummaPlan(M, N, K, pr, pc, bk, form=mgx.FORM_CRT, splits=q)
    stream = torch.cuda.Stream()
    plan.run(A, B, C, stream=stream)
    stream.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        plan.run(A, B, C, stream=stream)
    t = _time(g.replay, reps=3)
    e = mgx.error_vs_dd(A, B, C, row_start=M // 2 - 128, row_count=256)
    out.append({"config": "cfg4", "form": "crt", "moduli": q, "m": M, "n": N, "k": K, "grid": f"{pr}x{pc}",
                "blocks": pr * pc, "launches": "all blocks in one product (SUMMA plan)",
                "kernel_launches_per_product": mgx.launches_per_product(mgx.FORM_CRT, K, q),
                "product_work_items": plan.info()["work_tiles"], "tflops": 2 * M * N * K / t / 1e12,
                "seconds": t, "normwise_err": e["normwise"], "max_rel_err": e["max_rel"], "graph": True,
                "bit_identical_to_per_block": bool(torch.equal(C.view(torch.int64), per_block.view(torch.int64))),
                "moduli_from": "crt_choose_moduli"})
    del g
    plan.close()
    return out


def cfg5(db_path=None, model_path=None):
    """Regret (at 1e-15 and looser targets) and prediction accuracy of the learned model and of
    the regression baseline on the exhaustively measured held-out shapes."""
    from mgxbench_b200 import autotune as at
    from mgxbench_b200 import predictive as pr_mod
    db = at.SweepDB(db_path or pr_mod.DEFAULT_DB)
    train = [r for r in db.rows if r.get("set") == "train"]
    held = [r for r in db.rows if r.get("set") == "heldout"]
    mlp = at.MlpModel.load(model_path or pr_mod.DEFAULT_MODEL)
    return {"config": "cfg5", "train_rows": len(train),
            "heldout_shapes": len({(r["m"], r["n"], r["k"], r["exp_range"]) for r in held}),
            "heldout_rows": len(held), "mlp": at.evaluate(mlp, held),
            "regression": at.evaluate(at.RegressionModel().fit(train), held)}


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    which = [a for a in argv if a.startswith("cfg")] or ["cfg1", "cfg2", "cfg3", "cfg4", "cfg5"]
    for w in which:
        if w == "cfg5":
            res = cfg5(*[a for a in argv if not a.startswith("cfg")][:2])
        else:
            res = globals()[w]()
        for r in (res if isinstance(res, list) else [res]):
            print(json.dumps(r), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
