"""Autotuner for the FP64-accurate GEMM forms: which form, tile shape and split count to run.

The reference chooses a communication library with a regression of measured wall times on
matrix size (autotuning/predictive.py: `estimate` 100-127, a log-log piecewise power law;
`_physical_fit` 140-165, an (x^2, x^3) least-squares fit).  Here the candidates are this
library's kernel configurations and the choice must also meet an accuracy target, so the model
predicts both runtime and error:

  * `RegressionModel` -- the method without the network, in the reference's spirit: per
    candidate, log runtime = a + b log(MNK) by least squares, and log10 error looked up by
    (form, split count, exponent-range bucket).
  * `MlpModel` -- a 3-layer FP32 MLP (6 -> 64 -> 64 -> 2) over (log2 M, log2 N, log2 K,
    exponent range, tile id, split count), trained and evaluated on the GPU by the library's own
    CUDA kernels (mgx_mlp_gradients / mgx_mlp_adam_step / mgx_mlp_forward).

Both feed the same rule: the fastest candidate whose predicted error meets the target.
`SweepDB` is an append-only JSONL of measurements; `measure()` produces them with CUDA events
and the double-double error check.  `regret()` judges a model's choices against an exhaustive
measured sweep.
"""
from __future__ import annotations

import hashlib
import json
import math
import time
from dataclasses import dataclass
from pathlib import Path

import numpy as np

TILE_FP64 = 0          # native FP64 kernel (DMMA), 128 x 128 output tiles over the whole K range
TILE_OZAKI_128 = 1     # Ozaki INT8 kernel, 128 x 128 output tiles over the whole K range
# native FP64 kernel, 128 x 128 output tiles, K cut into 2 / 4 / 8 / 16 slices (split-K)
TILE_FP64_K2, TILE_FP64_K4, TILE_FP64_K8, TILE_FP64_K16 = 2, 3, 4, 5
# Ozaki INT8 kernel, 128 x 128 output tiles, K cut into 4 / 16 slices (split-K)
TILE_OZAKI_K4, TILE_OZAKI_K16 = 6, 7
# CRT form (Ozaki scheme II), 256 x 256 output tiles over the whole K range; its "splits" is the
# modulus count
TILE_CRT = 8
# native FP64 kernel, 64 x 128 output tiles (twice the work items of the 128 x 128 tile), over the
# whole K range or cut into 2 / 4 / 8 slices
TILE_FP64_T64, TILE_FP64_T64_K2, TILE_FP64_T64_K4, TILE_FP64_T64_K8 = 9, 10, 11, 12
# native FP64 kernel, 64 x 128 output tiles, stream-K: every CTA an equal share of all tiles' K
# blocks (its "ksplit" is 0)
TILE_FP64_T64_SK = 13
FP64_KSPLIT = {TILE_FP64: 1, TILE_FP64_K2: 2, TILE_FP64_K4: 4, TILE_FP64_K8: 8, TILE_FP64_K16: 16,
               TILE_FP64_T64: 1, TILE_FP64_T64_K2: 2, TILE_FP64_T64_K4: 4, TILE_FP64_T64_K8: 8,
               TILE_FP64_T64_SK: 0}
FP64_TILE_M = {TILE_FP64_T64: 64, TILE_FP64_T64_K2: 64, TILE_FP64_T64_K4: 64, TILE_FP64_T64_K8: 64,
               TILE_FP64_T64_SK: 64}
OZAKI_KSPLIT = {TILE_OZAKI_128: 1, TILE_OZAKI_K4: 4, TILE_OZAKI_K16: 16}
SPLITS = tuple(range(3, 10))
CRT_MODULI = (9, 11, 12, 13, 14, 15, 16)
CRT_KMAX = 130816
# A CRT candidate must predict an error this many times below the target: its error falls only
# ~10x per added modulus and grows with sqrt(K), so predictions near a target need a guard band
# (the slice form's falls ~100x per slice).  The band covers the measured / predicted error
# ratio of the CRT runs in the training set (99th percentile 1.72, maximum 1.87 on the packaged
# sweep).  Same constant in host/autotune.h.
CRT_ERROR_MARGIN = 2.0
ERROR_FLOOR = 1e-17


@dataclass(frozen=True)
class Candidate:
    tile: int
    splits: int

    @property
    def is_fp64(self) -> bool:
        return self.tile in FP64_KSPLIT

    @property
    def is_crt(self) -> bool:
        return self.tile == TILE_CRT

    @property
    def form(self) -> str:
        return "fp64" if self.is_fp64 else ("crt" if self.is_crt else "ozaki")

    @property
    def ksplit(self) -> int:
        """K slices (1: whole K; 0: the FP64 stream-K schedule)."""
        if self.tile in FP64_KSPLIT:
            return FP64_KSPLIT[self.tile]
        return OZAKI_KSPLIT.get(self.tile, 1)

    @property
    def tile_m(self) -> int:
        """Output tile height of an FP64 candidate (64 or 128)."""
        return FP64_TILE_M.get(self.tile, 128)

    @property
    def name(self) -> str:
        base = ("fp64" if self.tile_m == 128 else "fp64t64") if self.is_fp64 else f"{self.form}{self.splits}"
        if self.ksplit == 0:
            return base + "sk"
        return base if self.ksplit == 1 else f"{base}k{self.ksplit}"


SPLITK_WORKSPACE_LIMIT = 4 << 30   # bytes of split-K partial products a candidate may need


def ozaki_kmax(s):
    """Longest K one int32 accumulation of s-digit slice products takes (mgx_ozaki_kmax)."""
    return (2147483647 // (4096 * s)) & ~127


def splitk_applies(m, n, k, ksplit, splits=0):
    """A split-K candidate is offered when every slice gets a 32-wide K block and the partial
    products fit SPLITK_WORKSPACE_LIMIT; an Ozaki one also needs K within one int32 accumulation
    (the executables apply the same rule)."""
    if ksplit <= 1:   # whole K, or stream-K (its workspace is a few tens of MB at most)
        return True
    if splits and k > ozaki_kmax(splits):
        return False
    return (k + 31) // 32 >= ksplit and ksplit * m * n * 8 <= SPLITK_WORKSPACE_LIMIT


def candidates(m=None, n=None, k=None):
    """Every configuration, or those that apply to an m x n x k product."""
    out = [Candidate(t, 0) for t in (TILE_FP64, TILE_FP64_K2, TILE_FP64_K4, TILE_FP64_K8, TILE_FP64_K16,
                                     TILE_FP64_T64, TILE_FP64_T64_K2, TILE_FP64_T64_K4, TILE_FP64_T64_K8,
                                     TILE_FP64_T64_SK)]
    out += [Candidate(t, s) for t in (TILE_OZAKI_128, TILE_OZAKI_K4, TILE_OZAKI_K16) for s in SPLITS]
    out += [Candidate(TILE_CRT, q) for q in CRT_MODULI]
    if m is not None:
        out = [c for c in out if (k <= CRT_KMAX if c.is_crt else splitk_applies(m, n, k, c.ksplit, c.splits))]
    return out


def features(m, n, k, exp_range, cand: Candidate):
    return [math.log2(m), math.log2(n), math.log2(k), float(exp_range), float(cand.tile), float(cand.splits)]


# ------------------------------------------------------------------ measurements
def measure(m, n, k, exp_range, cands, seed=0, check_rows=32, reps=None):
    """Runtime (CUDA events, after one warm-up) and normwise error of each candidate on one
    synthetic problem: A, B with u * 2^e entries, e uniform in [-exp_range, exp_range]."""
    import torch
    import mgxbench_b200 as mgx
    A = torch.empty((m, k), dtype=torch.float64, device="cuda")
    B = torch.empty((k, n), dtype=torch.float64, device="cuda")
    C = torch.empty((m, n), dtype=torch.float64, device="cuda")
    kind = 2 if exp_range > 0 else 1
    mgx.fill_matrix(A, kind, e_range=int(exp_range), seed=seed)
    mgx.fill_matrix(B, kind, e_range=int(exp_range), seed=seed + 1)
    ws = mgx.OzakiWorkspace()
    flop = 2.0 * m * n * k
    if reps is None:
        reps = 1 if flop > 2e12 else (3 if flop > 1e11 else 10)
    out = []
    errors = {}
    for c in cands:
        def run():
            if c.is_fp64:
                mgx.gemm_fp64(A, B, C, ksplit=c.ksplit, workspace=ws, tile_m=c.tile_m)
            elif c.is_crt:
                mgx.gemm_ozaki_crt(A, B, C, moduli=c.splits, workspace=ws)
            else:
                mgx.gemm_ozaki(A, B, C, splits=c.splits, workspace=ws, ksplit=c.ksplit)
        run()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            run()
        e1.record()
        e1.synchronize()
        t = e0.elapsed_time(e1) / reps * 1e-3
        key = (c.form, c.ksplit, c.splits)  # results depend on the form, K slices and split count only
        if key not in errors:
            rows = min(check_rows, m)
            errors[key] = mgx.error_vs_dd(A, B, C, row_start=(m - rows) // 2, row_count=rows)["normwise"]
        out.append({"m": m, "n": n, "k": k, "exp_range": exp_range, "tile": c.tile, "splits": c.splits,
                    "seconds": t, "tflops": flop / t / 1e12, "error": max(errors[key], ERROR_FLOOR)})
    del A, B, C, ws
    # hand back the cached device memory (torch's and the library's scratch pool) so that a sweep
    # over hundreds of shapes up to 32768 does not accumulate it
    torch.cuda.synchronize()
    mgx.scratch_trim()
    torch.cuda.empty_cache()
    return out


class SweepDB:
    """Append-only JSONL of measurements; resuming skips keys already present."""

    def __init__(self, path):
        self.path = Path(path)
        self.rows = []
        if self.path.exists():
            self.rows = [json.loads(l) for l in self.path.read_text().splitlines() if l.strip()]

    @staticmethod
    def key(r):
        return (r["m"], r["n"], r["k"], r["exp_range"], r["tile"], r["splits"])

    def has(self, m, n, k, r, c: Candidate):
        return (m, n, k, r, c.tile, c.splits) in {self.key(x) for x in self.rows}

    def add(self, rows):
        self.path.parent.mkdir(parents=True, exist_ok=True)
        with self.path.open("a") as f:
            for r in rows:
                f.write(json.dumps(r) + "\n")
        self.rows.extend(rows)

    def digest(self) -> str:
        return hashlib.sha256("\n".join(json.dumps(r, sort_keys=True) for r in self.rows).encode()).hexdigest()[:16]


def random_shapes(count, seed, lo=256, hi=32768, rmax=40):
    rng = np.random.default_rng(seed)
    lg = rng.uniform(math.log2(lo), math.log2(hi), (count, 3))
    dims = np.round(np.exp2(lg)).astype(int)
    ranges = rng.integers(0, rmax + 1, count)
    return [(int(a), int(b), int(c), int(r)) for (a, b, c), r in zip(dims, ranges)]


def shape_fits(m, n, k, limit_bytes=100 * 2 ** 30):
    """Keeps a measurement within a bounded share of device memory (A, B, C and the largest
    workspace: the 9-slice Ozaki one plus at most SPLITK_WORKSPACE_LIMIT of split-K partial
    products, or the 16-modulus CRT one, residues of A, B and C rounded up to 256-row tiles)."""
    r = lambda x: (x + 255) // 256 * 256
    crt = 16 * (r(m) * k + r(n) * k + r(m) * r(n))
    return 8 * (m * k + k * n + m * n) + max(9 * (m + n) * k + SPLITK_WORKSPACE_LIMIT, crt) < limit_bytes


# ------------------------------------------------------------------ models
def _targets(rows):
    t = np.array([math.log(r["seconds"]) for r in rows])
    e = np.array([math.log10(max(r["error"], ERROR_FLOOR)) for r in rows])
    return t, e


class RegressionModel:
    """Per-candidate log-log runtime fit and a (form, splits, range bucket) error table."""

    def fit(self, rows):
        self.rt = {}
        by = {}
        for r in rows:
            by.setdefault((r["tile"], r["splits"]), []).append(r)
        for key, rs in by.items():
            x = np.array([math.log(r["m"] * r["n"] * r["k"]) for r in rs])
            y = np.array([math.log(r["seconds"]) for r in rs])
            if len(rs) >= 2 and np.ptp(x) > 0:
                b, a = np.polyfit(x, y, 1)
            else:
                a, b = float(np.mean(y) - np.mean(x)), 1.0
            self.rt[key] = (a, b)
        self.err = {}
        for r in rows:
            form = Candidate(r["tile"], r["splits"]).form
            self.err.setdefault((form, r["splits"], self._bucket(r["exp_range"])), []).append(
                math.log10(max(r["error"], ERROR_FLOOR)))
        self.err = {k: float(np.mean(v)) for k, v in self.err.items()}
        return self

    @staticmethod
    def _bucket(r):
        return min(int(r) // 5, 8)

    def predict(self, m, n, k, exp_range, cands):
        out = []
        for c in cands:
            a, b = self.rt.get((c.tile, c.splits), (0.0, 1.0))
            t = math.exp(a + b * math.log(m * n * k))
            e = self.err.get((c.form, c.splits, self._bucket(exp_range)))
            if e is None:
                near = [v for (f, s, bk), v in self.err.items() if f == c.form and s == c.splits]
                e = float(np.mean(near)) if near else 0.0
            out.append((t, 10.0 ** e))
        return out


class MlpModel:
    """The learned cost model, trained on the GPU with the library's MLP kernels."""

    def __init__(self):
        self.params = None
        self.xmean = self.xstd = self.ymean = self.ystd = None
        self.loss_history = []

    def fit(self, rows, epochs=1000, batch=256, lr=3e-3, seed=0):
        import torch
        import mgxbench_b200 as mgx
        X = np.array([features(r["m"], r["n"], r["k"], r["exp_range"], Candidate(r["tile"], r["splits"]))
                      for r in rows], np.float64)
        t, e = _targets(rows)
        Y = np.stack([t, e], axis=1)
        self.xmean, self.xstd = X.mean(0), X.std(0) + 1e-9
        self.ymean, self.ystd = Y.mean(0), Y.std(0) + 1e-9
        dX = torch.from_numpy(((X - self.xmean) / self.xstd).astype(np.float32)).cuda()
        dY = torch.from_numpy(((Y - self.ymean) / self.ystd).astype(np.float32)).cuda()
        w = torch.tensor([1.0, 1.0], dtype=torch.float32, device="cuda")
        P = torch.empty(mgx.mlp_param_count(), dtype=torch.float32, device="cuda")
        mgx.mlp_init(P, seed=seed + 12345)
        G, M, V = torch.empty_like(P), torch.zeros_like(P), torch.zeros_like(P)
        L = torch.empty(1, dtype=torch.float32, device="cuda")
        gen = torch.Generator(device="cuda")
        gen.manual_seed(seed)
        n = dX.shape[0]
        step = 0
        for ep in range(epochs):
            perm = torch.randperm(n, device="cuda", generator=gen)
            rate = lr * (0.5 * (1 + math.cos(math.pi * ep / epochs)) * 0.95 + 0.05)
            for b0 in range(0, n, batch):
                i = perm[b0:b0 + batch]
                mgx.mlp_gradients(dX[i].contiguous(), dY[i].contiguous(), w, P, G, L)
                step += 1
                mgx.mlp_adam_step(P, G, M, V, step, rate)
            if ep % 20 == 0 or ep == epochs - 1:
                mgx.mlp_gradients(dX, dY, w, P, G, L)
                self.loss_history.append((ep, L.item()))
        self.params = P
        return self

    def predict(self, m, n, k, exp_range, cands):
        import torch
        import mgxbench_b200 as mgx
        X = np.array([features(m, n, k, exp_range, c) for c in cands], np.float64)
        dX = torch.from_numpy(((X - self.xmean) / self.xstd).astype(np.float32)).cuda()
        out = mgx.mlp_forward(dX, self.params).cpu().numpy().astype(np.float64) * self.ystd + self.ymean
        return [(math.exp(a), 10.0 ** b) for a, b in out]

    def save(self, path, digest=""):
        meta = {"format": "mgx-mlp-v1", "layers": [6, 64, 64, 2], "activation": "tanh", "training_set": digest,
                "candidates": [[c.tile, c.splits] for c in candidates()],
                "xmean": self.xmean.tolist(), "xstd": self.xstd.tolist(), "ymean": self.ymean.tolist(),
                "ystd": self.ystd.tolist(), "params": self.params.cpu().numpy().tolist(),
                "loss_history": self.loss_history}
        Path(path).write_text(json.dumps(meta))

    @classmethod
    def load(cls, path):
        import torch
        d = json.loads(Path(path).read_text())
        mdl = cls()
        mdl.xmean, mdl.xstd = np.array(d["xmean"]), np.array(d["xstd"])
        mdl.ymean, mdl.ystd = np.array(d["ymean"]), np.array(d["ystd"])
        mdl.params = torch.tensor(d["params"], dtype=torch.float32, device="cuda")
        mdl.loss_history = d.get("loss_history", [])
        return mdl


def choose(model, m, n, k, exp_range, target, cands=None, margin=1.0, crt_margin=CRT_ERROR_MARGIN):
    """Fastest candidate whose predicted error is <= target / margin (target / (margin
    crt_margin) for the CRT form); the largest split count if none."""
    cands = cands or candidates(m, n, k)
    pred = model.predict(m, n, k, exp_range, cands)
    ok = [(t, c) for (t, e), c in zip(pred, cands) if e * margin * (crt_margin if c.is_crt else 1.0) <= target]
    if ok:
        return min(ok, key=lambda x: x[0])[1]
    return max(cands, key=lambda c: (c.splits, -c.tile))


def regret(model, sweep_rows, target, margin=1.0, crt_margin=CRT_ERROR_MARGIN):
    """Mean and max of t(chosen) / t(best feasible) - 1 over the shapes of an exhaustive sweep,
    and how many choices missed the accuracy target."""
    shapes = {}
    for r in sweep_rows:
        shapes.setdefault((r["m"], r["n"], r["k"], r["exp_range"]), []).append(r)
    regs, misses = [], 0
    for (m, n, k, er), rs in shapes.items():
        cands = [Candidate(r["tile"], r["splits"]) for r in rs]
        feasible = [r for r in rs if r["error"] <= target]
        if not feasible:
            continue
        best = min(r["seconds"] for r in feasible)
        c = choose(model, m, n, k, er, target, cands, margin, crt_margin)
        r = next(x for x in rs if x["tile"] == c.tile and x["splits"] == c.splits)
        if r["error"] > target:
            misses += 1
            regs.append(float("nan"))
        else:
            regs.append(r["seconds"] / best - 1.0)
    valid = [x for x in regs if x == x]
    return {"shapes": len(regs), "mean_regret": float(np.mean(valid)) if valid else float("nan"),
            "max_regret": float(np.max(valid)) if valid else float("nan"), "misses": misses,
            "miss_rate": misses / max(1, len(regs))}


def accuracy(model, sweep_rows):
    """How well a model predicts what was measured: median and 90th percentile of |ln(t_pred /
    t_meas)| and of |log10(err_pred / err_meas)| over every (shape, candidate) of a sweep."""
    shapes = {}
    for r in sweep_rows:
        shapes.setdefault((r["m"], r["n"], r["k"], r["exp_range"]), []).append(r)
    lt, le = [], []
    for (m, n, k, er), rs in shapes.items():
        pred = model.predict(m, n, k, er, [Candidate(r["tile"], r["splits"]) for r in rs])
        for (t, e), r in zip(pred, rs):
            lt.append(abs(math.log(t / r["seconds"])))
            le.append(abs(math.log10(max(e, ERROR_FLOOR) / max(r["error"], ERROR_FLOOR))))
    return {"runtime_abs_ln_median": float(np.median(lt)), "runtime_abs_ln_p90": float(np.quantile(lt, 0.9)),
            "error_abs_log10_median": float(np.median(le)), "error_abs_log10_p90": float(np.quantile(le, 0.9))}


TARGETS = (1e-15, 1e-13, 1e-11, 1e-9, 1e-7)


def evaluate(model, sweep_rows, targets=TARGETS):
    """Regret at each accuracy target (1e-15 first) and prediction accuracy on a sweep."""
    out = {"regret": {f"{t:.0e}": regret(model, sweep_rows, t) for t in targets},
           "accuracy": accuracy(model, sweep_rows)}
    out["mean_regret_over_targets"] = float(np.mean([v["mean_regret"] for v in out["regret"].values()]))
    out["misses_over_targets"] = int(sum(v["misses"] for v in out["regret"].values()))
    return out


def run_sweep(db_path, train_shapes=2000, heldout_shapes=500, seed=0, budget_s=None, log=print):
    """Measures the training set (one random candidate per shape) and the exhaustive held-out
    sweep (every candidate per shape), appending to the JSONL database as it goes."""
    db = SweepDB(db_path)
    rng = np.random.default_rng(seed)
    t0 = time.time()
    train = [s for s in random_shapes(train_shapes * 2, seed + 1) if shape_fits(*s[:3])][:train_shapes]
    held = [s for s in random_shapes(heldout_shapes * 2, seed + 2) if shape_fits(*s[:3])][:heldout_shapes]
    for i, (m, n, k, er) in enumerate(train):
        cs = candidates(m, n, k)
        c = cs[int(rng.integers(len(cs)))]
        if not db.has(m, n, k, er, c):
            rows = measure(m, n, k, er, [c], seed=i)
            for r in rows:
                r["set"] = "train"
            db.add(rows)
        if budget_s and time.time() - t0 > budget_s:
            log(f"budget reached after {i + 1} training shapes")
            return db
    for i, (m, n, k, er) in enumerate(held):
        todo = [c for c in candidates(m, n, k) if not db.has(m, n, k, er, c)]
        if todo:
            rows = measure(m, n, k, er, todo, seed=100000 + i)
            for r in rows:
                r["set"] = "heldout"
            db.add(rows)
        if budget_s and time.time() - t0 > budget_s:
            log(f"budget reached after {i + 1} held-out shapes")
            return db
    return db


def refresh_rows(db_path, tiles, seed=0, train_shapes=2000, heldout_shapes=500, budget_s=None, log=print):
    """Measures again the database rows of the given tile ids (after a change to those kernels),
    with the inputs the sweep used for each shape, and rewrites the database.  Resumable: a row
    already refreshed carries "refreshed": the tag, and a run that reaches the budget writes what
    it has."""
    db = SweepDB(db_path)
    tiles = set(tiles)
    tag = "tiles " + ",".join(str(t) for t in sorted(tiles))
    train = [s for s in random_shapes(train_shapes * 2, seed + 1) if shape_fits(*s[:3])][:train_shapes]
    held = [s for s in random_shapes(heldout_shapes * 2, seed + 2) if shape_fits(*s[:3])][:heldout_shapes]
    seeds = {("train", s): i for i, s in enumerate(train)}
    seeds.update({("heldout", s): 100000 + i for i, s in enumerate(held)})
    groups = {}
    for idx, r in enumerate(db.rows):
        if r["tile"] in tiles and r.get("refreshed") != tag:
            groups.setdefault((r.get("set"), (r["m"], r["n"], r["k"], r["exp_range"])), []).append(idx)
    t0 = time.time()
    done = 0
    for (which, shape), idxs in groups.items():
        if (which, shape) not in seeds:
            continue
        cands = [Candidate(db.rows[i]["tile"], db.rows[i]["splits"]) for i in idxs]
        for i, new in zip(idxs, measure(*shape, cands, seed=seeds[(which, shape)])):
            new["set"] = which
            new["refreshed"] = tag
            db.rows[i] = new
        done += 1
        if budget_s and time.time() - t0 > budget_s:
            log(f"budget reached after {done} of {len(groups)} shapes")
            break
    tmp = db.path.with_suffix(".tmp")
    tmp.write_text("".join(json.dumps(r) + "\n" for r in db.rows))
    tmp.replace(db.path)
    return db, done, len(groups)


def main(argv=None):
    """python -m mgxbench_b200.autotune {sweep,refresh,train,evaluate,choose} ...

    sweep     measure the training set and the exhaustive held-out sweep into a JSONL database
    refresh   measure again the database rows of some tile ids (after a change to their kernels)
    train     fit the MLP on the GPU from the database's training rows and save its weights
    evaluate  regret of the MLP and of the regression baseline against the held-out sweep
    choose    the configuration the saved MLP picks for one problem
    """
    import argparse
    ap = argparse.ArgumentParser(prog="mgxbench_b200.autotune", description=main.__doc__)
    sub = ap.add_subparsers(dest="cmd", required=True)
    sw = sub.add_parser("sweep")
    sw.add_argument("--db", required=True)
    sw.add_argument("--train", type=int, default=2000)
    sw.add_argument("--heldout", type=int, default=500)
    sw.add_argument("--seed", type=int, default=0)
    sw.add_argument("--budget", type=float, default=None, help="stop after this many seconds (resumable)")
    rf = sub.add_parser("refresh")
    rf.add_argument("--db", required=True)
    rf.add_argument("--tiles", required=True, help="comma-separated tile ids, e.g. 0,1,2,3,4,9,10,11,12,13")
    rf.add_argument("--seed", type=int, default=0)
    rf.add_argument("--budget", type=float, default=None, help="stop after this many seconds (resumable)")
    tr = sub.add_parser("train")
    tr.add_argument("--db", required=True)
    tr.add_argument("--out", required=True)
    tr.add_argument("--epochs", type=int, default=1000)
    ev = sub.add_parser("evaluate")
    ev.add_argument("--db", required=True)
    ev.add_argument("--model", required=True)
    ch = sub.add_parser("choose")
    ch.add_argument("--model", required=True)
    ch.add_argument("m", type=int)
    ch.add_argument("n", type=int)
    ch.add_argument("k", type=int)
    ch.add_argument("--exp-range", type=float, default=20)
    ch.add_argument("--target", type=float, default=1e-15)
    a = ap.parse_args(argv)
    if a.cmd == "sweep":
        db = run_sweep(a.db, a.train, a.heldout, a.seed, a.budget)
        print(json.dumps({"rows": len(db.rows), "digest": db.digest()}))
    elif a.cmd == "refresh":
        db, done, total = refresh_rows(a.db, [int(t) for t in a.tiles.split(",")], a.seed, budget_s=a.budget)
        print(json.dumps({"rows": len(db.rows), "shapes_refreshed": done, "shapes": total, "digest": db.digest()}))
    elif a.cmd == "train":
        db = SweepDB(a.db)
        rows = [r for r in db.rows if r.get("set") == "train"]
        mdl = MlpModel().fit(rows, epochs=a.epochs)
        mdl.save(a.out, db.digest())
        print(json.dumps({"trained_on": len(rows), "loss": mdl.loss_history[-1]}))
    elif a.cmd == "evaluate":
        db = SweepDB(a.db)
        train = [r for r in db.rows if r.get("set") == "train"]
        held = [r for r in db.rows if r.get("set") == "heldout"]
        out = {"mlp": evaluate(MlpModel.load(a.model), held),
               "regression": evaluate(RegressionModel().fit(train), held)}
        print(json.dumps(out, indent=1))
    elif a.cmd == "choose":
        c = choose(MlpModel.load(a.model), a.m, a.n, a.k, a.exp_range, a.target)
        print(json.dumps({"form": c.form, "tile": c.tile, "ksplit": c.ksplit, "splits": c.splits}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
