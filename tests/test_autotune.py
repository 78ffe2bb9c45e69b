"""Autotuner host logic without a GPU: candidate space, the regression baseline (the method in the
reference's autotuning/predictive.py spirit), the choice rule and the regret measure."""
import math

import numpy as np

from mgxbench_b200 import autotune as at


def synthetic_rows(shapes, seed=0):
    """A toy machine: FP64 at 30 TF/s with error 1e-15 * sqrt(K/1e3); Ozaki s at 4.5 POPS / (s(s+1)/2)
    plus a 1 GB/s-per-byte split cost, error 10^(-8 - 2(s-4)) for wide ranges; CRT with q moduli
    at 4.5 POPS / q plus its residue traffic, error 2 sqrt(K/6) 2^(-(L-3)/2)."""
    rng = np.random.default_rng(seed)
    rows = []
    for (m, n, k, er) in shapes:
        f = 2.0 * m * n * k
        for c in at.candidates(m, n, k):
            if c.is_fp64:
                # split-K and the 64-row tile help only products with few output tiles
                tiles = math.ceil(m / c.tile_m) * math.ceil(n / 128)
                ks = c.ksplit if c.ksplit else 148 / tiles   # stream-K fills every SM
                t = f / 30e12 * max(1.0, 148 / tiles) / min(ks, max(1.0, 148 / tiles)) + 3e-6 * max(ks, 1)
                e = 1e-15 * math.sqrt(k / 1e3 / max(ks, 1))
            elif c.is_crt:
                L = sum(math.log2(p) for p in (256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211,
                                               199, 197, 193)[:c.splits])
                t = f * c.splits / 4.5e15 + 12.0 * (m * k + k * n + m * n) / 3e12
                e = max(2 * math.sqrt(k / 6) * 2.0 ** (-(math.floor(L) - 2) / 2), 5e-17)
            else:
                t = f * c.splits * (c.splits + 1) / 2 / 4.5e15 + 8.0 * (m * k + k * n) / 3e12
                e = max(10.0 ** (-8 - 2 * (c.splits - 4)) * (1 if er > 8 else 0.1), 5e-17)
            t *= math.exp(rng.normal(0, 0.03))
            rows.append({"m": m, "n": n, "k": k, "exp_range": er, "tile": c.tile, "splits": c.splits,
                         "seconds": t, "error": e})
    return rows


def test_candidates_and_features():
    cs = at.candidates()
    assert cs[0].tile == at.TILE_FP64 and cs[0].splits == 0 and cs[0].ksplit == 1
    assert [c.ksplit for c in cs if c.is_fp64 and c.tile_m == 128] == [1, 2, 4, 8, 16]
    # the second FP64 tile shape (64 x 128) is a candidate of its own, with its own tile id
    assert [(c.tile, c.ksplit) for c in cs if c.is_fp64 and c.tile_m == 64] == [(9, 1), (10, 2), (11, 4), (12, 8),
                                                                                (13, 0)]
    assert next(c for c in cs if c.tile == 13).name == "fp64t64sk"
    assert {c.tile_m for c in cs if not c.is_fp64} == {128}
    assert [c.splits for c in cs if c.form == "ozaki" and c.ksplit == 1] == list(range(3, 10))
    assert sorted({c.ksplit for c in cs if c.form == "ozaki"}) == [1, 4, 16]
    assert [c.splits for c in cs if c.is_crt] == list(at.CRT_MODULI) and {c.ksplit for c in cs if c.is_crt} == {1}
    assert len({c.name for c in cs}) == len(cs) == 5 + 5 + 3 * 7 + 7
    oz5 = next(c for c in cs if c.splits == 5)
    f = at.features(1024, 2048, 4096, 20, oz5)
    assert f[:3] == [10.0, 11.0, 12.0] and f[3:] == [20.0, 1.0, 5.0]
    # split-K candidates only where the K range has the blocks and the slices fit the workspace cap
    small = at.candidates(300, 300, 100)            # 4 K blocks
    assert [c.ksplit for c in small if c.is_fp64 and c.tile_m == 128] == [1, 2, 4]
    assert [c.ksplit for c in small if c.is_fp64 and c.tile_m == 64] == [1, 2, 4, 0]
    assert sorted({c.ksplit for c in small if c.form == "ozaki"}) == [1, 4]
    big = at.candidates(32768, 32768, 32768)
    assert [c.ksplit for c in big if c.is_fp64] == [1, 1, 0] and {c.ksplit for c in big} == {0, 1}
    # an Ozaki K slice needs K within one int32 accumulation
    assert at.ozaki_kmax(9) == 58240 and not at.splitk_applies(64, 64, 60000, 4, 9)
    assert at.splitk_applies(64, 64, 60000, 4, 8)


def test_random_shapes_and_memory_bound():
    shapes = at.random_shapes(500, seed=1)
    dims = np.array([s[:3] for s in shapes])
    assert dims.min() >= 256 and dims.max() <= 32768
    assert all(0 <= s[3] <= 40 for s in shapes)
    assert at.shape_fits(32768, 32768, 32768) and not at.shape_fits(65536, 65536, 32768)


def test_regression_baseline_and_choice():
    train = synthetic_rows(at.random_shapes(300, seed=2))
    held = synthetic_rows(at.random_shapes(60, seed=3))
    reg = at.RegressionModel().fit(train)
    c = at.choose(reg, 8192, 8192, 8192, 20, 1e-15)
    assert c.tile == at.TILE_CRT and c.splits in (15, 16)
    c = at.choose(reg, 8192, 8192, 8192, 20, 1e-15, [x for x in at.candidates(8192, 8192, 8192) if x.form == "ozaki"])
    assert c.form == "ozaki" and c.splits in (8, 9)
    r = at.regret(reg, held, 1e-15)
    assert r["shapes"] == 60 and r["mean_regret"] >= 0.0
    # an oracle that knows the measurements has zero regret
    class Perfect:
        def predict(self, m, n, k, er, cands):
            out = []
            for cc in cands:
                x = next(x for x in held if (x["m"], x["n"], x["k"], x["exp_range"], x["tile"], x["splits"]) ==
                         (m, n, k, er, cc.tile, cc.splits))
                out.append((x["seconds"], x["error"]))
            return out
    p = at.regret(Perfect(), held, 1e-15, crt_margin=1.0)  # exact predictions need no guard band
    assert p["mean_regret"] == 0.0 and p["misses"] == 0


def test_sweep_db_append_and_resume(tmp_path):
    db = at.SweepDB(tmp_path / "s.jsonl")
    rows = synthetic_rows([(256, 512, 1024, 3)])
    db.add(rows[:3])
    db2 = at.SweepDB(tmp_path / "s.jsonl")
    assert len(db2.rows) == 3 and db2.has(256, 512, 1024, 3, at.candidates()[0])
    assert not db2.has(256, 512, 1024, 3, at.candidates()[5])
    assert len(db2.digest()) == 16


def test_refresh_rows_measures_again_with_the_sweep_inputs(tmp_path, monkeypatch):
    """refresh_rows measures again only the rows of the given tile ids, with the seed the sweep
    used for that shape (train: its index; held-out: 100000 + index), keeps the row order and the
    set, and skips rows it has already refreshed."""
    train = [s for s in at.random_shapes(8, 1) if at.shape_fits(*s[:3])][:4]
    held = [s for s in at.random_shapes(4, 2) if at.shape_fits(*s[:3])][:2]
    rows = []
    for i, s in enumerate(train):
        r = synthetic_rows([s])[i % 3]
        r["set"] = "train"
        rows.append(r)
    for s in held:
        for r in synthetic_rows([s])[:4]:
            r["set"] = "heldout"
            rows.append(r)
    db = at.SweepDB(tmp_path / "s.jsonl")
    db.add(rows)
    tiles = {at.TILE_FP64, at.TILE_FP64_K2}
    calls = []

    def fake_measure(m, n, k, er, cands, seed=0, **kw):
        calls.append(((m, n, k, er), tuple(c.tile for c in cands), seed))
        return [{"m": m, "n": n, "k": k, "exp_range": er, "tile": c.tile, "splits": c.splits, "seconds": 1.0,
                 "tflops": 1.0, "error": 1e-16} for c in cands]

    monkeypatch.setattr(at, "measure", fake_measure)
    out, done, total = at.refresh_rows(tmp_path / "s.jsonl", tiles, train_shapes=4, heldout_shapes=2, log=lambda *_: None)
    again = at.SweepDB(tmp_path / "s.jsonl").rows
    assert [at.SweepDB.key(r) for r in again] == [at.SweepDB.key(r) for r in rows]
    assert [r["set"] for r in again] == [r["set"] for r in rows]
    for old, new in zip(rows, again):
        assert (new["seconds"] == 1.0) == (old["tile"] in tiles)
        assert ("refreshed" in new) == (old["tile"] in tiles)
    seeds = {s: i for i, s in enumerate(train)}
    seeds.update({s: 100000 + i for i, s in enumerate(held)})
    assert calls and all(seed == seeds[shape] for shape, _, seed in calls)
    assert done == total == len(calls)
    calls.clear()
    at.refresh_rows(tmp_path / "s.jsonl", tiles, train_shapes=4, heldout_shapes=2, log=lambda *_: None)
    assert calls == []
