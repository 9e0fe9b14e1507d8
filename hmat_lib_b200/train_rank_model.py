"""Trains the library's rank model and writes it to a file.

    python -m hmat_lib_b200.train_rank_model --draws 2000 --out hmat_lib_b200/rank_model.f32

Every draw is a seeded kernel matrix (exponential or Matern-3/2 kernel with
length l ~ logU[0.02, 0.5] plus 1e-2 I, on 1D sorted, 2D or 3D Morton-ordered
points, n in {2048, 4096, 8192, 16384}, leaf 128) compressed from its points
(matrix-free build, so the kernel length reaches the features) by the plain
adaptive build at tol 1e-8 with feature recording on: each sketched block
contributes its 8 features and its Frobenius epsilon-rank (the training
target, as log2(rank + 1)).  The network is then trained by
the library's GPU kernels; the last 10% of the draws are held out and the
summary (sample counts, loss curve, held-out rank error, how often the
one-shot sketch width covers the true epsilon-rank) is written next to the
model as JSON.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import time

import numpy as np

from . import abi
from . import rank_model as RM
from . import workloads as W
from .hodlr import DeviceTree, HodlrError

KIND = {"gaussian": 0, "matern32": 1, "exponential": 2}


def draws(count: int, seed: int):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        out.append(dict(
            kind=str(rng.choice(["exponential", "matern32"])),
            dim=int(rng.choice([1, 2, 3], p=[0.1, 0.5, 0.4])),
            length=float(math.exp(rng.uniform(math.log(0.02), math.log(0.5)))),
            n=int(rng.choice([2048, 4096, 8192, 16384])),
            seed=int(seed * 100000 + i)))
    return out


def one_shot_width(r_pred: np.ndarray, margin: float = 0.1, extra: int = 40) -> np.ndarray:
    """First sketch width the build uses for a predicted rank (whole panels)."""
    w = np.ceil(np.maximum(r_pred, 1.0) * (1.0 + margin)) + extra
    return np.ceil(w / 32.0) * 32.0


def collect(specs, max_seconds: float):
    import torch
    lib = abi.load()
    lib.hodlr_b200_set_option(b"record_features", 1.0)
    rows, owner, skipped, t0 = [], [], 0, time.perf_counter()
    try:
        for i, d in enumerate(specs):
            if time.perf_counter() - t0 > max_seconds:
                break
            n, dim = d["n"], d["dim"]
            pts = W.points_morton(n, dim, d["seed"]) if dim > 1 else \
                W.points_1d_sorted(n, d["seed"])
            d_pts = torch.from_numpy(np.asfortranarray(pts).T.copy().reshape(-1)).cuda()
            h = (n // 128).bit_length() - 1
            try:
                t = DeviceTree.build_kernel(d_pts.data_ptr(), n, dim, KIND[d["kind"]],
                                            d["length"], 1e-2, h, 1e-8)
            except HodlrError as e:
                # a block outgrew the memory-bounded sketch (no label), or the
                # build failed otherwise
                skipped += 1
                print(f"draw {i}: build failed: {e}", flush=True)
                continue
            if (i + 1) % 100 == 0:
                print(f"{i + 1} draws, {time.perf_counter() - t0:.0f} s", flush=True)
            f = RM.build_features()
            t.free()
            rows.append(f)
            owner += [i] * len(f)
    finally:
        lib.hodlr_b200_set_option(b"record_features", 0.0)
    data = np.concatenate(rows) if rows else np.zeros((0, RM.FEATURE_ROW), np.float32)
    return data, np.array(owner), skipped, len(rows), time.perf_counter() - t0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--draws", type=int, default=2000)
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--max-minutes", type=float, default=25.0,
                    help="stop drawing new matrices after this long")
    ap.add_argument("--out", default=RM.MODEL_FILE)
    ap.add_argument("--save-data", default=None,
                    help="also write the collected rows and their draw indices (.npz)")
    ap.add_argument("--from-data", default=None,
                    help="train on rows saved by --save-data instead of drawing")
    args = ap.parse_args()

    if args.from_data:
        z = np.load(args.from_data)
        data, owner = z["data"], z["owner"]
        skipped, used, secs = int(z["skipped"]), int(z["used"]), float(z["secs"])
    else:
        specs = draws(args.draws, args.seed)
        data, owner, skipped, used, secs = collect(specs, args.max_minutes * 60.0)
    if args.save_data:
        np.savez(args.save_data, data=data, owner=owner, skipped=skipped, used=used, secs=secs)
    x, target, rank_fro = data[:, :8], RM.targets_of_ranks(data[:, 13]), data[:, 13]
    drawn = np.unique(owner)
    cut = drawn[int(0.9 * len(drawn))] if len(drawn) > 1 else np.inf
    train = owner < cut
    hold = ~train
    t0 = time.perf_counter()
    p, log = RM.train(x[train], target[train], steps=args.steps, batch=args.batch, lr=args.lr,
                      seed=args.seed)
    train_s = time.perf_counter() - t0
    summary = dict(draws_requested=args.draws, draws_used=used, draws_skipped=skipped,
                   collect_seconds=secs, samples=int(len(x)), train_samples=int(train.sum()),
                   holdout_samples=int(hold.sum()), steps=args.steps, batch=args.batch,
                   lr=args.lr, train_seconds=train_s, loss_every_100_steps=[float(v) for v in log])
    if hold.any():
        r_pred = np.exp2(RM.predict(p, x[hold]).astype(np.float64)) - 1.0
        r_true = rank_fro[hold].astype(np.float64)
        rel = np.abs(r_pred - r_true) / np.maximum(r_true, 1.0)
        covered = one_shot_width(r_pred) >= r_true + 8
        summary.update(holdout_median_rel_rank_error=float(np.median(rel)),
                       holdout_p90_rel_rank_error=float(np.quantile(rel, 0.9)),
                       holdout_one_shot_covers=float(np.mean(covered)),
                       holdout_mse_log2=float(np.mean((np.log2(r_pred + 1) -
                                                       np.log2(r_true + 1)) ** 2)))
    p.astype(np.float32).tofile(args.out)
    with open(args.out + ".json", "w") as fh:
        json.dump(summary, fh, indent=1)
    print(json.dumps({k: v for k, v in summary.items() if k != "loss_every_100_steps"}))


if __name__ == "__main__":
    main()
