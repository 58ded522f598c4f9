"""Train the rank MLP of the learned-rank sparsification (needs a GPU).

Training pairs are (features of an interface's compression matrix, kept
rank / min(m, w)) logged by plain factorizations (column-pivoted QR of every
interface) of synthetic 3-D diffusion matrices:

  * high-contrast channels k = 10^(3 sign g), g a Gaussian random field of
    correlation length 8 (the learned-rank workload), seeds 10-49, at
    tol in {1e-1, 1e-2, 1e-3}, on the 64^3 grid (12 levels) and the 32^3
    grid (10 levels);
  * log-normal coefficients k = exp(g) (the mixed-precision workload), seeds
    10-29, same tolerances, 64^3.

The network trains on the GPU with the library's own kernels (spq_mlp_train:
forward, backward and Adam in learned.cu).  It is then evaluated on the
held-out channel seeds 50-59 at 64^3, factorizing each matrix three ways:
plain pivoted QR, learned ranks with the trained network, and learned ranks
with a constant network that always predicts the training mean (the method
without the trained network).  Reported per tolerance: the fraction of
interfaces whose learned rank is within +-2 of the plain rank, the fallback
rate, the total sketch width and the factorization time.

Writes rank_mlp.npz (params, mean, std, meta) and report.json next to this
file unless --out is given.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from pspaqr_public_b200 import ParTree, scale_columns  # noqa: E402
from pspaqr_public_b200 import matrices as M  # noqa: E402
from pspaqr_public_b200 import tree as T  # noqa: E402

TOLS = (1e-1, 1e-2, 1e-3)
OVERSAMPLE = 32


def levels_for(n):
    return int(round(np.log2(n ** 3 / 128))) + 1


def make_tree(n, family, seed):
    gen = M.diffusion_binary if family == "binary" else M.diffusion_lognormal
    cp, ri, v = gen(n, 3, seed=seed)
    t = ParTree(levels_for(n), 0)
    t.set_coords_tensor(n, 3)
    t.partition((cp, ri, scale_columns(cp, v)))
    return t


def log_pairs(n, family, seeds, tols, verbose=True):
    feats, ys = [], []
    for s in seeds:
        t0 = time.time()
        t = make_tree(n, family, s)
        t.set_rank_log(True)
        for tol in tols:
            t.set_tol(tol)
            t.assemble()
            t.factorize()
        log = t.rank_log()
        feats.append(log["features"])
        ys.append(log["rank"] / np.maximum(log["kmin"], 1))
        if verbose:
            print(f"  {family} {n}^3 seed {s}: {len(log['rank'])} pairs ({time.time() - t0:.1f} s, "
                  f"device pool {t.pool_bytes() / 2**30:.1f} GiB)", flush=True)
        del t
    return np.concatenate(feats), np.concatenate(ys).astype(np.float32)


def constant_model(mean_y, nf):
    P, F = T.rank_model_size()
    p = np.zeros(P, np.float32)
    p[-1] = np.log(mean_y / (1.0 - mean_y))
    return {"params": p, "mean": np.zeros(F, np.float32), "std": np.ones(F, np.float32)}


def calibrate(model, mean_y, seeds, tols, q=0.95, n=64):
    """Sketch margins per tolerance: the q-quantile of (kept fraction - prediction)
    over the plain factorizations' pairs of the training seeds, for the network
    and for the constant predictor (prediction = training mean)."""
    out, cout = {}, {}
    for tol in tols:
        feats, ys = [], []
        for s in seeds:
            t = make_tree(n, "binary", s)
            t.set_tol(tol)
            t.set_rank_log(True)
            t.assemble()
            t.factorize()
            log = t.rank_log()
            feats.append(log["features"])
            ys.append(log["rank"] / np.maximum(log["kmin"], 1))
            del t
        X = np.concatenate(feats)
        y = np.concatenate(ys)
        p = T.mlp_predict(model["params"], (X - model["mean"]) / model["std"])
        out[repr(tol)] = float(max(np.quantile(y - p, q), 0.0))
        cout[repr(tol)] = float(max(np.quantile(y - mean_y, q), 0.0))
        print(f"calibration tol {tol}: {len(y)} pairs, margin {out[repr(tol)]:.4f} (network), "
              f"{cout[repr(tol)]:.4f} (constant)", flush=True)
    return out, cout


def evaluate(model, const, seeds, tols, n=64, oversample=OVERSAMPLE, margins=None, cmargins=None):
    rows = []
    for tol in tols:
        if margins is not None:
            model = dict(model, margin=margins[repr(tol)])
            const = dict(const, margin=cmargins[repr(tol)])
        agg = {"tol": tol, "interfaces": 0}
        for name in ("plain", "learned", "constant"):
            agg[name + "_s"] = 0.0
        for key in ("within2", "fallback", "sketch_cols", "c_within2", "c_fallback", "c_sketch_cols"):
            agg[key] = 0
        for s in seeds:
            t = make_tree(n, "binary", s)
            t.set_tol(tol)
            t.set_rank_model(None)
            t.assemble()
            t.factorize()
            t.assemble()
            t.factorize()
            agg["plain_s"] += t.times()["factorize"]
            cl = t.clusters()
            sp = np.array([c["sparsify"] for c in cl]) > 0
            plain = np.array([c["rank"] for c in cl])[sp]
            for name, m in (("learned", model), ("constant", const)):
                t.set_rank_model(m, oversample)
                t.assemble()
                t.factorize()
                cnt = t.learned_counts()
                ranks = np.array([c["rank"] for c in t.clusters()])[sp]
                pre = "" if name == "learned" else "c_"
                agg[pre + "within2"] += int(np.sum(np.abs(ranks - plain) <= 2))
                agg[pre + "fallback"] += int(cnt["fallback"])
                agg[pre + "sketch_cols"] += int(cnt["sketch_columns"])
                agg[name + "_s"] += t.times()["factorize"]
            agg["interfaces"] += int(sp.sum())
            del t
        N = max(agg["interfaces"], 1)
        rows.append({
            "tol": tol, "interfaces": agg["interfaces"], "oversample": oversample,
            "margin": model.get("margin", 0.0), "constant_margin": const.get("margin", 0.0),
            "learned": {"within2": agg["within2"] / N, "fallback_rate": agg["fallback"] / N,
                        "sketch_columns": agg["sketch_cols"], "factorize_s": agg["learned_s"] / len(seeds)},
            "constant": {"within2": agg["c_within2"] / N, "fallback_rate": agg["c_fallback"] / N,
                         "sketch_columns": agg["c_sketch_cols"], "factorize_s": agg["constant_s"] / len(seeds)},
            "plain_factorize_s": agg["plain_s"] / len(seeds),
        })
        print(json.dumps(rows[-1]), flush=True)
    return rows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--train-seeds", default="10-49")
    ap.add_argument("--lognormal-seeds", default="10-29")
    ap.add_argument("--eval-seeds", default="50-59")
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--no-eval", action="store_true")
    ap.add_argument("--eval-only", action="store_true", help="evaluate the model already in --out")
    ap.add_argument("--oversample", type=int, default=OVERSAMPLE,
                    help="sketch columns beyond the predicted rank in the evaluation")
    ap.add_argument("--report", default="report.json", help="report file name (in --out)")
    ap.add_argument("--calibrate", default="",
                    help="training seeds (e.g. 10-19) to calibrate the sketch margins on; stored in the model's meta")
    ap.add_argument("--quantile", type=float, default=0.95, help="quantile of the calibrated margins")
    args = ap.parse_args()

    def rng(s):
        a, b = (int(x) for x in s.split("-"))
        return list(range(a, b + 1))

    if args.eval_only:
        path = os.path.join(args.out, "rank_mlp.npz")
        z = np.load(path)
        meta = json.loads(str(z["meta"]))
        model = {k: z[k].astype(np.float32) for k in ("params", "mean", "std")}
        const = constant_model(meta["mean_target"], len(model["mean"]))
        if args.calibrate:
            m, c = calibrate(model, meta["mean_target"], rng(args.calibrate), TOLS, args.quantile)
            meta.update(margin_by_tol=m, const_margin_by_tol=c, margin_quantile=args.quantile,
                        margin_seeds=args.calibrate)
            np.savez(path, params=model["params"], mean=model["mean"], std=model["std"], loss=z["loss"],
                     meta=json.dumps(meta))
        margins = meta.get("margin_by_tol")
        report = {"meta": meta, "loss": z["loss"].tolist(),
                  "eval": evaluate(model, const, rng(args.eval_seeds), TOLS, oversample=args.oversample,
                                   margins=margins, cmargins=meta.get("const_margin_by_tol"))}
        with open(os.path.join(args.out, args.report), "w") as f:
            json.dump(report, f, indent=1)
        return
    t0 = time.time()
    parts = [log_pairs(64, "binary", rng(args.train_seeds), TOLS),
             log_pairs(32, "binary", rng(args.train_seeds), TOLS),
             log_pairs(64, "lognormal", rng(args.lognormal_seeds), TOLS)]
    X = np.concatenate([p[0] for p in parts])
    y = np.concatenate([p[1] for p in parts])
    print(f"{len(y)} training pairs in {time.time() - t0:.0f} s", flush=True)
    mean = X.mean(0).astype(np.float32)
    std = (X.std(0) + 1e-3).astype(np.float32)
    Xs = (X - mean) / std
    params = T.mlp_init(0)
    t1 = time.time()
    params, h1 = T.mlp_train(params, Xs, y, epochs=args.epochs, batch=4096, lr=3e-3, seed=1)
    params, h2 = T.mlp_train(params, Xs, y, epochs=args.epochs // 2, batch=4096, lr=5e-4, seed=2)
    hist = np.concatenate([h1, h2])
    print(f"trained in {time.time() - t1:.1f} s, loss {hist[0]:.5f} -> {hist[-1]:.5f}", flush=True)
    model = {"params": params, "mean": mean, "std": std}
    os.makedirs(args.out, exist_ok=True)
    meta = {"train_pairs": int(len(y)), "train_seeds_binary": args.train_seeds,
            "train_seeds_lognormal": args.lognormal_seeds, "tols": list(TOLS), "epochs": int(len(hist)),
            "final_loss": float(hist[-1]), "oversample": OVERSAMPLE, "mean_target": float(y.mean())}
    np.savez(os.path.join(args.out, "rank_mlp.npz"), params=params, mean=mean, std=std,
             loss=hist, meta=json.dumps(meta))
    report = {"meta": meta, "loss": hist.tolist()}
    if not args.no_eval:
        const = constant_model(float(y.mean()), X.shape[1])
        report["eval"] = evaluate(model, const, rng(args.eval_seeds), TOLS)
    with open(os.path.join(args.out, "report.json"), "w") as f:
        json.dump(report, f, indent=1)
    print("wrote", os.path.join(args.out, "rank_mlp.npz"), flush=True)


if __name__ == "__main__":
    main()
