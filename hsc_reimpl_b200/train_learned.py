"""Train the learned polynomial preconditioner on the GPU and write the model file.

    python -m hsc_reimpl_b200.train_learned [--trajectories 67 --steps 300] \
        [--out hsc_reimpl_b200/learned_poly_model.npz] [--report report.json]

Generates the training systems with the solver (learned.generate), trains the
16-64-64-8 MLP with the library's kernels (learned.Trainer), evaluates it
against the plain Neumann series on held-out trajectories (learned.evaluate)
and saves the BF16 parameters with the training record.
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np

from . import learned as L


def log(msg):
    print(msg, flush=True)


def split(data, idx):
    return {k: v[idx] for k, v in data.items()}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--trajectories", type=int, default=67)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--val-trajectories", type=int, default=3)
    ap.add_argument("--variants", type=int, default=4, help="node-position variants the trajectories cycle over")
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--batch", type=int, default=512)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--eval-steps", type=int, default=40)
    ap.add_argument("--eval-seeds", type=int, nargs="*", default=[9001, 9002])
    ap.add_argument("--dataset", default=None, help="reuse a dataset .npz instead of generating one")
    ap.add_argument("--save-dataset", default=None)
    ap.add_argument("--out", default=str(L.MODEL_PATH))
    ap.add_argument("--report", default=None)
    a = ap.parse_args(argv)
    t0 = time.time()
    bases = {}

    def base(v):
        if v not in bases:
            bases[v] = L.VehicleBase(v)
        return bases[v]

    if a.dataset:
        z = np.load(a.dataset)
        train = {k: z[f"train_{k}"] for k in ("features", "theta", "tau", "teacher", "teacher_iters")}
        val = {k: z[f"val_{k}"] for k in ("features", "theta", "tau", "teacher", "teacher_iters")}
    else:
        trajs = [L.VehicleTrajectory(base(i % a.variants), seed=i, steps=a.steps) for i in range(a.trajectories)]
        vtrajs = [L.VehicleTrajectory(base(i % a.variants), seed=5000 + i, steps=a.steps)
                  for i in range(a.val_trajectories)]
        tg = time.time()
        train = L.generate(trajs, log=log)
        val = L.generate(vtrajs, log=log)
        gen_s = time.time() - tg
        log(f"generated {len(train['features'])} training + {len(val['features'])} validation systems in {gen_s:.0f} s")
        if a.save_dataset:
            np.savez(a.save_dataset, **{f"train_{k}": v for k, v in train.items()},
                     **{f"val_{k}": v for k, v in val.items()})
    tr = L.Trainer(L.init_params(0), lr=a.lr, seed=0)
    l0 = tr.evaluate_loss(val)
    tt = time.time()
    hist = tr.fit(train, epochs=a.epochs, batch=a.batch, val=val, log=log)
    train_s = time.time() - tt
    params = tr.params_fp32()
    bits = L.bf16_bits(params)
    ev_variant = a.variants  # node positions not seen in training
    etrajs = [L.VehicleTrajectory(base(ev_variant), seed=s, steps=a.eval_steps) for s in a.eval_seeds]
    res = L.evaluate(bits, etrajs, log=log)
    summary = {k: {"mean_iterations": float(v["iters"].mean()), "median_iterations": float(np.median(v["iters"])),
                   "mean_pcg_ms": float(v["pcg_ms"].mean()), "mean_total_ms": float(v["total_ms"].mean()),
                   "max_full_relative_residual": float(v["full"].max()), "fallbacks": int(v["fallback"].sum())}
               for k, v in res.items()}
    meta = {"train_systems": int(len(train["features"])), "val_systems": int(len(val["features"])),
            "trajectories": a.trajectories, "steps": a.steps, "variants": a.variants, "epochs": a.epochs,
            "batch": a.batch, "lr": a.lr, "val_loss_init": l0, "val_loss_final": hist[-1].get("val_loss"),
            "train_seconds": train_s, "teacher_mean_iterations": float(np.mean(train["teacher_iters"])),
            "eval_variant": ev_variant, "eval_seeds": list(a.eval_seeds), "eval_steps": a.eval_steps,
            "eval": summary, "wall_seconds": time.time() - t0}
    L.save_model(a.out, params, meta)
    log(json.dumps(meta, indent=1))
    if a.report:
        with open(a.report, "w") as f:
            json.dump({"meta": meta, "history": hist}, f, indent=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
