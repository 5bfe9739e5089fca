"""Build the surrogate's training set from batched hydro runs and train it on the GPU.

  python -m diskgpu.train_surrogate --runs 4096 --grid 256 --tlim 16 --batch 1024 --out <dir>

(the defaults: 4096 sweep-law runs at 256^2 to t = 16, the set the shipped network in
diskgpu/data was trained on; about ten minutes of batched hydro on one B200).

Draws sweep points with the sweep law (diskgpu.sweep.draw, fixed seed), runs them in
batches of disks advanced together (dg_batch, mixed precision; same-grid disks step as one
group), fits gamma / Omega_p / saturated |C2|/|C0| from each disk's mode records, trains
the MLP on 95 % and reports its error on the 5 % held out against the hydro's own values.
Writes sweep_<grid>_dataset.npz, surrogate.npz (network, standardisation and report) and
report.json to --out.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import MIXED, Batch, params_physical
from . import sweep as S
from .analysis import linear_phase
from .surrogate import Surrogate


def fit_record(rec):
    """gamma / Omega_p over the linear phase and the late-time |C2|/|C0| of one disk (mean of
    the last quarter of its records)."""
    t, c0, c2, a2 = rec[:, 0], rec[:, 1], rec[:, 2], rec[:, 3]
    g, w, _ = linear_phase(t, c0, c2, a2)
    ratio = c2 / c0
    tail = ratio[-max(4, len(ratio) // 4):]
    return g, w, float(np.mean(tail))


def run_points(pts, tlim, batch=128, dtout=0.25):
    rows = []
    for s in range(0, len(pts), batch):
        chunk = pts[s: s + batch]
        params = []
        for pt in chunk:
            p, q = params_physical(pt.Qmin, pt.mass_ratio, pt.soft_over_r, pt.gamma)
            p.Nu = p.Nphi = pt.N
            p.amp, p.phase0, p.precision = pt.amp, pt.phase0, MIXED
            params.append((p, q))
        with Batch([p for p, _ in params]) as b:
            b.init_standard()
            recs, t, steps = b.advance(tlim, dtout=dtout, steps_per_launch=64)
        for pt, (p, q), rec, st in zip(chunk, params, recs, steps):
            g, w, sr = fit_record(rec)
            rows.append([pt.Qmin, pt.mass_ratio, pt.soft_over_r, pt.gamma, q, g, w, sr, st])
    return np.array(rows)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--runs", type=int, default=4096)
    ap.add_argument("--grid", type=int, default=256)
    ap.add_argument("--tlim", type=float, default=16.0)
    ap.add_argument("--batch", type=int, default=1024)
    ap.add_argument("--seed", type=int, default=12345)
    ap.add_argument("--epochs", type=int, default=400)
    ap.add_argument("--out", default=".")
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    pts = S.draw(a.runs, seed=a.seed, grids=(a.grid,))
    t0 = time.time()
    data = run_points(pts, a.tlim, batch=a.batch)
    t_hydro = time.time() - t0
    np.savez(os.path.join(a.out, f"sweep_{a.grid}_dataset.npz"), data=data,
             columns=np.array(["Qmin", "mass_ratio", "soft_over_r", "gamma_eos", "Qmin_achieved", "gamma",
                               "omega_p", "sat_ratio", "steps"]))
    X, Y = data[:, :4], data[:, 5:8]
    ok = np.all(np.isfinite(Y), axis=1)
    X, Y = X[ok], Y[ok]
    n_hold = max(1, int(round(0.05 * len(X))))
    Xtr, Ytr, Xho, Yho = X[:-n_hold], Y[:-n_hold], X[-n_hold:], Y[-n_hold:]
    sur = Surrogate(seed=1)
    t1 = time.time()
    hist = sur.fit(Xtr, Ytr, epochs=a.epochs, batch=min(256, len(Xtr)), lr=2e-3)
    t_train = time.time() - t1
    t2 = time.time()
    pred = sur.predict(Xho)
    t_pred = time.time() - t2
    err = np.abs(pred - Yho)
    rep = {
        "runs": int(a.runs), "grid": a.grid, "tlim": a.tlim, "finite": int(ok.sum()), "held_out": int(n_hold),
        "hydro_seconds": t_hydro, "train_seconds": t_train, "predict_seconds_held_out": t_pred,
        "hydro_seconds_per_run": t_hydro / a.runs,
        "mae_held_out": dict(zip(["gamma", "omega_p", "sat_ratio"], err.mean(axis=0).tolist())),
        "target_std": dict(zip(["gamma", "omega_p", "sat_ratio"], Y.std(axis=0).tolist())),
        "loss_first_last": [hist[0], hist[-1]],
    }
    sur.save(os.path.join(a.out, "surrogate.npz"), report=rep)
    with open(os.path.join(a.out, "report.json"), "w") as f:
        json.dump(rep, f, indent=1)
    print(json.dumps(rep))


if __name__ == "__main__":
    main()
