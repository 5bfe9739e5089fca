"""Surrogate-steered sweeps: the network proposes the next sweep points, the batched hydro
runs them and judges the network's error.

The question a sweep asks is often a level set of one result over the parameter space,
for example the disks whose m = 2 mode grows at a given rate (gamma = g*, the contour
between slowly and quickly growing disks).  A uniform draw of the sweep law spends most
of its hydro runs far from that contour.  The steered sweep:

  1. draws a large candidate pool from the sweep law (diskgpu.sweep.draw);
  2. each round, asks the surrogate for gamma on the pool and proposes the `batch` not yet
     run candidates closest to the contour, spread out: a candidate closer than
     `min_dist` (in standardised parameters) to an already proposed one is skipped;
  3. runs the proposals with the hydro (one batched launch sequence) and keeps the hydro's
     values, never the network's: the hydro is the judge;
  4. records the network's error on every run point; when a round's median error exceeds
     `bound`, the hydro takes over as the fallback: the network is refined on all hydro
     results so far (its own training set replayed beside them) before it proposes again,
     and the round is marked as a fallback round.

steer() and uniform() take the predictor and the hydro as callables, so the logic can be
exercised with stand-ins; hydro_gamma() is the real hydro (batched mixed-precision runs,
gamma from the linear phase of each disk's mode records).
"""
from __future__ import annotations

import numpy as np

from . import sweep as S


def features(points):
    """(Q_min, M_d/M_*, softening/r, Gamma) rows of sweep points: the surrogate's inputs."""
    return np.array([[p.Qmin, p.mass_ratio, p.soft_over_r, p.gamma] for p in points], dtype=np.float64)


def _standardise(X):
    lo = np.array([1.0, 0.2, 0.05, 1.5])
    span = np.array([1.0, 0.8, 0.15, 0.5])
    return (X - lo) / span


def propose(pred, X, taken, target, batch, min_dist):
    """Indices of the `batch` untaken candidates whose predicted value is closest to
    `target`, skipping any closer than min_dist (standardised) to one already chosen."""
    order = np.argsort(np.abs(pred - target))
    Z = _standardise(X)
    chosen = []
    for i in order:
        if taken[i]:
            continue
        if chosen and np.min(np.linalg.norm(Z[chosen] - Z[i], axis=1)) < min_dist:
            continue
        chosen.append(int(i))
        if len(chosen) == batch:
            break
    return chosen


def steer(predict, hydro, target, tol, budget, batch=16, pool=4096, seed=777, grid=256, bound=0.05,
          min_dist=0.05, refine=None):
    """Run at most `budget` hydro runs in rounds of `batch`, proposed by the surrogate.

    predict(X) -> predicted gamma for feature rows X; hydro(points) -> measured gamma per
    point; refine(X, y) (optional) updates the predictor on hydro results.  Returns a dict
    with the points run, the hydro values, the network's predictions and errors per run,
    the rounds that fell back to refining, and `hits`: runs whose hydro value lies within
    tol of target."""
    pts = S.draw(pool, seed=seed, grids=(grid,))
    X = features(pts)
    taken = np.zeros(len(pts), dtype=bool)
    run_idx, y_hydro, y_pred, fallback_rounds = [], [], [], []
    r = 0
    while len(run_idx) < budget:
        pred = np.asarray(predict(X), dtype=np.float64)
        nb = min(batch, budget - len(run_idx))
        idx = propose(pred, X, taken, target, nb, min_dist)
        if not idx:
            break
        taken[idx] = True
        y = np.asarray(hydro([pts[i] for i in idx]), dtype=np.float64)
        err = np.abs(pred[idx] - y)
        run_idx += idx
        y_hydro += y.tolist()
        y_pred += pred[idx].tolist()
        if np.nanmedian(err) > bound:
            fallback_rounds.append(r)
            if refine is not None:
                ok = np.isfinite(y_hydro)
                refine(X[run_idx][ok], np.asarray(y_hydro)[ok])
        r += 1
    y_hydro = np.asarray(y_hydro)
    y_pred = np.asarray(y_pred)
    return {"points": [pts[i] for i in run_idx], "gamma_hydro": y_hydro, "gamma_pred": y_pred,
            "abs_err": np.abs(y_pred - y_hydro), "fallback_rounds": fallback_rounds, "rounds": r,
            "hits": int(np.sum(np.abs(y_hydro - target) <= tol))}


def uniform(hydro, target, tol, budget, seed=778, grid=256):
    """The same budget spent on a uniform draw of the sweep law."""
    pts = S.draw(budget, seed=seed, grids=(grid,))
    y = np.asarray(hydro(pts), dtype=np.float64)
    return {"points": pts, "gamma_hydro": y, "hits": int(np.sum(np.abs(y - target) <= tol))}


def hydro_gamma(points, tlim=16.0, dtout=0.25, device=-1):
    """gamma of each sweep point from the batched mixed-precision hydro: the linear phase
    of its m = 2 records (t >= 1 until |C2|/|C0| > 0.05), NaN where no fit is possible."""
    from . import Batch
    from .analysis import linear_phase

    params = [S.point_params(p, "mixed", device) for p in points]
    out = []
    with Batch(params) as b:
        b.init_standard()
        recs, _, _ = b.advance(tlim, dtout=dtout)
    for rec in recs:
        try:
            g, _, _ = linear_phase(*rec.T)
        except ValueError:
            g = float("nan")
        out.append(g)
    return out


def surrogate_refiner(sur, replay_X=None, replay_Y=None, epochs=60, lr=5e-4):
    """refine(X, gamma) for steer(): a few epochs on the hydro results (only the gamma
    output is known for them; the other two outputs keep the network's own values as
    targets) with the training set replayed beside them, standardisation unchanged."""
    def refine(X, g):
        Yn = sur.predict(X)
        Yn[:, 0] = g
        XX, YY = X, Yn
        if replay_X is not None:
            XX = np.concatenate([replay_X, X])
            YY = np.concatenate([replay_Y, Yn])
        Xs, Ys = sur._norm(XX, YY)
        rng = np.random.default_rng(0)
        for _ in range(epochs):
            perm = rng.permutation(len(Xs))
            for s in range(0, len(Xs), 256):
                i = perm[s: s + 256]
                sur.net.train_step(Xs[i], Ys[i], lr)
    return refine
