"""Golden record for the surrogate-seeded lka98 eigen-solve (tests/test_surrogate_seed.py).

Runs the reference's own lka98.eigensolve on its standard disk (lka98/model.py) at
N = 100 and N = 300: the default solve_mode (a contour of 4 x 160 dlogdet calls around the
fixed LKA98 value, then Newton; eigensolve.py:156-211) and the seeded route (a contour of
4 x 16 calls around the shipped surrogate's prediction, then Newton), counting dlogdet
calls and wall time.  Needs the reference tree (lka98 is imported from it) and
numpy/scipy; no GPU:

    python tests/golden/make_lka98_seed.py [--ref REFERENCE_ROOT (default: $HEAVY_DISKS_REFERENCE)] [--sizes 100 300]
"""
import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "heavy-disks_b200"))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))

import numpy as np  # noqa: E402


def surrogate_seed():
    """(seed, prediction) of the shipped surrogate for the standard disk, evaluated by the
    FP64 oracle network (the same parameters the GPU network uses)."""
    import mlp_ref
    from diskgpu.surrogate import TRAINED, lka98_features, lka98_omega_guess, read_surrogate
    d = read_surrogate(TRAINED)
    n_in, width, depth, n_out = d["shape"]
    x = (lka98_features() - d["xm"]) / d["xs"]
    y = mlp_ref.forward(d["params"].astype(np.float64), x, n_in, width, depth, n_out)
    y = np.asarray(y[0] if isinstance(y, tuple) else y)[0] * d["ys"] + d["ym"]
    return lka98_omega_guess(y[0], y[1]), y


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("HEAVY_DISKS_REFERENCE", "/root/reference"))
    ap.add_argument("--sizes", type=int, nargs="+", default=[100, 300])
    a = ap.parse_args()
    sys.path.insert(0, a.ref)
    from lka98.eigensolve import LinearProblem, contour_root, solve_mode
    from lka98.model import DiskModel

    calls = {"n": 0}
    orig = LinearProblem.dlogdet

    def counted(self, w, h=1e-6):
        calls["n"] += 1
        return orig(self, w, h)

    LinearProblem.dlogdet = counted
    seed, pred = surrogate_seed()
    out = {"seed": [seed.real, seed.imag],
           "prediction": {"gamma": float(pred[0]), "omega_p": float(pred[1]), "sat_ratio": float(pred[2])},
           "cases": []}
    for N in a.sizes:
        P = LinearProblem.build(DiskModel(), N)
        calls["n"] = 0
        t0 = time.perf_counter()
        w, _, _, _ = solve_mode(P)
        t_def, c_def = time.perf_counter() - t0, calls["n"]
        calls["n"] = 0
        t0 = time.perf_counter()
        w0 = contour_root(P, seed, 0.35, 0.35, n=16)
        w2, _, _, _ = solve_mode(P, omega_guess=w0, localize=False)
        t_seed, c_seed = time.perf_counter() - t0, calls["n"]
        calls["n"] = 0
        w3, _, _, _ = solve_mode(P, omega_guess=seed, localize=False)
        out["cases"].append({"N": N, "root_default": [w.real, w.imag], "calls_default": c_def,
                             "seconds_default": t_def, "root_seeded": [w2.real, w2.imag], "calls_seeded": c_seed,
                             "seconds_seeded": t_seed, "newton_from_raw_seed": [w3.real, w3.imag],
                             "calls_newton_from_raw_seed": calls["n"]})
        print(json.dumps(out["cases"][-1]), flush=True)
    with open(os.path.join(HERE, "lka98_seed.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
