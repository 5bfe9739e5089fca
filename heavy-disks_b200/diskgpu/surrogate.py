"""Learned surrogate of the sweep: (Q_min, M_d/M_*, softening/r, Gamma) ->
(gamma, Omega_p, saturated |C2|/|C0|), an MLP trained and evaluated by the library's own
CUDA kernels (dg_mlp in include/diskgpu.h).  Inputs and targets are standardised with
statistics of the training set; the network sees O(1) numbers.
"""
from __future__ import annotations

import ctypes as C
import json
import os

import numpy as np

from . import DG_OK, DiskGPUError, lib

FEATURES = ("Qmin", "mass_ratio", "soft_over_r", "gamma")
TARGETS = ("gamma", "omega_p", "sat_ratio")


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class MLP:
    """Thin owner of a dg_mlp handle."""

    def __init__(self, n_in=4, width=256, depth=3, n_out=3, seed=1, device=-1):
        h = C.c_void_p()
        rc = lib().dg_mlp_create(n_in, width, depth, n_out, seed, device, C.byref(h))
        if rc != DG_OK:
            raise DiskGPUError(rc, "dg_mlp_create")
        self.h, self.shape = h, (n_in, width, depth, n_out)
        self.n_params = int(lib().dg_mlp_num_params(h))

    def _ck(self, rc):
        if rc != DG_OK:
            raise DiskGPUError(rc, lib().dg_mlp_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            lib().dg_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self):
        p = np.empty(self.n_params, dtype=np.float32)
        self._ck(lib().dg_mlp_get_params(self.h, _fp(p)))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        self._ck(lib().dg_mlp_set_params(self.h, _fp(p)))

    def forward(self, x):
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.empty((x.shape[0], self.shape[3]), dtype=np.float32)
        self._ck(lib().dg_mlp_forward(self.h, x.shape[0], _fp(x), _fp(y)))
        return y

    def loss_grad(self, x, t):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        g = np.empty(self.n_params, dtype=np.float32)
        self._ck(lib().dg_mlp_loss_grad(self.h, x.shape[0], _fp(x), _fp(t), _fp(loss), _fp(g)))
        return float(loss[0]), g

    def train_step(self, x, t, lr):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        self._ck(lib().dg_mlp_train_step(self.h, x.shape[0], _fp(x), _fp(t), lr, _fp(loss)))
        return float(loss[0])


class Surrogate:
    """Standardisation + MLP.  fit() trains on (X, Y) arrays in physical units."""

    def __init__(self, width=256, depth=3, seed=1, device=-1):
        self.net = MLP(len(FEATURES), width, depth, len(TARGETS), seed, device)
        self.xm = self.xs = self.ym = self.ys = None

    def _norm(self, X, Y=None):
        Xn = (np.asarray(X, dtype=np.float64) - self.xm) / self.xs
        if Y is None:
            return Xn.astype(np.float32)
        return Xn.astype(np.float32), ((np.asarray(Y, dtype=np.float64) - self.ym) / self.ys).astype(np.float32)

    def fit(self, X, Y, epochs=300, batch=256, lr=2e-3, seed=0):
        X = np.asarray(X, dtype=np.float64)
        Y = np.asarray(Y, dtype=np.float64)
        self.xm, self.xs = X.mean(axis=0), X.std(axis=0) + 1e-12
        self.ym, self.ys = Y.mean(axis=0), Y.std(axis=0) + 1e-12
        Xn, Yn = self._norm(X, Y)
        rng = np.random.default_rng(seed)
        hist = []
        n = len(Xn)
        for ep in range(epochs):
            perm = rng.permutation(n)
            tot = 0.0
            for s in range(0, n, batch):
                idx = perm[s: s + batch]
                tot += self.net.train_step(Xn[idx], Yn[idx], lr) * len(idx)
            hist.append(tot / n)
        return hist

    def predict(self, X):
        y = self.net.forward(self._norm(X)).astype(np.float64)
        return y * self.ys + self.ym

    def save(self, path, report=None):
        """Write the network and its standardisation: .npz (compressed, float32 parameters)
        or .json."""
        if str(path).endswith(".npz"):
            np.savez_compressed(path, shape=np.array(self.net.shape, dtype=np.int64), params=self.net.params(),
                                xm=self.xm, xs=self.xs, ym=self.ym, ys=self.ys,
                                report=np.array(json.dumps(report or {})))
            return
        with open(path, "w") as f:
            json.dump({"shape": list(self.net.shape), "params": self.net.params().tolist(), "xm": self.xm.tolist(),
                       "xs": self.xs.tolist(), "ym": self.ym.tolist(), "ys": self.ys.tolist()}, f)

    @classmethod
    def load(cls, path, device=-1):
        d = read_surrogate(path)
        s = cls(width=int(d["shape"][1]), depth=int(d["shape"][2]), device=device)
        s.net.set_params(np.asarray(d["params"], dtype=np.float32))
        s.xm, s.xs, s.ym, s.ys = d["xm"], d["xs"], d["ym"], d["ys"]
        return s


def read_surrogate(path):
    """The stored surrogate as plain arrays: shape, params (float32), xm, xs, ym, ys, report."""
    if str(path).endswith(".npz"):
        with np.load(path) as z:
            return {"shape": [int(v) for v in z["shape"]], "params": z["params"].astype(np.float32),
                    "xm": z["xm"], "xs": z["xs"], "ym": z["ym"], "ys": z["ys"],
                    "report": json.loads(str(z["report"])) if "report" in z else {}}
    with open(path) as f:
        d = json.load(f)
    return {"shape": d["shape"], "params": np.array(d["params"], dtype=np.float32), "xm": np.array(d["xm"]),
            "xs": np.array(d["xs"]), "ym": np.array(d["ym"]), "ys": np.array(d["ys"]), "report": {}}


# The surrogate trained on the sweep law with the package's own batched hydro (report inside
# the file), shipped with the package.
TRAINED = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "surrogate.npz")


def lka98_features(mstar=0.6, mdisk=0.4, Qmin=1.27, soft_over_r=0.05, gamma=2.0):
    """Surrogate inputs (Q_min, M_d/M_*, softening/r, Gamma) of an LKA98 disk.  The standard
    disk (lka98/model.py: m* = 0.6, m_D = 0.4; Q_min = 1.27 by lka98/EQUATIONS.md; Gamma = 2)
    is softened by ~0.02 r at its density peak, below the trained range, so the lowest
    trained value 0.05 stands in for it."""
    return np.array([[Qmin, mdisk / mstar, soft_over_r, gamma]])


def lka98_omega_guess(pred_gamma, pred_omega_p, m=2):
    """Seed for lka98.eigensolve: omega = m Omega_p - i gamma (the convention of
    lka98/eigensolve.py:153, where 3.15057 - 0.72278i means Omega_p = 1.5753, gamma = 0.7228).

    The hydro's disks differ from the linear model (softening, finite amplitude), so the seed
    is the centre of a coarse contour rather than a Newton start: lka98's
    contour_root(problem, seed, 0.35, 0.35, n=16) followed by solve_mode(problem, root,
    localize=False) finds the growing mode with 4 x 16 + a few dlogdet calls instead of the
    default 4 x 160 + a few."""
    return complex(m * pred_omega_p, -pred_gamma)
