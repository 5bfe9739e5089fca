"""Surrogate MLP kernels against the FP64 CPU oracle (oracle/mlp_ref.py)."""
import numpy as np
import pytest

import mlp_ref as R
from diskgpu.surrogate import MLP, Surrogate

pytestmark = pytest.mark.gpu
SHAPE = (4, 256, 3, 3)


def _data(n, seed=0):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(n, 4)).astype(np.float32)
    t = np.stack([np.sin(x[:, 0]) + 0.5 * x[:, 1] * x[:, 2], np.cos(x[:, 3]) * x[:, 0], x[:, 1] ** 2 - 0.3],
                 axis=1).astype(np.float32)
    return x, t


def test_forward_matches_fp64_oracle():
    net = MLP(*SHAPE, seed=3)
    x, _ = _data(500)
    y = net.forward(x)
    ref = R.forward(net.params(), x, *SHAPE)
    assert np.max(np.abs(y - ref)) <= 2e-4 * np.max(np.abs(ref)) + 1e-6


def test_gradient_matches_fp64_oracle():
    """Every parameter's gradient from the backward kernels vs the FP64 oracle."""
    net = MLP(*SHAPE, seed=5)
    x, t = _data(333, seed=1)
    loss, g = net.loss_grad(x, t)
    lref, gref = R.loss_grad(net.params(), x, t, *SHAPE)
    assert loss == pytest.approx(lref, rel=1e-4)
    # per layer, relative to the layer's gradient scale
    off = 0
    fin = 4
    for l in range(4):
        fo = 3 if l == 3 else 256
        for cnt in (fo * fin, fo):
            a, b = g[off: off + cnt], gref[off: off + cnt]
            assert np.max(np.abs(a - b)) <= 2e-3 * np.max(np.abs(b)) + 1e-9, (l, cnt)
            off += cnt
        fin = fo


def test_gradient_against_finite_differences():
    net = MLP(4, 32, 2, 3, seed=7)
    x, t = _data(64, seed=2)
    _, g = net.loss_grad(x, t)
    p0 = net.params().astype(np.float64)
    rng = np.random.default_rng(0)
    for k in rng.choice(len(p0), 12, replace=False):
        h = 1e-3
        lp = R.loss_grad(np.where(np.arange(len(p0)) == k, p0 + h, p0), x, t, 4, 32, 2, 3, round_bf16=False)[0]
        lm = R.loss_grad(np.where(np.arange(len(p0)) == k, p0 - h, p0), x, t, 4, 32, 2, 3, round_bf16=False)[0]
        fd = (lp - lm) / (2 * h)
        assert g[k] == pytest.approx(fd, rel=0.05, abs=2e-4)


def test_training_fits_a_smooth_map():
    x, t = _data(2048, seed=4)
    s = Surrogate(seed=2)
    hist = s.fit(x, t, epochs=60, batch=256, lr=2e-3)
    assert hist[-1] < 0.1 * hist[0]
    xv, tv = _data(512, seed=9)
    err = np.sqrt(np.mean((s.predict(xv) - tv) ** 2, axis=0)) / t.std(axis=0)
    assert np.all(err < 0.2)


def test_shipped_surrogate_on_gpu_matches_oracle():
    """The shipped network, loaded onto the GPU, predicts what the FP64 oracle predicts for
    its parameters (held-out sweep points and the LKA98 standard disk)."""
    import os

    from diskgpu.surrogate import TRAINED, lka98_features, read_surrogate
    d = read_surrogate(TRAINED)
    grid = int(d["report"].get("grid", 128))
    with np.load(os.path.join(os.path.dirname(TRAINED), f"sweep_{grid}_dataset.npz")) as z:
        X = np.concatenate([z["data"][-51:, :4], lka98_features()])
    sur = Surrogate.load(TRAINED)
    got = sur.predict(X)
    ref = np.asarray(R.forward(d["params"].astype(np.float64), (X - d["xm"]) / d["xs"], *d["shape"])) * d["ys"] + d["ym"]
    assert np.max(np.abs(got - ref) / d["ys"]) <= 1e-3
    sur.net.close()
