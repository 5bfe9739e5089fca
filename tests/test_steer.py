"""Surrogate-steered sweeps (diskgpu.steer): the network proposes sweep points near a
level set of gamma, the hydro runs them and judges the network's error, and the hydro
takes over (the network is refined) when that error exceeds the bound.

CPU tests use stand-ins for the network and the hydro (a smooth analytic gamma over the
sweep parameters); the GPU test runs the shipped surrogate against the batched hydro."""
import numpy as np
import pytest

from diskgpu import steer as T


def _truth(X):
    Q, mr, s, g = X.T if X.ndim == 2 else X
    return 1.2 * mr - 0.6 * (Q - 1.0) - 1.5 * (s - 0.05) + 0.2 * (g - 1.5)


def _hydro(points):
    return _truth(T.features(points))


def test_steered_sweep_finds_more_contour_points_than_uniform():
    rng = np.random.default_rng(0)
    pred = lambda X: _truth(X) + 0.01 * rng.standard_normal(len(X))
    st = T.steer(pred, _hydro, target=0.3, tol=0.03, budget=48, batch=12, pool=2048)
    un = T.uniform(_hydro, target=0.3, tol=0.03, budget=48)
    assert len(st["points"]) == 48 and st["rounds"] == 4
    assert st["hits"] >= 40 and st["hits"] > 3 * un["hits"]
    assert not st["fallback_rounds"]
    # the hydro's values are the ones kept
    np.testing.assert_allclose(st["gamma_hydro"], _truth(T.features(st["points"])))


def test_biased_network_falls_back_and_is_refined():
    state = {"bias": 0.2, "refined": 0}

    def pred(X):
        return _truth(X) + state["bias"]

    def refine(X, y):
        state["refined"] += 1
        state["bias"] = 0.0  # the stand-in learns the hydro's values exactly

    st = T.steer(pred, _hydro, target=0.3, tol=0.03, budget=36, batch=12, pool=2048, refine=refine, bound=0.05)
    assert st["fallback_rounds"] == [0] and state["refined"] == 1
    assert np.all(st["abs_err"][:12] > 0.15) and np.all(st["abs_err"][12:] < 1e-12)
    assert st["hits"] >= 20


def test_proposals_are_spread_and_unique():
    X = T.features(__import__("diskgpu.sweep", fromlist=["draw"]).draw(512, seed=1))
    taken = np.zeros(len(X), dtype=bool)
    idx = T.propose(_truth(X), X, taken, 0.3, 16, 0.1)
    assert len(set(idx)) == len(idx) == 16
    Z = T._standardise(X[idx])
    d = np.linalg.norm(Z[:, None] - Z[None], axis=2) + np.eye(len(idx)) * 9
    assert d.min() >= 0.1


@pytest.mark.gpu
def test_steered_hydro_sweep_beats_uniform_draw():
    """The shipped surrogate steers 48 hydro runs (256^2, mixed precision, t = 16: the grid
    and time of its training set) at the
    contour gamma = 0.5 +- 0.05; the same budget drawn uniformly from the sweep law lands
    fewer runs on it.  The hydro judges every proposal (the network's error is recorded)."""
    from diskgpu.surrogate import TRAINED, Surrogate
    sur = Surrogate.load(TRAINED)
    pred = lambda X: sur.predict(X)[:, 0]
    st = T.steer(pred, T.hydro_gamma, target=0.5, tol=0.05, budget=48, batch=16, pool=4096,
                 refine=T.surrogate_refiner(sur))
    un = T.uniform(T.hydro_gamma, target=0.5, tol=0.05, budget=48)
    assert len(st["points"]) == 48 and np.all(np.isfinite(st["abs_err"]))
    assert st["hits"] >= 1.5 * max(un["hits"], 1), (st["hits"], un["hits"])
