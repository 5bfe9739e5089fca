"""Batched sweeps: disks advanced together in one graph launch give exactly what they
give alone (the kernels are the same and the state updates are deterministic)."""
import numpy as np
import pytest

import diskgpu as D
from diskgpu import sweep as S

pytestmark = pytest.mark.gpu


def _params(pt, precision):
    p, _ = D.params_physical(pt.Qmin, pt.mass_ratio, pt.soft_over_r, pt.gamma)
    p.Nu = p.Nphi = pt.N
    p.amp = pt.amp
    p.phase0 = pt.phase0
    p.precision = D.MIXED if precision == "mixed" else D.FP64
    return p


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_batch_equals_individual_runs(precision):
    pts = S.draw(5, seed=11, grids=(128, 256))
    params = [_params(p, precision) for p in pts]
    tlim = 0.08
    with D.Batch(params) as b:
        b.init_standard()
        recs, t, steps = b.advance(tlim, steps_per_launch=8, dtout=0.02)
        states = [d.get_state() for d in b.disks]
    for k, p in enumerate(params):
        with D.Disk(p.Nu, p.Nphi, params=p, precision=precision) as d:
            d.init_standard()
            rec1, t1, n1 = d.advance(tlim, dtout=0.02)
            st1 = d.get_state()
        assert steps[k] == n1 and t[k] == t1
        for a, c in zip(states[k], st1):
            assert np.array_equal(a, c)
        assert recs[k].shape == rec1.shape
        assert np.allclose(recs[k], rec1, rtol=1e-10, atol=1e-13)


def test_grouped_batch_equals_ungrouped_and_lone(monkeypatch):
    """16 sweep disks over all four sweep grids plus two plain FP64 disks: the mixed disks
    form same-grid groups advanced by one launch per kernel (blockIdx.z = disk); the states
    are bit for bit the ones with grouping off (DISKGPU_BATCH_GROUPS=0, one graph branch
    per disk) and the ones of lone runs, the step counts and times equal; the mode records
    agree to 1e-10 (their FP64 sums are folded with atomics in a varying order; differences
    of ~2e-12 occur)."""
    pts = S.draw(16, seed=3, grids=(128, 256, 384, 512))
    params = [_params(p, "mixed") for p in pts] + [_params(p, "fp64") for p in pts[:2]]
    tlim = 0.03
    out = {}
    for grouped in ("1", "0"):
        monkeypatch.setenv("DISKGPU_BATCH_GROUPS", grouped)
        with D.Batch(params) as b:
            b.init_standard()
            recs, t, steps = b.advance(tlim, steps_per_launch=8, dtout=0.01)
            out[grouped] = ([d.get_state() for d in b.disks], recs, t, steps)
    (sa, ra, ta, na), (sb, rb, tb, nb) = out["1"], out["0"]
    assert np.array_equal(na, nb) and np.array_equal(ta, tb)
    for k in range(len(params)):
        for x, y in zip(sa[k], sb[k]):
            assert np.array_equal(x, y), k
        np.testing.assert_allclose(ra[k], rb[k], rtol=1e-10, atol=1e-13)
    for k in (0, 5, 16):
        p = params[k]
        with D.Disk(p.Nu, p.Nphi, params=p, precision="mixed" if p.precision == D.MIXED else "fp64") as d:
            d.init_standard()
            d.advance(tlim, dtout=0.01)
            for x, y in zip(sa[k], d.get_state()):
                assert np.array_equal(x, y), k


def test_grouped_1024_disks_equal_lone(monkeypatch):
    """Five 1024^2 sweep disks (two pairs that share a physics point and differ in seed
    phase and amplitude, so each pair is one step-rate class): grouped, the fused phi
    transform, u convolution and inverse phi transform run once per step for the whole
    group (blockIdx.y = disk; DISKGPU_BATCH_GROUPS=all, since 1024^2 disks step as branches
    of their own by default).  States bit for bit those with grouping off and those of a
    lone run; step counts and times equal; mode records to 1e-10."""
    pts = S.draw(5, seed=3, grids=(1024,))
    params = [_params(p, "mixed") for p in pts]
    for k, src, phase, amp in ((2, 0, 2.3, 3e-3), (3, 1, 0.2, 2e-3)):
        params[k] = _params(pts[src], "mixed")
        params[k].phase0, params[k].amp = phase, amp
    tlim = 0.01
    out = {}
    for grouped in ("all", "0"):
        monkeypatch.setenv("DISKGPU_BATCH_GROUPS", grouped)
        with D.Batch(params) as b:
            b.init_standard()
            recs, t, steps = b.advance(tlim, steps_per_launch=8, dtout=0.004)
            out[grouped] = ([d.get_state() for d in b.disks], recs, t, steps)
    (sa, ra, ta, na), (sb, rb, tb, nb) = out["all"], out["0"]
    assert np.array_equal(na, nb) and np.array_equal(ta, tb)
    assert min(na) > 40
    for k in range(len(params)):
        for x, y in zip(sa[k], sb[k]):
            assert np.array_equal(x, y), k
        np.testing.assert_allclose(ra[k], rb[k], rtol=1e-10, atol=1e-13)
    p = params[2]
    with D.Disk(p.Nu, p.Nphi, params=p, precision="mixed") as d:
        d.init_standard()
        d.advance(tlim, dtout=0.004)
        for x, y in zip(sa[2], d.get_state()):
            assert np.array_equal(x, y)


def test_direct_launches_equal_graph_replay(monkeypatch):
    """DISKGPU_BATCH_GRAPH=0 enqueues every launch's kernels directly (for profilers that
    see only kernels launched outside graphs): the same kernels in the same order, so the
    states equal the graph-replayed batch's bit for bit, with the same step counts."""
    pts = S.draw(6, seed=5, grids=(128, 256))
    params = [_params(p, "mixed") for p in pts]
    out = {}
    for mode in ("1", "0"):
        monkeypatch.setenv("DISKGPU_BATCH_GRAPH", mode)
        with D.Batch(params) as b:
            b.init_standard()
            recs, t, steps = b.advance(0.05, steps_per_launch=8, dtout=0.02)
            out[mode] = ([d.get_state() for d in b.disks], recs, t, steps)
    (sa, ra, ta, na), (sb, rb, tb, nb) = out["1"], out["0"]
    assert np.array_equal(na, nb) and np.array_equal(ta, tb)
    for k in range(len(params)):
        for x, y in zip(sa[k], sb[k]):
            assert np.array_equal(x, y), k
        np.testing.assert_allclose(ra[k], rb[k], rtol=1e-10, atol=1e-13)


def test_lanes_equal_unlimited_concurrency(monkeypatch):
    """DISKGPU_BATCH_LANES=2 lets at most two branches of a launch run at once (each branch
    follows the one two places before it): the same kernels per disk in the same order, so
    the states equal the unlimited batch's bit for bit."""
    pts = S.draw(7, seed=6, grids=(128, 256))
    params = [_params(p, "mixed") for p in pts]
    out = {}
    for lanes in ("0", "2"):
        monkeypatch.setenv("DISKGPU_BATCH_LANES", lanes)
        with D.Batch(params) as b:
            b.init_standard()
            recs, t, steps = b.advance(0.05, steps_per_launch=8, dtout=0.02)
            out[lanes] = ([d.get_state() for d in b.disks], recs, t, steps)
    (sa, ra, ta, na), (sb, rb, tb, nb) = out["0"], out["2"]
    assert np.array_equal(na, nb) and np.array_equal(ta, tb)
    for k in range(len(params)):
        for x, y in zip(sa[k], sb[k]):
            assert np.array_equal(x, y), k
        np.testing.assert_allclose(ra[k], rb[k], rtol=1e-10, atol=1e-13)
