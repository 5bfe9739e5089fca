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
        assert np.allclose(recs[k], rec1, rtol=1e-12, atol=1e-15)
