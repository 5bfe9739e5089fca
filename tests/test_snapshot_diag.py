"""Snapshot / restart (bit-exact continuation) and the per-step m = 0..8 diagnostics."""
import numpy as np
import pytest

import diskgpu as D

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_restart_continues_bit_for_bit(tmp_path, precision):
    path = str(tmp_path / "snap.bin")
    with D.Disk(128, 128, eps=0.01, amp=0.05, precision=precision) as a:
        a.init_standard()
        a.run_steps(10)
        a.save(path)
        a.run_steps(10)
        ta, na = a.time()
        Sa = a.get_state()
    with D.Disk(128, 128, eps=0.01, amp=0.05, precision=precision) as b:
        b.load(path)
        assert b.time()[1] == 10
        b.run_steps(10)
        tb, nb = b.time()
        Sb = b.get_state()
    assert (ta, na) == (tb, nb)
    for x, y in zip(Sa, Sb):
        assert np.array_equal(x, y)


def test_load_rejects_mismatched_handle(tmp_path):
    path = str(tmp_path / "snap.bin")
    with D.Disk(128, 128, eps=0.01) as a:
        a.init_standard()
        a.save(path)
    with D.Disk(128, 128, eps=0.02) as b:
        with pytest.raises(D.DiskGPUError):
            b.load(path)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_per_step_modes_match_dg_modes(precision):
    with D.Disk(128, 128, eps=0.01, amp=0.05, precision=precision) as d:
        d.init_standard()
        d.set_diagnostics(mmax=8, capacity=64)
        d.run_steps(20)
        t, Cm = d.diagnostics()
        assert len(t) == 20 and np.all(np.diff(t) > 0)
        ref = d.modes(8)
        assert np.allclose(Cm[-1], ref, rtol=1e-10, atol=1e-13)
        assert abs(Cm[-1, 0]) == pytest.approx(1.0, rel=1e-9)  # |C0| = mass / m_D
        assert abs(Cm[-1, 2]) > 10 * abs(Cm[-1, 3])             # the seeded m = 2 dominates
        d.set_diagnostics(capacity=0)
        d.run_steps(3)
        t2, _ = d.diagnostics()
        assert len(t2) == 0
