"""Disks of the batched-sweep law against the FP64 oracle: general Gamma, the S0 and K that
dg_params_physical maps a sweep point to, a seeded m = 2 phase, and every grid size of the
sweep (128^2 .. 512^2) on the mixed path.

The oracle's general-Gamma branch (hydro.hpp:45-46 with Gamma != 2) is pinned to the
reference build bit for bit by the golden fixtures ref_40x48_g1.5 and ref_32x40_g1.75
(tests/test_oracle.py); these tests put the GPU paths beside it.

Tolerances, as in tests/test_mixed.py: the plain FP64 path <= 1e-10 relative after 100
steps; the mixed path's perturbation fields within 2e-3 of the perturbation's own size
after the given steps in lockstep (the oracle's dt drives both; the device's own dt must
agree to 1e-5); gamma and Omega_p within 0.5 % of the FP64 path's."""
import numpy as np
import pytest

import diskgpu as D
import oracle as O
from diskgpu.analysis import fit_growth
from helpers import rel_err

pytestmark = pytest.mark.gpu

# sweep points (Q_min, M_d/M_*, softening/r, Gamma): the first maps without the K cap, the
# second is capped (its achieved Q_min is below the requested one)
POINTS = {"g1.5": (1.1, 0.3, 0.15, 1.5), "g1.75": (1.6, 0.8, 0.07, 1.75)}


def _physics(name):
    p, _ = D.params_physical(*POINTS[name])
    return p


def _oracle(p, N, amp, phase0, nthreads=8):
    return O.Disk(Nu=N, Nphi=N, eps=p.eps, amp=amp, gamma_gas=p.gamma_gas, Kpoly=p.Kpoly, S0=p.S0,
                  phase0=phase0, nthreads=nthreads)


def test_params_physical_matches_golden_physics():
    """The sweep points above map to the physics the general-Gamma golden fixtures were
    made with (so those fixtures pin exactly these disks)."""
    from helpers import golden_cases, golden_physics
    cases = golden_cases()
    for name, fixture in (("g1.5", "40x48_g1.5"), ("g1.75", "32x40_g1.75")):
        p = _physics(name)
        gam, K, S0 = golden_physics(cases[fixture])
        assert (p.gamma_gas, p.Kpoly, p.S0) == (gam, K, S0)
        assert p.eps == pytest.approx(float(cases[fixture]["eps"]), rel=1e-12)


@pytest.mark.parametrize("name", sorted(POINTS))
def test_fp64_sweep_point_vs_oracle_100_steps(name):
    """Plain FP64 path, 128^2, seeded phase, 100 steps: <= 1e-10 relative in all fields,
    dt to 1e-12 every step."""
    p = _physics(name)
    N, phase0 = 128, 0.7
    ref = _oracle(p, N, 1e-3, phase0)
    with D.Disk(N, N, precision="fp64", params=p, amp=1e-3, phase0=phase0) as d:
        d.init_standard()
        for _ in range(100):
            dt_ref = ref.step()
            dt = d.timestep(0.3)
            assert abs(dt - dt_ref) <= 1e-12 * dt_ref
            d.step(dt)
        S, vR, vp = d.get_state()
    Sr, vRr, vpr = ref.hyd.state()
    assert rel_err(S, Sr) < 1e-10
    assert rel_err(vp, vpr) < 1e-10
    assert np.max(np.abs(vR - vRr)) < 1e-10 * np.max(np.abs(vpr))


@pytest.mark.parametrize("N,name,steps", [(128, "g1.5", 150), (256, "g1.75", 100), (384, "g1.5", 60),
                                          (512, "g1.75", 60), (384, "std", 60), (512, "std", 60)])
def test_mixed_sweep_disk_vs_oracle(N, name, steps):
    """Mixed path on every sweep grid size, general Gamma (the expm1/log1p pressure and the
    pow sound speed of the mixed kernels) and the standard disk, seeded phase: perturbation
    fields within 2e-3 of the perturbation's size after `steps` lockstep steps."""
    p = D.default_params(eps=0.005) if name == "std" else _physics(name)
    phase0, amp = 0.4, 1e-2
    ref = _oracle(p, N, amp, phase0)
    S0 = ref.hyd.get("Sig").mean(axis=1, keepdims=True)
    with D.Disk(N, N, precision="mixed", params=p, amp=amp, phase0=phase0) as d:
        d.init_standard()
        for _ in range(steps):
            dt_ref = ref.step()
            dt = d.timestep(0.3)
            assert abs(dt - dt_ref) <= 1e-5 * dt_ref, (dt, dt_ref)
            d.step(dt_ref)
        S, vR, vp = d.get_state()
    Sr, vRr, vpr = ref.hyd.state()
    assert np.max(np.abs(S - Sr)) <= 2e-3 * np.max(np.abs(Sr - S0))
    assert np.max(np.abs(vR - vRr)) <= 2e-3 * np.max(np.abs(vRr))
    vp0 = vpr.mean(axis=1, keepdims=True)
    assert np.max(np.abs(vp - vpr)) <= 2e-3 * np.max(np.abs(vpr - vp0)) + 1e-9


@pytest.mark.parametrize("N,name", [(384, "std"), (512, "std"), (256, "g1.75")])
def test_growth_rate_and_pattern_speed_sweep_grids(N, name):
    """gamma and Omega_p of the m = 2 mode, mixed against the FP64 path on the same disk,
    seeded phase: within 0.5 %.  The standard disk (eps = 0.01) at the sweep's two largest
    grids, and the heavy Gamma = 1.75 sweep point (gamma ~ 0.8) at 256^2."""
    p = D.default_params(eps=0.01) if name == "std" else _physics(name)
    out = {}
    for prec in ("fp64", "mixed"):
        with D.Disk(N, N, params=p, amp=1e-3, phase0=1.1, precision=prec) as d:
            d.init_standard()
            rec, t, n = d.advance(6.0)
        out[prec] = fit_growth(rec[:, 0], rec[:, 2], rec[:, 3], tmin=2.0, tmax=6.0)
    g64, w64, _ = out["fp64"]
    gmx, wmx, _ = out["mixed"]
    assert g64 > 0.2
    assert abs(gmx - g64) <= 5e-3 * abs(g64), (gmx, g64)
    assert abs(wmx - w64) <= 5e-3 * abs(w64), (wmx, w64)
