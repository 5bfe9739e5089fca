"""Plain-method (FP64) GPU path against the reference (golden fixtures from the
reference build) and against the oracle at larger sizes.  Tolerance: <= 1e-10 relative
in Sigma, vR, vphi after 100 steps (the plain path's accuracy requirement); observed
errors are round-off (~1e-14)."""
import os
import subprocess

import numpy as np
import pytest

import diskgpu as D
import oracle as O
from helpers import GOLDEN, ROOT, golden_cases, golden_physics, rel_err

pytestmark = pytest.mark.gpu
CASES = golden_cases()
TOL = 1e-10


def _disk(g, **kw):
    gam, K, S0 = golden_physics(g)
    return D.Disk(int(g["Nu"]), int(g["Nphi"]), eps=float(g["eps"]), selfgrav=int(g["selfgrav"]),
                  amp=float(g["amp"]), gamma_gas=gam, Kpoly=K, S0=S0, **kw)


@pytest.mark.parametrize("name", sorted(CASES))
def test_golden_initial_state_and_gravity(name):
    g = CASES[name]
    with _disk(g) as d:
        d.init_standard()
        S, vR, vp = d.get_state()
        assert rel_err(S, g["Sig0"]) < 1e-14
        assert np.all(vR == 0)
        assert rel_err(vp, g["vp0"]) < 1e-13
        Phi = d.potential(g["Sig0"])
        assert rel_err(Phi, g["Phi0"]) < 1e-12
        gR, gp = d.forces(g["Phi0"])
        assert rel_err(gR, g["gR0"]) < 1e-12
        assert rel_err(gp, g["gp0"]) < 1e-12 * max(1.0, np.abs(g["gR0"]).max() / max(np.abs(g["gp0"]).max(), 1e-300))


@pytest.mark.parametrize("name", sorted(CASES))
def test_golden_steps(name):
    g = CASES[name]
    with _disk(g) as d:
        d.set_state(g["Sig0"], g["vR0"], g["vp0"])
        for k, dt_ref in enumerate(g["dt"]):
            dt = d.timestep(0.3)
            assert abs(dt - dt_ref) <= 1e-12 * dt_ref, (k, dt, dt_ref)
            d.step(dt)
        S, vR, vp = d.get_state()
    assert rel_err(S, g["SigN"]) < TOL
    assert rel_err(vp, g["vpN"]) < TOL
    assert rel_err(vR, g["vRN"]) < TOL * max(1.0, np.abs(g["vpN"]).max() / np.abs(g["vRN"]).max()) or \
        np.max(np.abs(vR - g["vRN"])) < TOL * np.abs(g["vpN"]).max()


def test_known_answer_fft_vs_direct_on_gpu():
    """test_kalnajs.cpp on the GPU solver: potential vs the direct O(N^4) sum < 1e-10."""
    k = D.KalnajsSolver(32, 32, 0.25, 1.0, 0.02)
    phi = (np.arange(32) + 0.5) * k.dphi
    S0 = 0.372 * np.exp(-(k.R - 0.45) ** 2 / 0.05)
    Sig = S0[:, None] * (1.0 + 0.3 * np.cos(2.0 * phi))[None, :]
    Pf = k.potential(Sig)
    Pd = O.Kalnajs(32, 32, eps=0.02).potential_direct(Sig)
    assert np.max(np.abs(Pf - Pd)) / np.max(np.abs(Pd)) < 1e-10


@pytest.mark.parametrize("N,steps", [(256, 100), (128, 100), (384, 20), (1024, 4)])
def test_fp64_vs_oracle_after_steps(N, steps):
    """The reference's CPU-runnable case (256^2, eps 0.005) for 100 steps, plus other sizes."""
    kw = dict(Nu=N, Nphi=N, eps=0.005, amp=1e-3)
    ref = O.Disk(nthreads=8, **kw)
    with D.Disk(N, N, eps=0.005, amp=1e-3) as d:
        d.init_standard()
        S, vR, vp = d.get_state()
        S0, vR0, vp0 = ref.hyd.state()
        assert rel_err(vp, vp0) < 1e-13
        for _ in range(steps):
            dt_ref = ref.step()
            dt = d.timestep(0.3)
            assert abs(dt - dt_ref) <= 1e-11 * dt_ref
            d.step(dt)
        S, vR, vp = d.get_state()
    Sr, vRr, vpr = ref.hyd.state()
    assert rel_err(S, Sr) < TOL
    assert rel_err(vp, vpr) < TOL
    assert np.max(np.abs(vR - vRr)) < TOL * np.max(np.abs(vpr))


@pytest.mark.parametrize("Nu,Nphi,steps", [(128, 384, 100), (384, 128, 60), (240, 180, 100)])
def test_fp64_nonsquare_vs_oracle_after_steps(Nu, Nphi, steps):
    """Non-square grids on the FP64 path, one of them with radix-3 and radix-5 transform
    lengths (240 x 180: padded u length 480, phi length 180): <= 1e-10 relative after the
    given steps, dt to 1e-11 every step."""
    ref = O.Disk(nthreads=8, Nu=Nu, Nphi=Nphi, eps=0.005, amp=1e-3)
    with D.Disk(Nu, Nphi, eps=0.005, amp=1e-3) as d:
        d.init_standard()
        for _ in range(steps):
            dt_ref = ref.step()
            dt = d.timestep(0.3)
            assert abs(dt - dt_ref) <= 1e-11 * dt_ref
            d.step(dt)
        S, vR, vp = d.get_state()
    Sr, vRr, vpr = ref.hyd.state()
    assert rel_err(S, Sr) < TOL
    assert rel_err(vp, vpr) < TOL
    assert np.max(np.abs(vR - vRr)) < TOL * np.max(np.abs(vpr))


def test_step_with_caller_forces_and_without_gravity():
    """DiskHydro::step(dt, gR, gp) with explicit forces, and with none."""
    rng = np.random.default_rng(3)
    ref = O.Disk(Nu=48, Nphi=40, eps=0.01, amp=0.05)
    S0, vR0, vp0 = ref.hyd.state()
    gR = rng.normal(size=S0.shape) * 0.1
    gp = rng.normal(size=S0.shape) * 0.1
    h = D.DiskHydro(48, 40)
    h.Sig, h.vR, h.vp = S0.copy(), vR0.copy(), vp0.copy()
    dt = h.timestep(0.3)
    assert dt == pytest.approx(ref.hyd.timestep(0.3), rel=1e-13)
    h.step(dt, gR, gp)
    ref.hyd.step(dt, gR, gp)
    S, vR, vp = ref.hyd.state()
    assert rel_err(h.Sig, S) < 1e-13 and rel_err(h.vp, vp) < 1e-13
    h.step(dt)
    ref.hyd.step(dt)
    S, vR, vp = ref.hyd.state()
    assert rel_err(h.Sig, S) < 1e-13 and rel_err(h.vp, vp) < 1e-13


def test_advance_loop_matches_reference_modes_table():
    """The device-resident diskmain.cpp loop: same records and step count as the reference."""
    gdir = os.path.join(GOLDEN, "diskdisk_ref_64_t1")
    argv = open(os.path.join(gdir, "argv.txt")).read().split()
    Nu, Nphi, eps, tlim = int(argv[0]), int(argv[1]), float(argv[2]), float(argv[3])
    with D.Disk(Nu, Nphi, eps=eps, amp=float(argv[5])) as d:
        d.init_standard()
        recs, t, steps = d.advance(tlim)
    want = [l.split() for l in open(os.path.join(gdir, "diskfft_modes.dat")).read().splitlines()[1:]]
    assert len(recs) == len(want)
    for r, w in zip(recs, want):
        assert "%.5f" % r[0] == w[0]
        for a, b in zip(r[1:], w[1:]):
            assert abs(a - float(b)) <= 2e-6 * max(abs(float(b)), 1e-12) + 1e-12
    last = open(os.path.join(gdir, "stdout.txt")).read().splitlines()[-1]
    assert last.endswith(f"steps={steps}")
    assert t == pytest.approx(tlim, abs=1e-12)


def test_advance_matches_stepwise_loop():
    """dg_advance (graphs, device dt) == the host loop of timestep + step."""
    with D.Disk(64, 64, eps=0.01) as a, D.Disk(64, 64, eps=0.01) as b:
        a.init_standard()
        b.init_standard()
        _, t, n = a.advance(0.2)
        tb = 0.0
        nb = 0
        while tb < 0.2:
            dt = b.timestep(0.3)
            if tb + dt > 0.2:
                dt = 0.2 - tb
            b.step(dt)
            tb += dt
            nb += 1
        assert n == nb
        for x, y in zip(a.get_state(), b.get_state()):
            assert rel_err(x, y) < 1e-13


def test_nonfinite_state_reported_not_faulted():
    """A NaN in the state surfaces as DG_ERR_NONFINITE from the next step (host-side fault injection)."""
    with D.Disk(32, 32) as d:
        d.init_standard()
        S, vR, vp = d.get_state()
        S[5, 7] = np.nan
        d.set_state(S, vR, vp)
        with pytest.raises(D.DiskGPUError) as e:
            d.step(1e-4)
        assert e.value.code == -3
        # the handle stays usable
        d.init_standard()
        d.step(d.timestep(0.3))


def test_cli_dropin_matches_reference_output(tmp_path):
    gdir = os.path.join(GOLDEN, "diskdisk_ref_64_t1")
    argv = open(os.path.join(gdir, "argv.txt")).read().split()
    exe = os.path.join(ROOT, "heavy-disks_b200", "bin", "diskdisk")
    res = subprocess.run([exe] + argv, cwd=tmp_path, capture_output=True, text=True, check=True)
    got = open(tmp_path / "diskfft_modes.dat").read().splitlines()
    want = open(os.path.join(gdir, "diskfft_modes.dat")).read().splitlines()
    assert got[0] == want[0] and len(got) == len(want)
    for g, w in zip(got[1:], want[1:]):
        gv, wv = g.split(), w.split()
        assert gv[0] == wv[0]
        for a, b in zip(gv[1:], wv[1:]):
            assert abs(float(a) - float(b)) <= 2e-6 * max(abs(float(b)), 1e-12) + 1e-12
    out = res.stdout.splitlines()
    ref_out = open(os.path.join(gdir, "stdout.txt")).read().splitlines()
    assert len(out) == len(ref_out)
    assert out[-1].split()[-1] == ref_out[-1].split()[-1]  # steps=N
