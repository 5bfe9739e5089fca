"""The CPU oracle against the reference's own outputs (no GPU).

The golden fixtures were produced by the reference sources compiled unmodified
(oracle/_ref, tests/golden/make_golden.py); the oracle restatement must reproduce
them bit for bit, and its FFT must agree with numpy's pocketfft."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from helpers import GOLDEN, golden_cases, golden_physics, rel_err

CASES = golden_cases()


@pytest.fixture(scope="module", autouse=True)
def _built():
    O.build()


@pytest.mark.parametrize("name", sorted(CASES))
def test_restatement_matches_reference_bitwise(name):
    g = CASES[name]
    Nu, Nphi = int(g["Nu"]), int(g["Nphi"])
    gam, K, S0 = golden_physics(g)
    d = O.Disk(Nu=Nu, Nphi=Nphi, eps=float(g["eps"]), selfgrav=int(g["selfgrav"]), amp=float(g["amp"]),
               gamma_gas=gam, Kpoly=K, S0=S0)
    S, vR, vp = d.hyd.state()
    assert np.array_equal(S, g["Sig0"]) and np.array_equal(vR, g["vR0"]) and np.array_equal(vp, g["vp0"])
    Phi = d.grav.potential(S)
    gR, gp = d.grav.forces(Phi)
    assert np.array_equal(Phi, g["Phi0"])
    assert np.array_equal(gR, g["gR0"]) and np.array_equal(gp, g["gp0"])
    dts = [d.step() for _ in range(int(g["nsteps"]))]
    assert np.array_equal(np.array(dts), g["dt"])
    S, vR, vp = d.hyd.state()
    assert np.array_equal(S, g["SigN"]) and np.array_equal(vR, g["vRN"]) and np.array_equal(vp, g["vpN"])
    c2, ph2 = d.cm(2)
    assert c2 == float(g["c2"]) and ph2 == float(g["ph2"])


def test_known_answer_fft_vs_direct():
    """test_kalnajs.cpp:9-43: FFT potential vs direct O(N^4) sum, rel < 1e-10."""
    k = O.Kalnajs(32, 32, eps=0.02)
    R = np.exp(np.log(0.25) + (np.arange(32) + 0.5) * np.log(4.0) / 32)
    phi = (np.arange(32) + 0.5) * 2 * np.pi / 32
    S0 = 0.372 * np.exp(-(R - 0.45) ** 2 / 0.05)
    Sig = S0[:, None] * (1.0 + 0.3 * np.cos(2.0 * phi))[None, :]
    Pf, Pd = k.potential(Sig), k.potential_direct(Sig)
    rel = np.max(np.abs(Pf - Pd)) / np.max(np.abs(Pd))
    assert rel < 1e-10
    # the reference's own printout of the same test
    txt = open(os.path.join(GOLDEN, "test_kalnajs_ref.txt")).read()
    assert "exit=0" in txt
    assert f"max|Phi| = {np.max(np.abs(Pd)):.6e}" in txt
    assert f"fft={Pf[16, 0]:.6e} dir={Pd[16, 0]:.6e}" in txt


@pytest.mark.parametrize("shape", [(8, 12), (48, 40), (24, 27), (64, 30), (16, 50)])
def test_fft_shim_matches_numpy(shape):
    """The project FFT backing the FFTW shim vs numpy.fft (pocketfft)."""
    rng = np.random.default_rng(1)
    Nu, Nphi = shape
    k = O.Kalnajs(Nu, Nphi, eps=0.01)
    # khat is the r2c of the sampled kernel; recompute it with numpy
    M = 2 * Nu
    du = np.log(4.0) / Nu
    dphi = 2 * np.pi / Nphi
    p = np.arange(M)
    ioff = np.where(p <= M // 2, p, p - M)
    Kr = 1.0 / np.sqrt(2 * np.cosh(ioff[:, None] * du) - 2 * np.cos(np.arange(Nphi)[None, :] * dphi) + 0.01)
    ref = np.fft.rfft2(Kr)
    got = k.khat()
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < 1e-13
    # and the potential of a random field against a numpy convolution
    Sig = rng.random((Nu, Nphi))
    R = np.exp(np.log(0.25) + (np.arange(Nu) + 0.5) * du)
    buf = np.zeros((M, Nphi))
    buf[:Nu] = (R ** 1.5)[:, None] * Sig
    V = np.fft.irfft2(np.fft.rfft2(buf) * ref, s=(M, Nphi))[:Nu]
    Phi_np = -du * dphi * V / np.sqrt(R)[:, None]
    assert rel_err(k.potential(Sig), Phi_np) < 1e-12


def test_oracle_run_matches_reference_modes(tmp_path):
    """orc_run (diskmain.cpp loop) reproduces the reference diskdisk mode table."""
    gdir = os.path.join(GOLDEN, "diskdisk_ref_64_t1")
    argv = open(os.path.join(gdir, "argv.txt")).read().split()
    Nu, Nphi, eps, tlim, sg, amp = int(argv[0]), int(argv[1]), float(argv[2]), float(argv[3]), int(argv[4]), float(argv[5])
    d = O.Disk(Nu=Nu, Nphi=Nphi, eps=eps, tlim=tlim, selfgrav=sg, amp=amp)
    recs = []
    t, tnext, step = 0.0, 0.0, 0
    while t < tlim:
        if t >= tnext - 1e-12:
            c0, _ = d.cm(0)
            c2, ph2 = d.cm(2)
            recs.append("%.5f %.6e %.6e %.6e" % (t, c0, c2, ph2))
            tnext += 0.25
        dt = d.hyd.timestep(0.3)
        if t + dt > tlim:
            dt = tlim - t
        gR, gp = d.gravity()
        d.hyd.step(dt, gR, gp)
        t += dt
        step += 1
    want = open(os.path.join(gdir, "diskfft_modes.dat")).read().splitlines()
    assert want[0] == "# t  |C0|  |C2|  arg(C2)"
    assert want[1:] == recs
    last = open(os.path.join(gdir, "stdout.txt")).read().splitlines()[-1]
    assert last.endswith(f"steps={step}")


@pytest.mark.skipif(not os.path.exists(os.path.join(O.REF_DIR, "refdump")),
                    reason="reference build (oracle/_ref) not present")
def test_restatement_matches_reference_build_live(tmp_path):
    """Against the live reference build at a size not in the fixtures."""
    out = tmp_path / "d.bin"
    subprocess.run([os.path.join(O.REF_DIR, "refdump"), "40", "36", "0.01", "1", "0.05", "7", str(out)], check=True)
    r = O.read_refdump(str(out))
    d = O.Disk(Nu=40, Nphi=36, eps=0.01, amp=0.05)
    for _ in range(7):
        d.step()
    S, vR, vp = d.hyd.state()
    assert np.array_equal(S, r["SigN"]) and np.array_equal(vp, r["vpN"])
