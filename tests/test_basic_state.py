"""FP64 elliptic-integral basic state (host code of the library, no GPU) against scipy and
against the reference's FFT-based equilibrium, and the sweep-parameter map."""
import numpy as np
import pytest
from scipy.integrate import quad
from scipy.special import ellipk

import diskgpu as D
import oracle as O


def _g_scipy(R, eps, S0=0.372):
    """-dPhi/dR of the softened disk by scipy quadrature of the same closed form."""
    def phi(Rf):
        f = lambda Rp: S0 * np.exp(-(Rp - 0.45) ** 2 / 0.05) * Rp * 4 * ellipk(
            4 * Rf * Rp / ((Rf + Rp) ** 2 + eps * Rf * Rp)) / np.sqrt((Rf + Rp) ** 2 + eps * Rf * Rp)
        return -quad(f, 0.25, 1.0, points=[Rf], limit=400, epsabs=1e-14, epsrel=1e-13)[0]
    h = 1e-5
    return -(phi(R + h) - phi(R - h)) / (2 * h)


@pytest.mark.parametrize("R,eps", [(0.3, 0.005), (0.5, 0.005), (0.7, 0.02), (0.9, 0.0025)])
def test_disk_force_matches_scipy(R, eps):
    got = D.rotation_curve_elliptic(np.array([R, R * 1.01]), eps=eps)["gR"][0]
    assert got == pytest.approx(_g_scipy(R, eps), rel=2e-7)


def test_elliptic_vs_fft_equilibrium_stated_error():
    """The two basic states differ by the FFT solver's discretisation: the median error
    falls as N^-2 (6e-5 at 64^2, 2e-5 at 128^2) and the maximum, set by the one-sided
    force differences at the outer edge, as N^-1 (4.6e-3, 2.3e-3)."""
    med, mx = [], []
    for N in (64, 128):
        d = O.Disk(Nu=N, Nphi=N, eps=0.005, amp=0.0, nthreads=4)
        R = d.hyd.get("R")
        vf = d.hyd.get("vp")[:, 0]
        ve = np.sqrt(D.rotation_curve_elliptic(R, eps=0.005)["vphi2"])
        e = np.abs(ve - vf) / vf
        med.append(np.median(e))
        mx.append(e.max())
    assert mx[1] < 3e-3 and med[1] < 3e-5
    assert med[1] < 0.5 * med[0] and mx[1] < 0.6 * mx[0]


@pytest.mark.parametrize("args", [(1.0, 0.2, 0.1, 1.8), (1.5, 0.2, 0.1, 1.8), (1.0, 0.5, 0.1, 1.8),
                                  (1.0, 0.667, 0.0707, 2.0)])
def test_params_physical_hits_target(args):
    Qmin, ratio, soft, gam = args
    p, q = D.params_physical(*args)
    assert q == pytest.approx(Qmin, rel=1e-6)
    assert p.eps == pytest.approx(soft ** 2) and p.gamma_gas == gam
    m = quad(lambda R: 2 * np.pi * R * p.S0 * np.exp(-(R - 0.45) ** 2 / 0.05), 0.25, 1.0)[0]
    assert m == pytest.approx(ratio * 0.6, rel=1e-10)
    n = 96
    R = np.exp(np.log(0.25) + (np.arange(n) + 0.5) * np.log(4) / n)
    o = D.rotation_curve_elliptic(R, S0=p.S0, Kpoly=p.Kpoly, eps=p.eps, gamma_gas=p.gamma_gas)
    body = np.exp(-(R - 0.45) ** 2 / 0.05) >= 0.1
    assert o["Q"][body].min() == pytest.approx(Qmin, rel=1e-6)
    assert np.all(o["vphi2"][body] > 0) and np.all(o["kappa2"][body] > 0)


def test_params_physical_caps_unreachable_q():
    """Heavy hot disks of this family cannot reach Q_min = 1.5: K stops at the maximum."""
    p, q = D.params_physical(1.5, 1.0, 0.2, 2.0)
    assert q < 1.5
    n = 96
    R = np.exp(np.log(0.25) + (np.arange(n) + 0.5) * np.log(4) / n)
    body = np.exp(-(R - 0.45) ** 2 / 0.05) >= 0.1
    for f in (0.9, 1.1):
        o = D.rotation_curve_elliptic(R, S0=p.S0, Kpoly=p.Kpoly * f, eps=p.eps, gamma_gas=2.0)
        assert o["Q"][body].min() <= q + 1e-6


@pytest.mark.gpu
def test_init_standard_elliptic_rotation_curve():
    with D.Disk(128, 64, eps=0.005, basic_state="elliptic") as d:
        d.init_standard()
        S, vR, vp = d.get_state()
        ve = np.sqrt(D.rotation_curve_elliptic(d.R, eps=0.005)["vphi2"])
        assert np.max(np.abs(vp[:, 0] - ve) / ve) < 1e-12
