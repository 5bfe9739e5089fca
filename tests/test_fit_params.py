"""Host-side ABI services, no GPU: the growth fit (dg_fit_growth, dg_fit_phases) against
the numpy fitters on the reference's own 256^2 run through saturation, and the sweep
parameter file (dg_params_write / dg_params_read)."""
import os

import numpy as np
import pytest

import diskgpu as D
from diskgpu import analysis as A
from diskgpu import sweep as S
from helpers import GOLDEN

REC = np.loadtxt(os.path.join(GOLDEN, "diskdisk_ref_256_e0.005_t20", "diskfft_modes.dat"))


@pytest.mark.parametrize("window", [(2.0, 6.0), (None, None), (1.0, None), (None, 12.0)])
def test_fit_growth_matches_numpy(window):
    g, w, n = D.fit_growth(REC, *window)
    g2, w2, n2 = A.fit_growth(REC[:, 0], REC[:, 2], REC[:, 3], tmin=window[0], tmax=window[1])
    assert n == n2
    assert g == pytest.approx(g2, rel=1e-12) and w == pytest.approx(w2, rel=1e-12)


def test_fit_phases_match_numpy_and_the_readme():
    (g, w, n), (r, ws, ns) = D.fit_phases(REC)
    g2, w2, n2 = A.linear_phase(*REC.T)
    r2, ws2, ns2 = A.saturated_phase(*REC.T)
    assert (n, ns) == (n2, ns2)
    assert g == pytest.approx(g2, rel=1e-12) and w == pytest.approx(w2, rel=1e-12)
    assert r == pytest.approx(r2, rel=1e-12) and ws == pytest.approx(ws2, rel=1e-12)
    # diskfft/README.md:37 (gamma 0.717 at 256^2) and README.md:41-42 (0.24; 1.46 -> 1.34)
    assert abs(g - 0.717) < 0.02 and abs(r - 0.24) < 0.01 and abs(w - 1.46) < 0.01


def test_fit_unwraps_the_phase():
    t = np.linspace(0, 5, 41)
    arg = np.angle(np.exp(-2j * 1.5 * t))  # pattern speed 1.5, wrapped into (-pi, pi]
    rec = np.stack([t, np.ones_like(t), 1e-3 * np.exp(0.4 * t), arg], axis=1)
    g, w, n = D.fit_growth(rec)
    assert n == 41 and g == pytest.approx(0.4, rel=1e-12) and w == pytest.approx(1.5, rel=1e-12)


def test_fit_rejects_short_windows():
    with pytest.raises(D.DiskGPUError) as e:
        D.fit_growth(REC, 30.0, 40.0)
    assert e.value.code == -1 and "fewer than two" in str(e.value)
    (_, _, _), (r, w, n) = D.fit_phases(REC[:20])  # never saturated
    assert n == 0 and np.isnan(r)


def test_params_file_round_trip(tmp_path):
    pts = S.draw(12, seed=7)
    path = tmp_path / "sweep.txt"
    S.write_sweep_file(path, pts)
    back = S.read_sweep_file(path)
    assert len(back) == 12
    for pt, q in zip(pts, back):
        want = S.point_params(pt)
        for f, _ in D.Params._fields_:
            assert getattr(q, f) == getattr(want, f), f


def test_params_file_sweep_coordinates_and_comments(tmp_path):
    path = tmp_path / "sweep.txt"
    path.write_text("# two disks\n"
                    "Qmin=1.1 mass_ratio=0.3 soft_over_r=0.15 gamma_gas=1.5 Nu=256 Nphi=256 precision=mixed\n"
                    "\n"
                    "Nu=64 Nphi=96 eps=0.01 amp=0.05   # plain keys, defaults for the rest\n")
    a, b = D.read_params(path)
    p, _ = D.params_physical(1.1, 0.3, 0.15, 1.5)
    assert (a.eps, a.gamma_gas, a.Kpoly, a.S0) == (p.eps, p.gamma_gas, p.Kpoly, p.S0)
    assert (a.Nu, a.Nphi, a.precision) == (256, 256, D.MIXED)
    d = D.default_params()
    assert (b.Nu, b.Nphi, b.eps, b.amp, b.Kpoly, b.precision) == (64, 96, 0.01, 0.05, d.Kpoly, D.FP64)


@pytest.mark.parametrize("text,what", [("Nu=64 bogus=1\n", "unknown key"), ("Nu=abc\n", "bad value"),
                                       ("Nu 64\n", "key=value"), ("Qmin=1.2 Nu=64\n", "go together")])
def test_params_file_errors_name_the_line(tmp_path, text, what):
    path = tmp_path / "bad.txt"
    path.write_text("# header\n" + text)
    with pytest.raises(D.DiskGPUError) as e:
        D.read_params(path)
    assert e.value.code == -1 and "line 2" in str(e.value) and what in str(e.value)
