"""FP64 post-processing of mode records: growth rate and pattern speed of the m=2 spiral.

The reference derived gamma and Omega_p off-line from diskfft_modes.dat
(diskfft/README.md:26-29,37).  The convention follows Cm() (diskmain.cpp:72-84):
C_m = sum Sigma e^{-i m phi} dA / m_D, so a pattern rotating at Omega_p has
arg C_2 = -2 Omega_p t + const, and a growing mode |C_2| ~ e^{gamma t}.
"""
from __future__ import annotations

import numpy as np


def fit_growth(t, c2, arg2, tmin=None, tmax=None):
    """Least-squares (FP64) gamma = d ln|C2|/dt and Omega_p = -1/2 d(arg C2)/dt (unwrapped)
    over tmin <= t <= tmax.  Returns (gamma, omega_p, n_points)."""
    t = np.asarray(t, dtype=np.float64)
    c2 = np.asarray(c2, dtype=np.float64)
    ph = np.unwrap(np.asarray(arg2, dtype=np.float64))
    sel = np.ones_like(t, dtype=bool)
    if tmin is not None:
        sel &= t >= tmin
    if tmax is not None:
        sel &= t <= tmax
    sel &= c2 > 0
    if sel.sum() < 2:
        raise ValueError("need at least two records in the fit window")
    A = np.vstack([t[sel], np.ones(sel.sum())]).T
    g = np.linalg.lstsq(A, np.log(c2[sel]), rcond=None)[0][0]
    w = np.linalg.lstsq(A, ph[sel], rcond=None)[0][0]
    return float(g), float(-0.5 * w), int(sel.sum())


def saturation_ratio(c0, c2, tail=8):
    """Saturated |C2|/|C0|: the mean over the last `tail` records."""
    c0 = np.asarray(c0, dtype=np.float64)[-tail:]
    c2 = np.asarray(c2, dtype=np.float64)[-tail:]
    return float(np.mean(c2 / c0))


def linear_phase(t, c0, c2, arg2, t0=1.0, ratio_end=0.05):
    """gamma, Omega_p of the exponential phase: records from t0 (past the seed's transient)
    until |C2|/|C0| first exceeds ratio_end (the mode is still linear there).
    Returns (gamma, omega_p, n_points)."""
    t = np.asarray(t, dtype=np.float64)
    ratio = np.asarray(c2, dtype=np.float64) / np.asarray(c0, dtype=np.float64)
    hit = np.flatnonzero(ratio > ratio_end)
    tend = t[hit[0]] if len(hit) else t[-1]
    sel = (t >= t0) & (t <= tend)
    if sel.sum() < 4:
        sel = t >= 0.5 * t0
    return fit_growth(t[sel], np.asarray(c2)[sel], np.asarray(arg2)[sel])


def saturated_phase(t, c0, c2, arg2, ratio_min=0.15):
    """Mean |C2|/|C0| and pattern speed over the records where the mode has saturated
    (|C2|/|C0| >= ratio_min, from its first crossing to its last).  Returns
    (ratio, omega_p, n_points)."""
    t = np.asarray(t, dtype=np.float64)
    ratio = np.asarray(c2, dtype=np.float64) / np.asarray(c0, dtype=np.float64)
    hit = np.flatnonzero(ratio >= ratio_min)
    if len(hit) < 2:
        raise ValueError("the mode never saturated above ratio_min")
    sel = slice(hit[0], hit[-1] + 1)
    _, w, n = fit_growth(t[sel], np.asarray(c2)[sel], np.asarray(arg2)[sel])
    return float(np.mean(ratio[sel])), w, n
