"""ctypes binding of the plain-C oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by the
CPU-baseline leg of bench.py, to check results against.  Nothing in the product imports it.
It restates diskfft/src/{hydro.hpp,kalnajs.hpp,diskmain.cpp}; see diskoracle.h.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")


class OrcParams(C.Structure):
    _fields_ = [
        ("Nu", C.c_int), ("Nphi", C.c_int),
        ("eps", C.c_double), ("tlim", C.c_double),
        ("selfgrav", C.c_int), ("amp", C.c_double), ("nthreads", C.c_int),
        ("Rin", C.c_double), ("Rout", C.c_double), ("R0", C.c_double), ("w2", C.c_double),
        ("S0", C.c_double), ("Kpoly", C.c_double), ("gamma_gas", C.c_double),
        ("gmstar", C.c_double), ("G", C.c_double), ("phase0", C.c_double),
    ]


def build() -> None:
    """Compile liboracle.so (and oracle/_ref when the reference tree is present)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        D = C.POINTER(C.c_double)
        L.orc_hydro_create.restype = P
        L.orc_hydro_create.argtypes = [C.c_int, C.c_int] + [C.c_double] * 5
        L.orc_hydro_destroy.argtypes = [P]
        L.orc_hydro_field.restype = D
        L.orc_hydro_field.argtypes = [P, C.c_int]
        L.orc_set_threads.argtypes = [P, C.c_int]
        L.orc_timestep.restype = C.c_double
        L.orc_timestep.argtypes = [P, C.c_double]
        for f in ("orc_source",):
            getattr(L, f).argtypes = [P, C.c_double, D, D]
        L.orc_transportR.argtypes = [P, C.c_double]
        L.orc_transportPhi.argtypes = [P, C.c_double]
        L.orc_step.argtypes = [P, C.c_double, D, D]
        L.orc_kalnajs_create.restype = P
        L.orc_kalnajs_create.argtypes = [C.c_int, C.c_int] + [C.c_double] * 4 + [C.c_int]
        L.orc_kalnajs_destroy.argtypes = [P]
        L.orc_potential.argtypes = [P, D, D]
        L.orc_forces.argtypes = [P, D, D, D]
        L.orc_potential_direct.argtypes = [P, D, D]
        L.orc_khat.restype = D
        L.orc_khat.argtypes = [P]
        L.orc_params_default.argtypes = [C.POINTER(OrcParams)]
        L.orc_init_standard.argtypes = [C.POINTER(OrcParams), P, P]
        L.orc_disk_mass.restype = C.c_double
        L.orc_disk_mass.argtypes = [P]
        L.orc_cm.argtypes = [P, C.c_int, C.c_double, D, D]
        L.orc_run.restype = C.c_long
        L.orc_run.argtypes = [C.POINTER(OrcParams), P, P, C.c_long, D, C.c_void_p]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def default_params(**kw) -> OrcParams:
    p = OrcParams()
    lib().orc_params_default(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class Hydro:
    """CPU DiskHydro (diskfft/src/hydro.hpp:20-180)."""

    def __init__(self, Nu, Nphi, Rin=0.25, Rout=1.0, K=0.25, gamma=2.0, gmstar=0.6, nthreads=1):
        self.Nu, self.Nphi = Nu, Nphi
        self.h = lib().orc_hydro_create(Nu, Nphi, Rin, Rout, K, gamma, gmstar)
        lib().orc_set_threads(self.h, nthreads)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_hydro_destroy(self.h)
            self.h = None

    def _field(self, which, n):
        p = lib().orc_hydro_field(self.h, which)
        return np.ctypeslib.as_array(p, shape=(n,))

    def get(self, name):
        which = {"Sig": 0, "vR": 1, "vp": 2, "R": 3, "Rf": 4, "Vol": 5}[name]
        n = {3: self.Nu, 4: self.Nu + 1, 5: self.Nu}.get(which, self.Nu * self.Nphi)
        a = self._field(which, n).copy()
        return a if n != self.Nu * self.Nphi else a.reshape(self.Nu, self.Nphi)

    def set_state(self, Sig, vR, vp):
        n = self.Nu * self.Nphi
        for w, a in ((0, Sig), (1, vR), (2, vp)):
            self._field(w, n)[:] = np.ascontiguousarray(a, dtype=np.float64).ravel()

    def state(self):
        return self.get("Sig"), self.get("vR"), self.get("vp")

    def timestep(self, cfl=0.3):
        return lib().orc_timestep(self.h, cfl)

    def step(self, dt, gR=None, gp=None):
        a = np.ascontiguousarray(gR, dtype=np.float64) if gR is not None else None
        b = np.ascontiguousarray(gp, dtype=np.float64) if gp is not None else None
        lib().orc_step(self.h, dt, _dp(a) if a is not None else None, _dp(b) if b is not None else None)


class Kalnajs:
    """CPU KalnajsSolver (diskfft/src/kalnajs.hpp:19-117)."""

    def __init__(self, Nu, Nphi, Rin=0.25, Rout=1.0, eps=0.02, G=1.0, nthreads=1):
        self.Nu, self.Nphi = Nu, Nphi
        self.k = lib().orc_kalnajs_create(Nu, Nphi, Rin, Rout, eps, G, nthreads)

    def __del__(self):
        if getattr(self, "k", None):
            lib().orc_kalnajs_destroy(self.k)
            self.k = None

    def potential(self, Sig):
        s = np.ascontiguousarray(Sig, dtype=np.float64)
        out = np.empty((self.Nu, self.Nphi))
        lib().orc_potential(self.k, _dp(s), _dp(out))
        return out

    def potential_direct(self, Sig):
        s = np.ascontiguousarray(Sig, dtype=np.float64)
        out = np.empty((self.Nu, self.Nphi))
        lib().orc_potential_direct(self.k, _dp(s), _dp(out))
        return out

    def forces(self, Phi):
        p = np.ascontiguousarray(Phi, dtype=np.float64)
        gR = np.empty((self.Nu, self.Nphi))
        gp = np.empty((self.Nu, self.Nphi))
        lib().orc_forces(self.k, _dp(p), _dp(gR), _dp(gp))
        return gR, gp

    def khat(self):
        M, Nc = 2 * self.Nu, self.Nphi // 2 + 1
        a = np.ctypeslib.as_array(lib().orc_khat(self.k), shape=(M * Nc * 2,)).copy()
        return (a[0::2] + 1j * a[1::2]).reshape(M, Nc)


class Disk:
    """The diskdisk driver (diskfft/src/diskmain.cpp): standard disk, seed, loop."""

    def __init__(self, **kw):
        self.p = default_params(**kw)
        p = self.p
        self.hyd = Hydro(p.Nu, p.Nphi, p.Rin, p.Rout, p.Kpoly, p.gamma_gas, p.gmstar, p.nthreads)
        self.grav = Kalnajs(p.Nu, p.Nphi, p.Rin, p.Rout, p.eps, p.G, p.nthreads)
        lib().orc_init_standard(C.byref(p), self.hyd.h, self.grav.k)
        self.mD = lib().orc_disk_mass(self.hyd.h)

    def cm(self, m):
        mag, ph = C.c_double(), C.c_double()
        lib().orc_cm(self.hyd.h, m, self.mD, C.byref(mag), C.byref(ph))
        return mag.value, ph.value

    def gravity(self):
        Phi = self.grav.potential(self.hyd.get("Sig"))
        return self.grav.forces(Phi)

    def step(self):
        """One loop body of diskmain.cpp:100-108 without the tlim clip; returns dt."""
        dt = self.hyd.timestep(0.3)
        if self.p.selfgrav:
            gR, gp = self.gravity()
            self.hyd.step(dt, gR, gp)
        else:
            self.hyd.step(dt)
        return dt

    def run(self, max_steps=-1):
        t = C.c_double()
        n = lib().orc_run(C.byref(self.p), self.hyd.h, self.grav.k, max_steps, C.byref(t), None)
        return n, t.value


def read_refdump(path):
    """Parse the binary written by oracle/_ref/refdump (layout in refdump.cpp)."""
    with open(path, "rb") as f:
        Nu, Nphi, nsteps, selfgrav = np.frombuffer(f.read(16), dtype=np.int32)
        eps, amp, mD = np.frombuffer(f.read(24), dtype=np.float64)
        n = int(Nu) * int(Nphi)

        def arr(k):
            return np.frombuffer(f.read(8 * k), dtype=np.float64).copy()

        out = {"Nu": int(Nu), "Nphi": int(Nphi), "nsteps": int(nsteps), "selfgrav": int(selfgrav),
               "eps": float(eps), "amp": float(amp), "mD": float(mD)}
        for name in ("Sig0", "vR0", "vp0", "Phi0", "gR0", "gp0"):
            out[name] = arr(n).reshape(Nu, Nphi)
        out["dt"] = arr(int(nsteps))
        for name in ("SigN", "vRN", "vpN"):
            out[name] = arr(n).reshape(Nu, Nphi)
        out["c0"], out["ph0"], out["c2"], out["ph2"] = arr(4)
    return out
