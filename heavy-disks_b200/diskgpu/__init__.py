"""ctypes binding of libdiskgpu.so, the B200 diskfft time step (include/diskgpu.h).

The classes mirror the reference's C++ interface so that callers written against
diskfft/src/hydro.hpp and kalnajs.hpp (and Python drivers such as lka98/) read the same:

  DiskHydro(Nu, Nphi, Rin, Rout, K, gamma, GMstar)      hydro.hpp:28   .timestep(cfl) .step(dt, gR, gp)
  KalnajsSolver(Nu, Nphi, Rin, Rout, eps, G, nthreads)  kalnajs.hpp:25 .potential(Sigma) .forces(Phi)
  Disk(Nu, Nphi, eps, selfgrav, amp, ...)               the diskdisk driver (diskmain.cpp)

Errors from the library raise DiskGPUError carrying the status code and message.  There
is no CPU fallback: if the shared library is missing or no CUDA device is present, the
calls fail.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdiskgpu.so")

FP64 = 0
MIXED = 1

DG_OK = 0
STATUS = {
    -1: "DG_ERR_INVALID", -2: "DG_ERR_CUDA", -3: "DG_ERR_NONFINITE", -4: "DG_ERR_UNSUPPORTED",
    -5: "DG_ERR_NOMEM", -6: "DG_ERR_TIMEOUT", -7: "DG_ERR_STATE",
}


class DiskGPUError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class Params(C.Structure):
    _fields_ = [
        ("Nu", C.c_int), ("Nphi", C.c_int),
        ("Rin", C.c_double), ("Rout", C.c_double),
        ("Kpoly", C.c_double), ("gamma_gas", C.c_double), ("gmstar", C.c_double), ("G", C.c_double),
        ("eps", C.c_double), ("selfgrav", C.c_int), ("amp", C.c_double), ("phase0", C.c_double),
        ("R0", C.c_double), ("w2", C.c_double), ("S0", C.c_double),
        ("precision", C.c_int), ("device", C.c_int), ("basic_state", C.c_int),
    ]


class Record(C.Structure):
    _fields_ = [("t", C.c_double), ("c0", C.c_double), ("c2", C.c_double), ("arg2", C.c_double)]


# every symbol the C ABI exports (include/diskgpu.h)
EXPORTS = (
    "dg_params_default", "dg_create", "dg_destroy", "dg_last_error", "dg_status_string", "dg_grid",
    "dg_init_standard", "dg_set_state", "dg_get_state", "dg_timestep", "dg_step", "dg_step_forces",
    "dg_potential", "dg_forces", "dg_disk_mass", "dg_modes", "dg_conserved", "dg_advance", "dg_time",
    "dg_set_stream", "dg_run_steps", "dg_step_host", "dg_profile_enable", "dg_profile_read", "dg_kernels_per_step", "dg_tuning_info",
    "dg_timestep_static", "dg_rotation_curve_elliptic", "dg_params_physical",
    "dg_batch_create", "dg_batch_destroy", "dg_batch_last_error", "dg_batch_size", "dg_batch_disk",
    "dg_batch_init_standard", "dg_batch_advance", "dg_save", "dg_load", "dg_set_diagnostics",
    "dg_diagnostics_read", "dg_mlp_create", "dg_mlp_destroy", "dg_mlp_last_error", "dg_mlp_num_params",
    "dg_mlp_get_params", "dg_mlp_set_params", "dg_mlp_forward", "dg_mlp_loss_grad", "dg_mlp_train_step",
    "dg_capture_graph", "dg_advance_cb", "dg_fit_growth", "dg_fit_phases", "dg_params_write", "dg_params_read",
)

RECORD_FN = C.CFUNCTYPE(None, C.POINTER(Record), C.c_void_p)

BASIC_FFT, BASIC_ELLIPTIC = 0, 1

PROF_HYDRO, PROF_GRAVITY, PROF_CFL, PROF_GRAV_PHI_FWD, PROF_GRAV_U, PROF_GRAV_PHI_INV, PROF_N = 0, 1, 2, 3, 4, 5, 6
PROF_NAMES = ("hydro", "gravity", "cfl", "grav_phi_fwd", "grav_u", "grav_phi_inv")

_lib = None


def lib():
    """Load libdiskgpu.so (raises OSError if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} not found: build it with `make -C heavy-disks_b200` "
                      "(or __graft_entry__.build())")
    L = C.CDLL(LIB_PATH)
    H = C.c_void_p
    D = C.POINTER(C.c_double)
    L.dg_params_default.argtypes = [C.POINTER(Params)]
    L.dg_create.argtypes = [C.POINTER(Params), C.POINTER(H)]
    L.dg_destroy.argtypes = [H]
    L.dg_destroy.restype = None
    L.dg_last_error.argtypes = [H]
    L.dg_last_error.restype = C.c_char_p
    L.dg_status_string.argtypes = [C.c_int]
    L.dg_status_string.restype = C.c_char_p
    L.dg_grid.argtypes = [H, D, D, D]
    L.dg_init_standard.argtypes = [H]
    L.dg_set_state.argtypes = [H, D, D, D]
    L.dg_get_state.argtypes = [H, D, D, D]
    L.dg_timestep.argtypes = [H, C.c_double, D]
    L.dg_step.argtypes = [H, C.c_double]
    L.dg_step_forces.argtypes = [H, C.c_double, D, D]
    L.dg_potential.argtypes = [H, D, D]
    L.dg_forces.argtypes = [H, D, D, D]
    L.dg_disk_mass.argtypes = [H, D]
    L.dg_modes.argtypes = [H, C.c_int, D]
    L.dg_conserved.argtypes = [H, D, D]
    L.dg_advance.argtypes = [H, C.c_double, C.c_double, C.c_double, C.POINTER(Record), C.c_int,
                             C.POINTER(C.c_int), D, C.POINTER(C.c_longlong)]
    L.dg_time.argtypes = [H, D, C.POINTER(C.c_longlong)]
    L.dg_set_stream.argtypes = [H, C.c_void_p]
    L.dg_run_steps.argtypes = [H, C.c_int, C.c_double, C.c_int]
    L.dg_step_host.argtypes = [H, C.c_double, D, D, D, D]
    L.dg_profile_enable.argtypes = [H, C.c_int]
    L.dg_profile_read.argtypes = [H, D, C.POINTER(C.c_longlong)]
    L.dg_kernels_per_step.argtypes = [H]
    L.dg_tuning_info.argtypes = [H, C.c_char_p, C.c_int]
    L.dg_rotation_curve_elliptic.argtypes = [C.POINTER(Params), C.c_int, D, D, D, D, D]
    L.dg_params_physical.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double, C.POINTER(Params), D]
    L.dg_batch_create.argtypes = [C.c_int, C.POINTER(Params), C.POINTER(H)]
    L.dg_batch_destroy.argtypes = [H]
    L.dg_batch_destroy.restype = None
    L.dg_batch_last_error.argtypes = [H]
    L.dg_batch_last_error.restype = C.c_char_p
    L.dg_batch_size.argtypes = [H]
    L.dg_batch_disk.argtypes = [H, C.c_int]
    L.dg_batch_disk.restype = H
    L.dg_batch_init_standard.argtypes = [H]
    L.dg_batch_advance.argtypes = [H, C.c_double, C.c_double, C.c_double, C.c_int, C.POINTER(Record), C.c_int,
                                   C.POINTER(C.c_int), D, C.POINTER(C.c_longlong)]
    L.dg_save.argtypes = [H, C.c_char_p]
    L.dg_load.argtypes = [H, C.c_char_p]
    L.dg_set_diagnostics.argtypes = [H, C.c_int, C.c_int]
    L.dg_diagnostics_read.argtypes = [H, D, C.c_int, C.POINTER(C.c_int)]
    Fp = C.POINTER(C.c_float)
    L.dg_mlp_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_ulonglong, C.c_int, C.POINTER(H)]
    L.dg_mlp_destroy.argtypes = [H]
    L.dg_mlp_destroy.restype = None
    L.dg_mlp_last_error.argtypes = [H]
    L.dg_mlp_last_error.restype = C.c_char_p
    L.dg_mlp_num_params.argtypes = [H]
    L.dg_mlp_num_params.restype = C.c_longlong
    L.dg_mlp_get_params.argtypes = [H, Fp]
    L.dg_mlp_set_params.argtypes = [H, Fp]
    L.dg_mlp_forward.argtypes = [H, C.c_int, Fp, Fp]
    L.dg_mlp_loss_grad.argtypes = [H, C.c_int, Fp, Fp, Fp, Fp]
    L.dg_mlp_train_step.argtypes = [H, C.c_int, Fp, Fp, C.c_float, Fp]
    L.dg_capture_graph.argtypes = [H]
    L.dg_advance_cb.argtypes = [H, C.c_double, C.c_double, C.c_double, RECORD_FN, C.c_void_p, C.POINTER(C.c_int), D,
                                C.POINTER(C.c_longlong)]
    L.dg_fit_growth.argtypes = [C.POINTER(Record), C.c_int, C.c_double, C.c_double, D, D, C.POINTER(C.c_int)]
    L.dg_fit_phases.argtypes = [C.POINTER(Record), C.c_int, C.c_double, C.c_double, C.c_double, D]
    L.dg_params_write.argtypes = [C.c_char_p, C.POINTER(Params), C.c_int]
    L.dg_params_read.argtypes = [C.c_char_p, C.POINTER(Params), C.c_int, C.POINTER(C.c_int)]
    L.dg_timestep_static.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_double,
                                     C.c_double, C.c_double, C.c_double, C.c_double, C.c_void_p, C.c_void_p]
    _lib = L
    return L


def _dp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def _f64(a, shape):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.size != int(np.prod(shape)):
        raise ValueError(f"expected {shape} elements, got {a.shape}")
    return a


def default_params(**kw) -> Params:
    p = Params()
    lib().dg_params_default(C.byref(p))
    for k, v in kw.items():
        if k == "precision" and isinstance(v, str):
            v = {"fp64": FP64, "mixed": MIXED}[v]
        if k == "basic_state" and isinstance(v, str):
            v = {"fft": BASIC_FFT, "elliptic": BASIC_ELLIPTIC}[v]
        setattr(p, k, v)
    return p


def rotation_curve_elliptic(R, **kw):
    """FP64 elliptic-integral basic state at radii R: dict of gR, vphi2, kappa2, Q."""
    p = default_params(**kw)
    R = np.ascontiguousarray(R, dtype=np.float64)
    out = {k: np.empty_like(R) for k in ("gR", "vphi2", "kappa2", "Q")}
    rc = lib().dg_rotation_curve_elliptic(C.byref(p), len(R), _dp(R), _dp(out["gR"]), _dp(out["vphi2"]),
                                          _dp(out["kappa2"]), _dp(out["Q"]))
    if rc != DG_OK:
        raise DiskGPUError(rc, "dg_rotation_curve_elliptic")
    return out


def params_physical(Qmin, mass_ratio, soft_over_r, gamma_gas, **kw):
    """(dg_params, achieved Q_min) for a sweep point (Q_min, M_d/M_*, softening/r, Gamma)."""
    p = default_params(**kw)
    q = C.c_double()
    rc = lib().dg_params_physical(Qmin, mass_ratio, soft_over_r, gamma_gas, C.byref(p), C.byref(q))
    if rc != DG_OK:
        raise DiskGPUError(rc, "dg_params_physical")
    return p, q.value


def _records(rec):
    """(n, 4) array of t, |C0|, |C2|, arg C2 -> ctypes Record array."""
    rec = np.asarray(rec, dtype=np.float64).reshape(-1, 4)
    arr = (Record * max(len(rec), 1))()
    for k, (t, c0, c2, a2) in enumerate(rec):
        arr[k].t, arr[k].c0, arr[k].c2, arr[k].arg2 = t, c0, c2, a2
    return arr, len(rec)


def fit_growth(rec, tmin=None, tmax=None):
    """dg_fit_growth: FP64 least-squares gamma = d ln|C2|/dt and Omega_p = -1/2 d arg C2/dt
    over tmin <= t <= tmax; returns (gamma, omega_p, n_points)."""
    arr, n = _records(rec)
    g, w, k = C.c_double(), C.c_double(), C.c_int()
    rc = lib().dg_fit_growth(arr, n, np.nan if tmin is None else tmin, np.nan if tmax is None else tmax,
                             C.byref(g), C.byref(w), C.byref(k))
    if rc != DG_OK:
        raise DiskGPUError(rc, lib().dg_last_error(None).decode())
    return g.value, w.value, k.value


def fit_phases(rec, t0=1.0, ratio_end=0.05, ratio_min=0.15):
    """dg_fit_phases: ((gamma, Omega_p, n) of the linear phase, (|C2|/|C0|, Omega_p, n) of the
    saturated phase)."""
    arr, n = _records(rec)
    out = np.zeros(6)
    rc = lib().dg_fit_phases(arr, n, t0, ratio_end, ratio_min, _dp(out))
    if rc != DG_OK:
        raise DiskGPUError(rc, lib().dg_last_error(None).decode())
    return (out[0], out[1], int(out[2])), (out[3], out[4], int(out[5]))


def write_params(path, params_list):
    """dg_params_write: the plain-text parameter file of a sweep (one disk per line)."""
    arr = (Params * max(len(params_list), 1))(*[Params.from_buffer_copy(p) for p in params_list])
    rc = lib().dg_params_write(os.fsencode(path), arr, len(params_list))
    if rc != DG_OK:
        raise DiskGPUError(rc, lib().dg_last_error(None).decode())


def read_params(path, max_disks=1 << 16):
    """dg_params_read: the disks of a parameter file as a list of Params."""
    arr = (Params * max_disks)()
    n = C.c_int()
    rc = lib().dg_params_read(os.fsencode(path), arr, max_disks, C.byref(n))
    if rc != DG_OK:
        raise DiskGPUError(rc, lib().dg_last_error(None).decode())
    return [Params.from_buffer_copy(arr[k]) for k in range(n.value)]


class Disk:
    """One disk on one GPU: the handle of include/diskgpu.h."""

    def __init__(self, Nu=128, Nphi=128, eps=0.02, selfgrav=1, amp=None, precision="fp64", params=None, **kw):
        """With `params` (a Params), the disk takes them with Nu, Nphi, precision and any
        keyword given here replacing theirs (amp only when given); otherwise the standard
        disk of default_params with these values (amp 1e-3 unless given)."""
        if params is not None:
            self.p = Params.from_buffer_copy(params)
            over = dict(Nu=Nu, Nphi=Nphi, precision=precision, **kw)
            if amp is not None:
                over["amp"] = amp
            for k, v in over.items():
                if k == "precision" and isinstance(v, str):
                    v = {"fp64": FP64, "mixed": MIXED}[v]
                setattr(self.p, k, v)
        else:
            self.p = default_params(Nu=Nu, Nphi=Nphi, eps=eps, selfgrav=selfgrav, amp=1e-3 if amp is None else amp,
                                    precision=precision, **kw)
        self.Nu, self.Nphi = Nu, Nphi
        h = C.c_void_p()
        rc = lib().dg_create(C.byref(self.p), C.byref(h))
        if rc != DG_OK:
            raise DiskGPUError(rc, lib().dg_last_error(None).decode())
        self.h = h
        self.R = np.empty(Nu)
        self.Rf = np.empty(Nu + 1)
        self.Vol = np.empty(Nu)
        self._ck(lib().dg_grid(self.h, _dp(self.R), _dp(self.Rf), _dp(self.Vol)))
        self.dphi = 2.0 * np.pi / Nphi

    def _ck(self, rc):
        if rc != DG_OK:
            raise DiskGPUError(rc, lib().dg_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            lib().dg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def shape(self):
        return (self.Nu, self.Nphi)

    def init_standard(self):
        self._ck(lib().dg_init_standard(self.h))

    def set_state(self, Sig, vR, vp):
        s, a, b = (_f64(x, self.shape) for x in (Sig, vR, vp))
        self._ck(lib().dg_set_state(self.h, _dp(s), _dp(a), _dp(b)))

    def get_state(self):
        s, a, b = (np.empty(self.shape) for _ in range(3))
        self._ck(lib().dg_get_state(self.h, _dp(s), _dp(a), _dp(b)))
        return s, a, b

    def timestep(self, cfl=0.3):
        dt = C.c_double()
        self._ck(lib().dg_timestep(self.h, cfl, C.byref(dt)))
        return dt.value

    def step(self, dt):
        """potential -> forces -> hydro step (diskmain.cpp:102-105)."""
        self._ck(lib().dg_step(self.h, dt))

    def step_forces(self, dt, gR=None, gp=None):
        """DiskHydro::step(dt, gR, gp) with caller forces (hydro.hpp:63)."""
        a = None if gR is None else _f64(gR, self.shape)
        b = None if gp is None else _f64(gp, self.shape)
        self._ck(lib().dg_step_forces(self.h, dt, _dp(a), _dp(b)))

    def potential(self, Sig):
        s = _f64(Sig, self.shape)
        out = np.empty(self.shape)
        self._ck(lib().dg_potential(self.h, _dp(s), _dp(out)))
        return out

    def forces(self, Phi):
        f = _f64(Phi, self.shape)
        gR, gp = np.empty(self.shape), np.empty(self.shape)
        self._ck(lib().dg_forces(self.h, _dp(f), _dp(gR), _dp(gp)))
        return gR, gp

    def modes(self, mmax=2):
        """C_m = sum Sigma e^{-i m phi} dA / m_D, m = 0..mmax (diskmain.cpp:72-84)."""
        buf = np.empty(2 * (mmax + 1))
        self._ck(lib().dg_modes(self.h, mmax, _dp(buf)))
        return buf[0::2] + 1j * buf[1::2]

    def cm(self, m):
        """(|C_m|, arg C_m) as Cm() in diskmain.cpp:72-84."""
        c = self.modes(max(m, 0))[m]
        return abs(c), float(np.angle(c))

    def conserved(self):
        m, L = C.c_double(), C.c_double()
        self._ck(lib().dg_conserved(self.h, C.byref(m), C.byref(L)))
        return m.value, L.value

    def disk_mass(self):
        m = C.c_double()
        self._ck(lib().dg_disk_mass(self.h, C.byref(m)))
        return m.value

    def time(self):
        t, n = C.c_double(), C.c_longlong()
        self._ck(lib().dg_time(self.h, C.byref(t), C.byref(n)))
        return t.value, n.value

    def advance(self, tlim, cfl=0.3, dtout=0.25, max_rec=None, on_record=None):
        """Run the diskmain.cpp loop to tlim on the device; returns (records, t, steps)
        with records an (n, 4) array of t, |C0|, |C2|, arg C2.  With on_record(t, c0, c2,
        arg2) every record is also handed over as soon as the host drains it
        (dg_advance_cb)."""
        if on_record is not None:
            got = []

            def cb(r, _user):
                rr = r.contents
                got.append((rr.t, rr.c0, rr.c2, rr.arg2))
                on_record(*got[-1])

            fn = RECORD_FN(cb)
            n, t, s = C.c_int(), C.c_double(), C.c_longlong()
            self._ck(lib().dg_advance_cb(self.h, tlim, cfl, dtout, fn, None, C.byref(n), C.byref(t), C.byref(s)))
            return np.array(got, dtype=np.float64).reshape(-1, 4), t.value, s.value
        t0, _ = self.time()
        if max_rec is None:
            max_rec = int(max(tlim - t0, 0) / dtout) + 8
        recs = (Record * max_rec)()
        n, t, s = C.c_int(), C.c_double(), C.c_longlong()
        self._ck(lib().dg_advance(self.h, tlim, cfl, dtout, recs, max_rec, C.byref(n), C.byref(t), C.byref(s)))
        out = np.array([[r.t, r.c0, r.c2, r.arg2] for r in recs[: n.value]]).reshape(-1, 4)
        return out, t.value, s.value


    def save(self, path):
        self._ck(lib().dg_save(self.h, os.fsencode(path)))

    def load(self, path):
        self._ck(lib().dg_load(self.h, os.fsencode(path)))

    def set_diagnostics(self, mmax=8, capacity=4096):
        """Record C_0..C_mmax on the device every step (capacity 0 = off)."""
        self._ck(lib().dg_set_diagnostics(self.h, mmax, capacity))
        self._diag_mmax = mmax

    def diagnostics(self, max_rows=1 << 20):
        """Drain the per-step ring: (t[n], C[n, mmax+1] complex)."""
        mm = getattr(self, "_diag_mmax", 8)
        w = 1 + 2 * (mm + 1)
        buf = np.empty(max_rows * w)
        n = C.c_int()
        self._ck(lib().dg_diagnostics_read(self.h, _dp(buf), max_rows, C.byref(n)))
        rows = buf[: n.value * w].reshape(n.value, w)
        return rows[:, 0].copy(), rows[:, 1::2] + 1j * rows[:, 2::2]

    # ---- GPU-side extensions ----
    def set_stream(self, stream_ptr):
        """Queue all work of this disk on a caller CUDA stream (int handle; 0 = own stream)."""
        self._ck(lib().dg_set_stream(self.h, C.c_void_p(stream_ptr or None)))

    def run_steps(self, nsteps, cfl=0.3, sync=True):
        """nsteps device-resident steps with device-side dt (no host sync when sync=False)."""
        self._ck(lib().dg_run_steps(self.h, nsteps, cfl, 1 if sync else 0))

    def capture_graph(self):
        """Record the 64-step device-loop graph now, so no later call pays for it."""
        self._ck(lib().dg_capture_graph(self.h))

    def step_host(self, Sig, vR, vp, cfl=0.3):
        """One reference-style step on host arrays (float64, C-contiguous), in place; returns dt."""
        for a in (Sig, vR, vp):
            if a.dtype != np.float64 or not a.flags.c_contiguous or a.size != self.Nu * self.Nphi:
                raise ValueError("step_host needs C-contiguous float64 arrays of Nu*Nphi")
        dt = C.c_double()
        self._ck(lib().dg_step_host(self.h, cfl, _dp(Sig), _dp(vR), _dp(vp), C.byref(dt)))
        return dt.value

    def profile(self, on=True):
        self._ck(lib().dg_profile_enable(self.h, 1 if on else 0))

    def profile_read(self):
        """{phase: (ms, launches)} accumulated since the last read."""
        ms = np.zeros(PROF_N)
        cnt = (C.c_longlong * PROF_N)()
        self._ck(lib().dg_profile_read(self.h, _dp(ms), cnt))
        return {PROF_NAMES[k]: (float(ms[k]), int(cnt[k])) for k in range(PROF_N)}

    def tuning(self):
        """The autotuner's choices for this disk (one line of text)."""
        buf = C.create_string_buffer(512)
        self._ck(lib().dg_tuning_info(self.h, buf, 512))
        return buf.value.decode()

    def kernels_per_step(self):
        """How many of this library's kernels one time step launches."""
        n = lib().dg_kernels_per_step(self.h)
        if n < 0:
            raise DiskGPUError(n, "dg_kernels_per_step")
        return n


class _BorrowedDisk(Disk):
    """A disk owned by a Batch (no destroy on close)."""

    def __init__(self, handle, params):
        self.h = handle
        self.p = params
        self.Nu, self.Nphi = params.Nu, params.Nphi
        self.R = np.empty(self.Nu)
        self.Rf = np.empty(self.Nu + 1)
        self.Vol = np.empty(self.Nu)
        self._ck(lib().dg_grid(self.h, _dp(self.R), _dp(self.Rf), _dp(self.Vol)))
        self.dphi = 2.0 * np.pi / self.Nphi

    def close(self):
        self.h = None


class Batch:
    """Many independent disks advanced by one CUDA graph per launch (dg_batch)."""

    def __init__(self, params_list):
        arr = (Params * len(params_list))(*[Params.from_buffer_copy(p) for p in params_list])
        h = C.c_void_p()
        rc = lib().dg_batch_create(len(params_list), arr, C.byref(h))
        if rc != DG_OK:
            raise DiskGPUError(rc, lib().dg_last_error(None).decode())
        self.h = h
        self.n = len(params_list)
        self.disks = [_BorrowedDisk(lib().dg_batch_disk(h, k), Params.from_buffer_copy(params_list[k]))
                      for k in range(self.n)]

    def _ck(self, rc):
        if rc != DG_OK:
            raise DiskGPUError(rc, lib().dg_batch_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            for d in self.disks:
                d.close()
            lib().dg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def init_standard(self):
        self._ck(lib().dg_batch_init_standard(self.h))

    def advance(self, tlim, cfl=0.3, dtout=0.25, steps_per_launch=16, max_rec=None):
        """Advance all disks to tlim; returns (list of (n_k, 4) record arrays, t[n], steps[n])."""
        if max_rec is None:
            max_rec = int(tlim / dtout) + 8
        recs = (Record * (self.n * max_rec))()
        nrec = (C.c_int * self.n)()
        t = np.zeros(self.n)
        s = (C.c_longlong * self.n)()
        self._ck(lib().dg_batch_advance(self.h, tlim, cfl, dtout, steps_per_launch, recs, max_rec, nrec, _dp(t), s))
        out = []
        for k in range(self.n):
            rr = recs[k * max_rec: k * max_rec + nrec[k]]
            out.append(np.array([[r.t, r.c0, r.c2, r.arg2] for r in rr]).reshape(-1, 4))
        return out, t, np.array(list(s))


class DiskHydro:
    """Mirror of diskfft::DiskHydro (hydro.hpp:20-180) backed by the GPU step."""

    def __init__(self, Nu, Nphi, Rin=0.25, Rout=1.0, K=0.25, gamma=2.0, GMstar=0.6, precision="fp64"):
        self._d = Disk(Nu, Nphi, selfgrav=0, Rin=Rin, Rout=Rout, Kpoly=K, gamma_gas=gamma, gmstar=GMstar,
                       precision=precision)
        self.Nu, self.Nphi = Nu, Nphi
        self.R, self.Rf, self.Vol = self._d.R, self._d.Rf, self._d.Vol
        self.dphi = self._d.dphi
        self.Sig = np.zeros((Nu, Nphi))
        self.vR = np.zeros((Nu, Nphi))
        self.vp = np.zeros((Nu, Nphi))
        self._dirty = True

    def _push(self):
        self._d.set_state(self.Sig, self.vR, self.vp)

    def timestep(self, cfl):
        self._push()
        return self._d.timestep(cfl)

    def step(self, dt, gR=None, gp=None):
        self._push()
        self._d.step_forces(dt, gR, gp)
        self.Sig, self.vR, self.vp = self._d.get_state()


class KalnajsSolver:
    """Mirror of diskfft::KalnajsSolver (kalnajs.hpp:19-117) backed by the GPU FFT."""

    def __init__(self, Nu, Nphi, Rin=0.25, Rout=1.0, eps=0.02, G=1.0, nthreads=1):
        self._d = Disk(Nu, Nphi, eps=eps, selfgrav=1, Rin=Rin, Rout=Rout, G=G)
        self.Nu, self.Nphi = Nu, Nphi
        self.R = self._d.R
        self.dphi = self._d.dphi

    def potential(self, Sigma):
        return self._d.potential(Sigma)

    def forces(self, Phi):
        return self._d.forces(Phi)
