"""Benchmark of the diskfft time step on B200: zone-updates/s (hydro + FFT gravity).

One "step" is one time step of one disk: dt (device CFL reduction fused in the hydro
epilogue), the Kalnajs gravity convolution and the fused hydro sweep.  At N GPUs every
rank advances its own disk (independent disks, weak scaling) and `value` is the total
zone-updates/s of the job, timed on the device as the max over ranks.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision mixed|fp64]
                  [--size 1024] [--chunk 64] [--cold-steps 200] [--impl ours|reference]

After exactly W untimed warm-up steps, the K timed steps run as dg_run_steps calls of
--chunk steps (each one launch of the captured step loop, the way dg_advance runs a disk;
the graph is recorded before the warm-up, so no timed call pays for it), with L2 flushed
before every call and CUDA events around it.  --repeats more timed regions of K steps give
the spread.  Then --cold-steps single steps, each after an L2 flush, give the cold per-step
time and, with per-kernel events, the roofline of every kernel of the step.  On one GPU the
line also carries `fp64_same_disk` (the plain FP64 path on the same disk, timed over the
same K steps, and the mixed/FP64 ratio the metric names), `cufft_gravity` (the same padded
convolution through cuFFT, as a timing comparison only) and `batched_sweep` (256 disks of
the sweep law, grids 128^2..512^2, advanced together by dg_batch; inside it `batched_1024`,
16 sweep-law disks all at 1024^2 as one graph branch each (with the grouped kernels'
figure beside it), and their ratio to the plain FP64 path at 1024^2).

--impl reference times the reference's own CPU implementation (diskfft/src hydro.hpp +
kalnajs.hpp compiled unmodified against the FFTW-API shim, with the reference Makefile's
-O3 and FP contraction: oracle/_ref/refbench_fast_v4, or _v3 on hosts without AVX-512) on
the host cores for the same workload; under torchrun only rank 0 runs it.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "heavy-disks_b200"))

METRIC = "zone-updates/s/GPU (hydro+FFT gravity), mixed vs FP64 plain at matched γ,Ω_p"
UNIT = "zone-updates/s"
REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def refbench_path():
    """The timing build of the reference for this host: x86-64-v4 where the CPU has
    AVX-512 (the reference Makefile's -march=native on such hosts), else x86-64-v3."""
    avx512 = False
    try:
        with open("/proc/cpuinfo") as f:
            avx512 = any(l.startswith("flags") and " avx512f" in l for l in f)
    except OSError:
        pass
    for name in (("refbench_fast_v4",) if avx512 else ()) + ("refbench_fast_v3", "refbench"):
        p = os.path.join(REF_DIR, name)
        if os.path.exists(p):
            return p
    return None


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10240)
    ap.add_argument("--warmup", type=int, default=50)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--size", type=int, default=1024)
    ap.add_argument("--eps", type=float, default=0.005)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--chunk", type=int, default=64, help="steps per timed iteration (one graph launch)")
    ap.add_argument("--cold-steps", type=int, default=200,
                    help="single steps with a flushed L2, timed and profiled per kernel")
    ap.add_argument("--fp64-steps", type=int, default=None,
                    help="steps of the plain FP64 path on the same disk (default: --steps; 0: skip it)")
    ap.add_argument("--repeats", type=int, default=5, help="extra timed regions of K steps for the spread")
    ap.add_argument("--cufft", type=int, default=1, help="time the cuFFT form of the gravity (0: skip)")
    ap.add_argument("--drift-steps", type=int, default=0,
                    help="steps with the per-step m = 0..8 diagnostic on, reporting the FP64 mass and angular "
                         "momentum drift (0: skip)")
    ap.add_argument("--batch-disks", type=int, default=256,
                    help="disks of the batched sweep measurement (0: skip it)")
    ap.add_argument("--batch-tlim", type=float, default=0.5,
                    help="time the batched sweep advances (long enough that the last launch's pass-through "
                         "steps of disks already at tlim are a small part of the timed region)")
    ap.add_argument("--batch-grids", default="128,256,384,512", help="grid sizes the batch draws from")
    ap.add_argument("--batch-seed", type=int, default=12345, help="seed of the batch's sweep-law draw")
    ap.add_argument("--batch1024-disks", type=int, default=16,
                    help="disks of the batched 1024^2 measurement (sweep-law physics, every grid 1024^2; 0: skip)")
    ap.add_argument("--batch1024-tlim", type=float, default=0.25, help="time the batched 1024^2 disks advance")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def workload(a):
    return {
        "workload": f"single standard heavy disk {a.size}x{a.size} (log R x phi), gravity on a "
                    f"{2 * a.size}x{a.size} zero-padded grid, eps={a.eps}, m=2 seed amp 1e-3, "
                    "one time step = CFL dt + Kalnajs gravity + van-Leer MUSCL hydro",
        "Nu": a.size, "Nphi": a.size, "eps": a.eps,
    }


# ---------------------------------------------------------------------------------
# CPU reference (host cores)

def run_refbench(size, eps, threads, warm, steps):
    out = subprocess.run([refbench_path(), str(size), str(size), repr(eps), str(threads), str(warm), str(steps)],
                         capture_output=True, text=True, check=True).stdout
    return json.loads(out.strip().splitlines()[-1])


def cpu_sample(size, eps, seconds=10.0):
    """Bounded sample of the reference build: estimate the step time, then time ~`seconds`."""
    threads = os.cpu_count() or 1
    if refbench_path() is None:
        return None
    probe = run_refbench(size, eps, threads, 1, 2)
    per = probe["seconds"] / 2
    steps = max(3, min(2000, int(seconds / max(per, 1e-6))))
    r = run_refbench(size, eps, threads, 1, steps)
    return {"value": r["zone_updates_per_s"], "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"{steps} steps of the {size}x{size} disk (eps {eps}) by the reference's DiskHydro + "
                      f"KalnajsSolver compiled unmodified with the project FFTW-API shim (not FFTW), "
                      f"-O3 with FP contraction ({os.path.basename(refbench_path())}), {threads} OpenMP "
                      f"threads, wall clock"}


def reference_arm(a, rank):
    if rank != 0:
        return
    if refbench_path() is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/refbench not built"}))
        return
    threads = os.cpu_count() or 1
    r = run_refbench(a.size, a.eps, threads, max(a.warmup, 1), a.steps)
    v = r["zone_updates_per_s"]
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": 1e3 * r["seconds"] / a.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": workload(a),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"{a.steps} timed steps after {max(a.warmup, 1)} warm-up, reference "
                                   "sources compiled unmodified with the project FFTW-API shim, -O3 with FP "
                                   f"contraction ({os.path.basename(refbench_path())})"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------------
# clocks during the timed region

class ClockSampler:
    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []
        self.window = None  # (t0, t1) host wall clock of the timed region

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

        def collect(lo, hi):
            sm, mx, reasons = [], None, set()
            for ts, l in self.lines:
                if not (lo <= ts <= hi):
                    continue
                f = [x.strip() for x in l.split(",")]
                if len(f) < 10:
                    continue
                try:
                    sm.append(float(f[2]))
                    mx = float(f[3])
                except ValueError:
                    continue
                for k, n in enumerate(names):
                    if f[6 + k].lower().startswith("active"):
                        reasons.add(n)
            return sm, mx, reasons

        where = "timed region"
        lo, hi = self.window if self.window else (0.0, float("inf"))
        sm, mx, reasons = collect(lo, hi + 0.05)
        if not sm:  # region shorter than the sampling period: take the loaded warm-up + timed span
            where = "warm-up and timed region"
            sm, mx, reasons = collect(0.0, float("inf"))
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "window": where}


def physical_gpu_index(local):
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [x.strip() for x in vis.split(",") if x.strip()]
        if local < len(ids) and ids[local].isdigit():
            return int(ids[local])
    return local


def measured_peaks():
    """(HBM GB/s, dense BF16 TFLOP/s, kind).  The sustained tensor figure applies: the
    gravity GEMMs are timed inside a seconds-long loop of steps."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), float(pk.get("bf16_tflops_sustained", pk["bf16_tflops"])), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, 1400.0, "fallback"


def ncu_traffic(precision, size):
    """DRAM bytes per launch of each kernel (dram__bytes_read.sum + dram__bytes_write.sum)
    from the committed ncu summary of this workload, or {} when none was captured."""
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            return json.load(f).get(f"{precision}_{size}", {})
    except (OSError, ValueError):
        return {}


def gravity_parts(precision, Nu, Nphi):
    """(phase, kernel, bound, work per launch, unit of work) of the three gravity parts."""
    M = 2 * Nu
    if precision == "fp64":
        # HBM-bound FFT passes; algorithmic bytes: Sigma in + half spectrum out (phi forward),
        # spectrum in/out + khat (u convolution), spectrum in + Phi out (phi inverse)
        nc = Nphi // 2 + 1
        spec = 16 * M * nc
        return [("grav_phi_fwd", "FP64 smem FFT, phi forward (k_phi_fwd)", "hbm", 8 * Nu * Nphi + spec, "B"),
                ("grav_u", "FP64 smem FFT, u convolution x khat (k_u_conv)", "hbm", 2 * spec + spec, "B"),
                ("grav_phi_inv", "FP64 smem FFT, phi inverse + scaling (k_phi_inv)", "hbm", spec + 8 * Nu * Nphi, "B")]
    # split-BF16 tcgen05 products: 3 MMAs per term, 2 flops per MAC
    g1 = 6 * Nphi * Nu * Nphi
    g1name = "phi DFT GEMM (k_gemm_split, split-BF16)"
    if Nu == 1024 and Nphi == 1024:  # fused two-stage transform: 4 rows per CTA, 2 products
        g1 = (Nu // 4) * (6 * 128 * 64 * 32 + 6 * 128 * 64 * 64)
        g1name = "fused phi transform (k_phifwd: real 32-point + complex 32-point tcgen05 stages)"
    g4 = 6 * Nu * Nphi * Nphi
    g4name = "inverse phi DFT GEMM + potential scaling (k_gemm_split)"
    if Nu == 1024 and Nphi == 1024:  # fused two-stage inverse: 4 rows per CTA, 2 products
        g4 = (Nu // 4) * (6 * 128 * 64 * 64 + 6 * 128 * 32 * 64)
        g4name = ("fused inverse phi transform (k_phiinv: complex 32-point + real-output 32-point tcgen05 "
                  "stages, potential scaling)")
    if Nphi == 4096 and Nu % 1024 == 0 and Nu != 1024:  # four-step 64 x 64 phi transforms, two products each
        g1 = 6 * 128 * (Nu * 64) * 64 + 6 * (64 * Nu) * 128 * 128
        g1name = "four-step phi transform (two k_gemm_split passes: real 64-point over j1, twiddle, complex 64-point)"
        g4 = 6 * (64 * Nu) * 128 * 128 + 6 * (64 * Nu) * 64 * 128
        g4name = ("four-step inverse phi transform (two k_gemm_split passes: complex 64-point, twiddle, real-output "
                  "64-point, potential scaling)")
    if Nu % 1024 == 0:
        A, nm = Nu // 32, ((Nphi // 2 + 1) + 3) // 4 * 4
        u = 6 * 128 * (nm * A) * 64 + 2 * 6 * (nm * 64) * (2 * A) * (2 * A) + 6 * (nm * A) * 64 * 128
        uname = ("fused factored u convolution (k_uconv: 64 x 32 Cooley-Tukey in four tcgen05 stages)"
                 if Nu == 1024 else "factored u convolution (four k_gemm_split passes)")
    else:
        u = 6 * Nphi * 2 * Nu * Nu + 6 * Nu * Nphi * 2 * Nu
        uname = "dense u DFT x khat (two k_gemm_split passes)"
    return [("grav_phi_fwd", g1name, "tensor", g1, "flop"),
            ("grav_u", uname, "tensor", u, "flop"),
            ("grav_phi_inv", g4name, "tensor", g4, "flop")]


def chunk_sizes(steps, chunk):
    chunk = max(1, min(chunk, steps))
    return [chunk] * (steps // chunk) + ([steps % chunk] if steps % chunk else [])


def warm_up(disk, stream, flush, warmup, chunk):
    """Exactly `warmup` untimed steps as dg_run_steps calls of up to `chunk` steps, after
    recording the step graph (which runs nothing)."""
    import torch
    disk.capture_graph()
    with torch.cuda.stream(stream):
        for n in (chunk_sizes(warmup, chunk) if warmup > 0 else []):
            flush.zero_()
            disk.run_steps(n, 0.3, sync=False)
        torch.cuda.synchronize()


def timed_region(disk, stream, flush, steps, chunk):
    """Device milliseconds of `steps` steps run as dg_run_steps calls of `chunk` steps, L2
    flushed before every call (outside the events), CUDA events around each call."""
    import torch
    sizes = chunk_sizes(steps, chunk)
    with torch.cuda.stream(stream):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in sizes]
        for k, n in enumerate(sizes):
            flush.zero_()
            ev[k][0].record(stream)
            disk.run_steps(n, 0.3, sync=False)
            ev[k][1].record(stream)
        torch.cuda.synchronize()
    return sum(b.elapsed_time(e) for b, e in ev)


def spread(ms_list, steps):
    per = sorted(m / steps for m in ms_list)
    return {"regions": len(per), "median_ms_per_step": statistics.median(per), "min_ms_per_step": per[0],
            "max_ms_per_step": per[-1]}


def fp64_same_disk(a, device, stream, flush, phase0, steps, chunk):
    """The plain FP64 path (the reference's arithmetic) on the same disk, with the same
    warm-up, the same K timed steps in the same chunks, and the same repeats."""
    import diskgpu as D
    N = a.size
    with D.Disk(N, N, eps=a.eps, amp=1e-3, precision="fp64", phase0=phase0, device=device) as d:
        d.init_standard()
        d.set_stream(stream.cuda_stream)
        warm_up(d, stream, flush, max(a.warmup, 3), chunk)
        ms = timed_region(d, stream, flush, steps, chunk)
        reps = [timed_region(d, stream, flush, steps, chunk) for _ in range(a.repeats)]
        d.run_steps(0, 0.3, sync=True)
    return {"value": N * N * steps / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms / steps, "steps": steps,
            "repeats": spread(reps, steps) if reps else None,
            "how": "same disk, warm-up, K steps, chunks and L2 flushes as the headline, precision fp64 "
                   "(k_hydro64 + three shared-memory FFT passes)"}


def khat_table(Nu, Nphi, eps):
    """The Green's-function spectrum of kalnajs.hpp:105-116 (r2c of the softened kernel at
    wrapped radial offsets), real and even, FP64: the multiplier of the cuFFT comparison."""
    import numpy as np
    M = 2 * Nu
    du, dphi = np.log(4.0) / Nu, 2 * np.pi / Nphi
    p = np.arange(M)
    ioff = np.where(p <= M // 2, p, p - M)
    K = 1.0 / np.sqrt(2.0 * np.cosh(ioff * du)[:, None] - 2.0 * np.cos(np.arange(Nphi) * dphi)[None, :] + eps)
    return np.fft.rfft2(K)


def cufft_gravity(a, device, flush, disk64_potential):
    """Timing comparison only (the product never calls cuFFT): the same zero-padded
    2 Nu x Nphi convolution as kalnajs.hpp:48-63 through cuFFT (torch.fft: D2Z / Z2D in
    FP64, R2C / C2R in FP32), with the khat multiply, padding and scaling as torch
    elementwise kernels, recorded in a CUDA graph and replayed after an L2 flush."""
    import numpy as np
    import torch
    N = a.size
    Nu = Nphi = N
    M = 2 * Nu
    du, dphi = np.log(4.0) / Nu, 2 * np.pi / Nphi
    R = np.exp(np.log(0.25) + (np.arange(Nu) + 0.5) * du)
    kh = khat_table(Nu, Nphi, a.eps)
    rng = np.random.default_rng(5)
    S0 = 0.372 * np.exp(-(R - 0.45) ** 2 / 0.05)
    Sig = S0[:, None] * (1 + 1e-3 * np.cos(2 * (np.arange(Nphi) + 0.5) * dphi))[None, :] + 1e-4 * rng.random((Nu, Nphi))
    ref = disk64_potential(Sig)
    out = {}
    for dt, name in ((torch.float64, "fp64"), (torch.float32, "fp32")):
        ct = torch.complex128 if dt == torch.float64 else torch.complex64
        khd = torch.from_numpy(kh).to(device=f"cuda:{device}", dtype=ct)
        r32 = torch.from_numpy(R ** 1.5).to(device=f"cuda:{device}", dtype=dt)[:, None]
        sc = torch.from_numpy(-du * dphi / np.sqrt(R)).to(device=f"cuda:{device}", dtype=dt)[:, None]
        sig = torch.from_numpy(Sig).to(device=f"cuda:{device}", dtype=dt)
        pad = torch.zeros((M, Nphi), dtype=dt, device=f"cuda:{device}")
        phi = torch.empty((Nu, Nphi), dtype=dt, device=f"cuda:{device}")

        def conv():
            pad[:Nu].copy_(sig * r32)
            v = torch.fft.irfft2(torch.fft.rfft2(pad) * khd, s=(M, Nphi))
            phi.copy_(v[:Nu] * sc)

        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            for _ in range(3):
                conv()
        torch.cuda.current_stream().wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            conv()
        reps = 50
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
        for b, e in ev:
            flush.zero_()
            b.record()
            g.replay()
            e.record()
        torch.cuda.synchronize()
        ms = sum(b.elapsed_time(e) for b, e in ev) / reps
        err = float(np.max(np.abs(phi.double().cpu().numpy() - ref)) / np.max(np.abs(ref)))
        out[name] = {"ms_per_convolution": ms, "rel_err_vs_fp64_path": err}
        del g
    return out


def batched_sweep(a, device, grouped=True, ndisks=None, grids=None, tlim=None):
    """Throughput of a batched sweep: `--batch-disks` disks drawn by the sweep law (grids
    128^2..512^2, Q_min, M_d/M_*, softening/r, Gamma; seed 12345), mixed precision, advanced
    together by dg_batch (one graph launch advances every disk 64 steps; same-grid disks
    as groups, one launch per kernel, unless grouped is False).  ndisks / grids / tlim
    override the batch options (the batched 1024^2 measurement)."""
    import torch
    import diskgpu as D
    from diskgpu import sweep as S
    os.environ["DISKGPU_BATCH_GROUPS"] = "all" if grouped else "0"
    grid_list = grids or tuple(int(g) for g in a.batch_grids.split(","))
    tlim = a.batch_tlim if tlim is None else tlim
    pts = S.draw(ndisks or a.batch_disks, seed=a.batch_seed, grids=grid_list)
    params = [S.point_params(pt, "mixed", device) for pt in pts]
    with D.Batch(params) as b:
        b.init_standard()
        _, _, s0 = b.advance(0.01, steps_per_launch=64)  # captures the graph
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, _, s1 = b.advance(0.01 + tlim, steps_per_launch=64)
        el = time.perf_counter() - t0
    os.environ.pop("DISKGPU_BATCH_GROUPS", None)
    zu = float(sum(pt.N * pt.N * (int(x1) - int(x0)) for pt, x0, x1 in zip(pts, s0, s1)))
    # executed split-BF16 gravity flops of a disk step (dense products up to 512^2: 36 N^3;
    # the fused factored transforms at 1024^2)
    step_flops = {N: float(sum(p[3] for p in gravity_parts("mixed", N, N))) for N in set(pt.N for pt in pts)}
    flops = float(sum(step_flops[pt.N] * (int(x1) - int(x0)) for pt, x0, x1 in zip(pts, s0, s1)))
    grids = {}
    for pt in pts:
        grids[pt.N] = grids.get(pt.N, 0) + 1
    hbm_peak, tc_peak, kind = measured_peaks()
    hyd = 32.0 * zu / el / 1e9
    return {"value": zu / el, "unit": UNIT, "disks": len(pts), "grids": {f"{k}^2": v for k, v in sorted(grids.items())},
            "zone_updates": zu, "seconds": el, "sim_time": tlim, "grouped": grouped,
            "hydro_algorithmic_GBps": hyd, "hydro_frac_of_hbm": hyd / hbm_peak,
            "gravity_executed_TFLOPs": flops / el / 1e12, "gravity_frac_of_tensor": flops / el / 1e12 / tc_peak,
            "peak_kind": kind,
            "how": "wall clock around dg_batch_advance (graph launches of 64 steps per disk, the host reads "
                   "every disk's control block between launches); algorithmic rates over the whole job: 32 B per "
                   "zone-update for the hydro, the executed split-BF16 flops of each disk-step's gravity products "
                   "(36 N^3 for the dense products)"}


TRAFFIC_KEYS = {"hydro": "hydro", "grav_phi_fwd": "grav_phi_fwd", "grav_u": "grav_u", "grav_phi_inv": "grav_phi_inv"}


# ---------------------------------------------------------------------------------

def main():
    a = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        reference_arm(a, rank)
        return

    import numpy as np
    import torch
    import torch.distributed as dist

    import diskgpu as D

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    N = a.size
    rng = np.random.default_rng(12345 + rank)
    phase0 = float(rng.uniform(0, np.pi))
    disk = D.Disk(N, N, eps=a.eps, amp=1e-3, precision=a.precision, phase0=phase0, device=local)
    disk.init_standard()
    stream = torch.cuda.Stream()
    disk.set_stream(stream.cuda_stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    kps = disk.kernels_per_step()

    # timed iterations: one dg_run_steps call of `chunk` steps each (a CUDA graph of the
    # device-resident step loop, as dg_advance runs it), L2 flushed before every iteration;
    # exactly W warm-up steps before them, the graph recorded first
    chunk = max(1, min(a.chunk, a.steps))
    warm = max(a.warmup, 3)
    clk = ClockSampler(physical_gpu_index(local)).__enter__()
    warm_up(disk, stream, flush, warm, chunk)
    t_wait = time.time()
    while clk.proc and not clk.lines and time.time() - t_wait < 3.0:  # the sampler is running
        time.sleep(0.02)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t_wall0 = time.time()
    ms = timed_region(disk, stream, flush, a.steps, chunk)
    clk.window = (t_wall0, time.time())
    clk.__exit__(None, None, None)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    reps = [timed_region(disk, stream, flush, a.steps, chunk) for _ in range(a.repeats)]
    t_dev = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t_dev, op=dist.ReduceOp.MAX)
    ms_max = float(t_dev.item())
    disk.run_steps(0, 0.3, sync=True)  # surfaces any device-side error of the timed steps
    zones = N * N
    value = world * zones * a.steps / (ms_max * 1e-3)

    # ---- optional: per-step m = 0..8 diagnostics and the drift of the FP64 global sums ----
    drift = None
    if a.drift_steps > 0:
        disk.set_diagnostics(8, a.drift_steps + 8)
        m0, L0 = disk.conserved()
        with torch.cuda.stream(stream):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            disk.run_steps(a.drift_steps, 0.3, sync=False)
            e1.record(stream)
            torch.cuda.synchronize()
        m1, L1 = disk.conserved()
        tdg, Cdg = disk.diagnostics()
        disk.set_diagnostics(8, 0)
        drift = {"steps": a.drift_steps, "rows": int(len(tdg)), "ms_per_step_with_diagnostics":
                 e0.elapsed_time(e1) / a.drift_steps, "mass_rel_drift": (m1 - m0) / m0,
                 "angmom_rel_drift": (L1 - L0) / L0, "C0_max_dev": float(np.max(np.abs(Cdg[:, 0] - 1.0))),
                 "C2_abs_last": float(abs(Cdg[-1, 2])) if len(Cdg) else None}

    # ---- single steps with a cold L2 (flushed before each), then the per-kernel split ----
    cold_n = max(1, min(a.cold_steps, a.steps))
    with torch.cuda.stream(stream):
        evc = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(cold_n)]
        for k in range(cold_n):
            flush.zero_()
            evc[k][0].record(stream)
            disk.run_steps(1, 0.3, sync=False)
            evc[k][1].record(stream)
        torch.cuda.synchronize()
        cold_ms = sum(s.elapsed_time(e) for s, e in evc) / cold_n
        disk.profile(True)
        for k in range(cold_n):
            flush.zero_()
            disk.run_steps(1, 0.3, sync=False)
        torch.cuda.synchronize()
        prof = disk.profile_read()
        disk.profile(False)

    # ---- roofline of every kernel of the step (live CUDA-event times, cold L2) ----
    hbm_peak, tc_peak, peak_kind = measured_peaks()
    traffic = ncu_traffic(a.precision, N)
    word = 8 if a.precision == "fp64" else 4
    # read Sigma, vR, vphi, Phi; write Sigma, vR, vphi (+ the split-BF16 gravity operand,
    # 2 x 2 bytes, that the mixed hydro kernel writes for the next step's gravity)
    hyd_bytes = (7 * word + (4 if a.precision == "mixed" else 0)) * zones

    def entry(phase, kernel, bound, work, unit_kind):
        t, n = prof.get(phase, (0.0, 0))
        if not n:
            return None
        ms1 = t / n
        if unit_kind == "B":
            ach, peak, unit = work / (ms1 * 1e-3) / 1e9, hbm_peak, "GB/s"
        else:
            ach, peak, unit = work / (ms1 * 1e-3) / 1e12, tc_peak, "TFLOP/s"
        tr = traffic.get(TRAFFIC_KEYS.get(phase, ""))
        e = {"kernel": kernel, "bound": bound, "achieved": ach, "peak": peak, "unit": unit, "frac": ach / peak,
             "traffic": tr, "ms_per_launch": ms1, "share_of_step": ms1 / cold_ms,
             "peak_kind": peak_kind + (" (sustained bf16)" if unit_kind == "flop" else " (copy)")}
        e["bytes_alg_per_launch" if unit_kind == "B" else "flops_executed_per_launch"] = work
        return e

    if a.precision == "mixed":
        tuned = disk.tuning()
        form = next((f for f in ("packed", "tile", "warp") if ("hydro " + f) in tuned), "tile")
        hyd_name = {
            "packed": "fused hydro sweep (k_hydro32p: 16 x 58 tiles, TMA-staged fields, FP32x2 column pairs, "
                      "source + R sweep + phi sweep + CFL)",
            "tile": "fused hydro sweep (k_hydro32t: 16 x 58 tiles, source + R sweep + phi sweep + CFL)",
            "warp": "fused hydro sweep (k_hydro32w: warp-marching rows, source + R sweep + phi sweep + CFL)",
        }[form]
    else:
        hyd_name = "fused hydro sweep (k_hydro64: source + R sweep + phi sweep + CFL)"
    roof_all = [entry("hydro", hyd_name, "hbm", hyd_bytes, "B")]
    for ph, kern, bound, work, kind in gravity_parts(a.precision, N, N):
        e = entry(ph, kern, bound, work, kind)
        if e is not None and a.precision == "mixed":
            e["flops_fft_nominal_whole_gravity"] = 5 * (2 * N * N) * int(np.log2(2 * N * N)) * 2
        roof_all.append(e)
    roof_all = [e for e in roof_all if e is not None]
    roof = max(roof_all, key=lambda e: e["ms_per_launch"])
    share = {k: v[0] / (cold_ms * cold_n) for k, v in prof.items() if v[1]}

    # ---- end to end through the C ABI on host buffers (pinned), every step ----
    e2e = None
    if a.e2e_steps > 0:
        S, vR, vp = disk.get_state()
        hs = [torch.from_numpy(x).pin_memory() for x in (S, vR, vp)]
        arrs = [t.numpy() for t in hs]
        with torch.cuda.stream(stream):
            disk.step_host(*arrs)  # warm
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(a.e2e_steps):
                disk.step_host(*arrs)
            el = time.perf_counter() - t0
        e2e = {"value": world * zones * a.e2e_steps / el if world == 1 else None, "unit": UNIT,
               "h2d_bytes_per_step": 3 * 8 * zones, "d2h_bytes_per_step": 3 * 8 * zones + 8,
               "how": "dg_step_host per step: FP64 host state (pinned) -> device, CFL dt, gravity, hydro, "
                      "state -> host; wall clock"}
        if world > 1:
            t_e = torch.tensor([el], dtype=torch.float64, device="cuda")
            dist.all_reduce(t_e, op=dist.ReduceOp.MAX)
            e2e["value"] = world * zones * a.e2e_steps / float(t_e.item())

    # ---- end to end through the device-resident loop: host state in, dg_advance over the
    # same K steps' worth of simulated time with its mode records, final state out ----
    e2e_loop = None
    if a.e2e_steps > 0 and world == 1:
        S, vR, vp = disk.get_state()
        t_now, n_now = disk.time()
        dt_est = t_now / max(n_now, 1)
        span = dt_est * a.steps
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        disk.set_state(S, vR, vp)
        recs, t1, n1 = disk.advance(span, dtout=span / 8)
        S2, _, _ = disk.get_state()
        el = time.perf_counter() - t0
        e2e_loop = {"value": zones * n1 / el, "unit": UNIT, "steps": int(n1), "records": int(len(recs)),
                    "h2d_bytes": 3 * 8 * zones, "d2h_bytes": 3 * 8 * zones + int(recs.nbytes),
                    "how": "dg_set_state (FP64 host state) -> dg_advance over the simulated time of about K steps "
                           "with mode records every eighth of it -> dg_get_state; wall clock; the state crosses PCIe "
                           "once each way, not every step"}

    # ---- the plain FP64 path on the same disk, and a batched sweep (one rank) ----
    fp64 = batch = cufft = None
    if world == 1 and a.precision == "mixed":
        f64_steps = a.steps if a.fp64_steps is None else a.fp64_steps
        if f64_steps > 0:
            fp64 = fp64_same_disk(a, local, stream, flush, phase0, f64_steps, chunk)
            fp64["mixed_over_fp64"] = value / fp64["value"]
            if reps and fp64.get("repeats"):
                fp64["mixed_over_fp64_median_of_repeats"] = (fp64["repeats"]["median_ms_per_step"] /
                                                             spread(reps, a.steps)["median_ms_per_step"])
        if a.cufft:
            with D.Disk(N, N, eps=a.eps, precision="fp64", device=local) as d64:
                cufft = cufft_gravity(a, local, flush, d64.potential)
            grav_ms = sum(prof[k][0] / prof[k][1] for k in ("grav_phi_fwd", "grav_u", "grav_phi_inv") if prof[k][1])
            cufft["tcgen05_gravity_ms"] = grav_ms
            cufft["note"] = ("timing comparison only: cuFFT through torch.fft on the same padded "
                             f"{2 * N}x{N} convolution, graph-replayed after an L2 flush; tcgen05_gravity_ms = the "
                             "mixed step's three gravity kernels, each timed alone after an L2 flush")
        if a.batch_disks > 0:
            batch = batched_sweep(a, local, grouped=True)
            batch["ungrouped"] = batched_sweep(a, local, grouped=False)["value"]
        if a.batch1024_disks > 0:
            # the default: one graph branch per 1024^2 disk; beside it the grouped kernels
            b1k = batched_sweep(a, local, grouped=False, ndisks=a.batch1024_disks, grids=(1024,),
                                tlim=a.batch1024_tlim)
            b1k["grouped_value"] = batched_sweep(a, local, grouped=True, ndisks=a.batch1024_disks, grids=(1024,),
                                                 tlim=a.batch1024_tlim)["value"]
            if fp64 is not None and N == 1024:
                b1k["over_fp64_plain_1024"] = b1k["value"] / fp64["value"]
            batch = dict(batch or {}, batched_1024=b1k)

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_sample(N, a.eps)

    if rank == 0:
        cfg = workload(a)
        cfg.update({"precision": a.precision,
                    "timed_iteration": f"one dg_run_steps call of {chunk} steps (a CUDA graph of the "
                                       "device-resident step loop)",
                    "l2": f"flushed (256 MiB device write, outside the timed events) before every timed "
                          f"iteration of {chunk} steps; within an iteration the disk's fields stay resident "
                          "as in a production run",
                    "cold_l2_single_step": {"ms_per_step": cold_ms, "steps": cold_n,
                                            "note": "one step per timed iteration, L2 flushed before each"},
                    "stream": "caller stream via dg_set_stream", "phase_share_cold": share,
                    "kernels_per_step": kps, "autotuner": disk.tuning()})
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": warm, "ms_per_step": ms_max / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if a.precision == "fp64" else "f32 state + f64 basic state, split-bf16 DFT",
            "data": "synthetic (standard heavy disk, seeded m=2 phase)", "config": cfg,
            "roofline": roof, "roofline_all": roof_all, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": kps * a.steps, "clocks": clk.summary(),
            "repeats": spread(reps, a.steps) if reps else None, "e2e_device_loop": e2e_loop,
            "fp64_same_disk": fp64, "cufft_gravity": cufft, "batched_sweep": batch, "conservation": drift,
        }
        print(json.dumps(line))
    disk.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
