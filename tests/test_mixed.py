"""Mixed-precision path (FP32 perturbation about an FP64 basic state, split-BF16 tcgen05
DFT gravity) against the FP64 oracle.

Tolerances (stated per check): the split-BF16 products carry ~2^-16 relative error per
term, so the gravity of a field agrees with the FP64 potential to <= 2e-4 relative; the
perturbation fields after 100 steps agree to <= 2e-3 of the perturbation's own size;
gamma and Omega_p from the same run agree to <= 0.5 % (the mixed path's accuracy
requirement)."""
import os

import numpy as np
import pytest

import diskgpu as D
import oracle as O
from diskgpu.analysis import fit_growth
from helpers import rel_err

pytestmark = pytest.mark.gpu


def _field(Nu, Nphi, seed=0):
    rng = np.random.default_rng(seed)
    R = np.exp(np.log(0.25) + (np.arange(Nu) + 0.5) * np.log(4.0) / Nu)
    phi = (np.arange(Nphi) + 0.5) * 2 * np.pi / Nphi
    S0 = 0.372 * np.exp(-(R - 0.45) ** 2 / 0.05)
    pert = 0.05 * np.cos(2 * phi)[None, :] + 0.02 * np.sin(3 * phi + 1)[None, :] * np.sin(7 * R)[:, None]
    return S0[:, None] * (1 + pert) + 1e-3 * rng.random((Nu, Nphi))


@pytest.mark.parametrize("Nu,Nphi", [(128, 128), (256, 256), (128, 384), (512, 256), (1024, 256), (1024, 1024),
                                     (2048, 128), (4096, 128), (128, 2048), (128, 4096), (2048, 4096),
                                     (4096, 4096)])
def test_tensor_core_potential_vs_fp64(Nu, Nphi):
    """The split-BF16 DFT convolution against the FP64 FFT potential (<= 2e-4 rel).  The
    grids reach every form: dense u and phi products (128..512), the fused transforms
    (1024^2), the four-pass factored u convolution with A = 64 and 128 (Nu = 2048, 4096),
    the dense phi products at K = 2048 and 4096, and the four-step 64 x 64 phi transforms
    (Nphi = 4096 beside a four-pass u convolution)."""
    Sig = _field(Nu, Nphi)
    ref = O.Kalnajs(Nu, Nphi, eps=0.01).potential(Sig)
    with D.Disk(Nu, Nphi, eps=0.01, precision="mixed") as d:
        got = d.potential(Sig)
    assert rel_err(got, ref) < 2e-4
    # the non-axisymmetric part alone (what the mixed step actually convolves)
    pert = Sig - Sig.mean(axis=1, keepdims=True)
    refp = O.Kalnajs(Nu, Nphi, eps=0.01).potential(pert)
    with D.Disk(Nu, Nphi, eps=0.01, precision="mixed") as d:
        gotp = d.potential(pert)
    assert rel_err(gotp, refp) < 2e-4


@pytest.mark.parametrize("Nu,Nphi", [(256, 256), (512, 384), (2048, 128), (4096, 4096)])
def test_persistent_products_match_tile_products(Nu, Nphi, monkeypatch):
    """Every gravity product on the persistent warp-specialised kernel (DISKGPU_STAGES=8 in
    every slot, and 16: its 128 x 256 tiles where N is a multiple of 256; products whose N
    is not a multiple of 128 stay on the tile kernel) against
    the tile kernel (stages by K): the same contractions in the same K order, so the
    potentials agree to FP32 round-off, and both meet the FP64 potential to 2e-4.  The grids
    reach the dense products, the four-pass factored u convolution and the four-step phi
    transforms (whose first forward and last inverse passes load blocked operands)."""
    Sig = _field(Nu, Nphi)
    out = {}
    for stages in ("0,0,0,0,0,0", "8,8,8,8,8,8", "16,16,16,16,16,16"):
        monkeypatch.setenv("DISKGPU_STAGES", stages)
        with D.Disk(Nu, Nphi, eps=0.01, precision="mixed") as d:
            d.init_standard()  # applies the fixed stages (the tuner runs on the first state)
            assert "gravity stages fixed " + stages.replace(",", " ") in d.tuning()
            out[stages] = d.potential(Sig)
    ref = O.Kalnajs(Nu, Nphi, eps=0.01).potential(Sig)
    tile = out["0,0,0,0,0,0"]
    for pers in (out["8,8,8,8,8,8"], out["16,16,16,16,16,16"]):
        assert rel_err(pers, ref) < 2e-4
        assert rel_err(pers, tile) < 1e-6, rel_err(pers, tile)


def test_state_roundtrip_mixed():
    with D.Disk(128, 128, eps=0.01, precision="mixed") as d:
        d.init_standard()
        S, vR, vp = d.get_state()
        ref = O.Disk(Nu=128, Nphi=128, eps=0.01)
        Sr, vRr, vpr = ref.hyd.state()
        # the perturbation (amp 1e-3 of Sigma0) survives FP32 storage to ~1e-7 of itself
        pr = Sr - Sr.mean(axis=1, keepdims=True)
        assert np.max(np.abs((S - Sr))) <= 1e-6 * np.max(np.abs(pr))
        assert rel_err(vp, vpr) < 1e-12
        m, L = d.conserved()
        assert m == pytest.approx(ref.mD, rel=1e-12)


@pytest.mark.parametrize("N,steps", [(256, 100), (128, 200), (1024, 50)])
def test_mixed_vs_fp64_after_steps(N, steps):
    """Mixed-path fields after the given steps (dt from the oracle's CFL, checked against the
    device's) against the FP64 oracle stepped in lockstep; 1024^2 runs the fused transforms
    and the packed hydro."""
    ref = O.Disk(Nu=N, Nphi=N, eps=0.005, amp=1e-3, nthreads=os.cpu_count() or 8)
    S0 = ref.hyd.get("Sig").mean(axis=1, keepdims=True)
    with D.Disk(N, N, eps=0.005, amp=1e-3, precision="mixed") as d:
        d.init_standard()
        for _ in range(steps):
            dt_ref = ref.step()
            dt = d.timestep(0.3)
            assert abs(dt - dt_ref) <= 1e-5 * dt_ref
            d.step(dt_ref)
        S, vR, vp = d.get_state()
    Sr, vRr, vpr = ref.hyd.state()
    # errors measured against the size of the perturbation itself
    assert np.max(np.abs(S - Sr)) <= 2e-3 * np.max(np.abs(Sr - S0))
    assert np.max(np.abs(vR - vRr)) <= 2e-3 * np.max(np.abs(vRr))
    vp0 = vpr.mean(axis=1, keepdims=True)
    assert np.max(np.abs(vp - vpr)) <= 2e-3 * np.max(np.abs(vpr - vp0)) + 1e-9


@pytest.mark.parametrize("Nu,Nphi,steps,vtol", [(256, 384, 80, 2e-3), (384, 256, 80, 2e-3), (128, 512, 100, 2e-3),
                                                (512, 128, 80, 2e-3), (1024, 2048, 30, 2e-3), (2048, 1024, 16, 1e-2)])
def test_mixed_nonsquare_vs_fp64_after_steps(Nu, Nphi, steps, vtol):
    """Non-square grids in lockstep with the FP64 oracle: the hydro tiles' partial last
    column tile and periodic wrap at other widths than the radial extent, rectangular dense
    products, the fused u convolution beside the dense phi products (1024 x 2048) and the
    four-pass u convolution beside them (2048 x 1024).  Sigma within 2e-3 of the
    perturbation's size everywhere; the velocities within 2e-3, except at 2048 x 1024,
    where after 16 steps the velocity perturbation is still young and the split-BF16
    potential's error (within the 2e-4 of the potential tests) is differenced over twice
    the 1024^2 radial resolution: 1e-2 there (measured 4e-3)."""
    ref = O.Disk(Nu=Nu, Nphi=Nphi, eps=0.005, amp=1e-3, nthreads=os.cpu_count() or 8)
    S0 = ref.hyd.get("Sig").mean(axis=1, keepdims=True)
    with D.Disk(Nu, Nphi, eps=0.005, amp=1e-3, precision="mixed") as d:
        d.init_standard()
        for _ in range(steps):
            dt_ref = ref.step()
            dt = d.timestep(0.3)
            assert abs(dt - dt_ref) <= 1e-5 * dt_ref
            d.step(dt_ref)
        S, vR, vp = d.get_state()
    Sr, vRr, vpr = ref.hyd.state()
    assert np.max(np.abs(S - Sr)) <= 2e-3 * np.max(np.abs(Sr - S0))
    assert np.max(np.abs(vR - vRr)) <= vtol * np.max(np.abs(vRr))
    vp0 = vpr.mean(axis=1, keepdims=True)
    assert np.max(np.abs(vp - vpr)) <= vtol * np.max(np.abs(vpr - vp0)) + 1e-9


@pytest.mark.parametrize("Nu,Nphi", [(128, 128), (256, 384)])
def test_mixed_caller_forces_and_no_gravity_vs_oracle(Nu, Nphi):
    """The mixed hydro's other two force forms against the oracle stepped in lockstep:
    30 steps with the caller's forces (DiskHydro::step(dt, gR, gp) through dg_step_forces:
    the oracle's own Kalnajs forces of its current state, passed as FP64 arrays), then 30
    with no force at all (DiskHydro::step(dt)).  The perturbation fields within 2e-3 of
    their size."""
    ref = O.Disk(Nu=Nu, Nphi=Nphi, eps=0.01, amp=1e-2, nthreads=os.cpu_count() or 8)
    S0 = ref.hyd.get("Sig").mean(axis=1, keepdims=True)
    with D.Disk(Nu, Nphi, eps=0.01, amp=1e-2, precision="mixed") as d:
        d.init_standard()
        for _ in range(30):
            dt = ref.hyd.timestep(0.3)
            gR, gp = ref.gravity()
            ref.hyd.step(dt, gR, gp)
            d.step_forces(dt, gR, gp)
        for _ in range(30):
            dt = ref.hyd.timestep(0.3)
            ref.hyd.step(dt)
            d.step_forces(dt)
        S, vR, vp = d.get_state()
    Sr, vRr, vpr = ref.hyd.state()
    assert np.max(np.abs(S - Sr)) <= 2e-3 * np.max(np.abs(Sr - S0)), np.max(np.abs(S - Sr)) / np.max(np.abs(Sr - S0))
    assert np.max(np.abs(vR - vRr)) <= 2e-3 * np.max(np.abs(vRr)), np.max(np.abs(vR - vRr)) / np.max(np.abs(vRr))
    vp0 = vpr.mean(axis=1, keepdims=True)
    assert np.max(np.abs(vp - vpr)) <= 2e-3 * np.max(np.abs(vpr - vp0)) + 1e-9


def test_growth_rate_and_pattern_speed_match_fp64():
    """gamma, Omega_p of the m=2 mode from mixed and FP64 runs of the same disk (<= 0.5 %)."""
    kw = dict(eps=0.01, amp=1e-3)
    out = {}
    for prec in ("fp64", "mixed"):
        with D.Disk(128, 128, precision=prec, **kw) as d:
            d.init_standard()
            rec, t, n = d.advance(6.0)
        out[prec] = fit_growth(rec[:, 0], rec[:, 2], rec[:, 3], tmin=2.0, tmax=6.0)
    g64, w64, _ = out["fp64"]
    gmx, wmx, _ = out["mixed"]
    assert g64 > 0.2
    assert abs(gmx - g64) <= 5e-3 * abs(g64)
    assert abs(wmx - w64) <= 5e-3 * abs(w64)


def test_growth_and_saturation_match_fp64_1024():
    """The 1024^2 disk of the headline workload (eps 0.005, m = 2 seed 1e-3) run through
    saturation (t = 20) on both paths; the mixed one runs every fused kernel, the packed
    hydro and the row-tile hand-over.  Linear phase: gamma and Omega_p within 0.5 % of the
    FP64 path's; saturated |C2|/|C0| within 2 %."""
    from diskgpu.analysis import linear_phase, saturated_phase
    kw = dict(eps=0.005, amp=1e-3)
    out = {}
    for prec in ("fp64", "mixed"):
        with D.Disk(1024, 1024, precision=prec, **kw) as d:
            d.init_standard()
            rec, t, n = d.advance(20.0)
        out[prec] = (linear_phase(*rec.T), saturated_phase(*rec.T))
    (g64, w64, _), (r64, _, _) = out["fp64"]
    (gmx, wmx, _), (rmx, _, _) = out["mixed"]
    assert g64 > 0.2 and r64 > 0.15
    assert abs(gmx - g64) <= 5e-3 * abs(g64), (gmx, g64)
    assert abs(wmx - w64) <= 5e-3 * abs(w64), (wmx, w64)
    assert abs(rmx - r64) <= 0.02 * r64, (rmx, r64)


def test_mixed_vs_fp64_4096_after_steps():
    """The 4096^2 disk (four-pass u convolution with A = 128, four-step 64 x 64 phi
    transforms, packed hydro) 12 steps in lockstep with the FP64 oracle: sigma within 2e-3
    of the perturbation's size, as at the smaller grids.  The velocity perturbations are held
    to 5e-2 of their size: after 12 steps at this resolution they are still ~3e-7, and the
    split-BF16 potential's relative error (<= 2e-4 of the perturbation's potential, the
    bound of the potential tests) differenced over du = ln 4 / 4096 and dphi = 2 pi / 4096
    gives force errors of a few percent of the forces that have built them so far; the
    ratio does not grow with the steps while the forces are steady."""
    N, steps = 4096, 12
    ref = O.Disk(Nu=N, Nphi=N, eps=0.005, amp=1e-3, nthreads=os.cpu_count() or 8)
    S0 = ref.hyd.get("Sig").mean(axis=1, keepdims=True)
    with D.Disk(N, N, eps=0.005, amp=1e-3, precision="mixed") as d:
        d.init_standard()
        for _ in range(steps):
            dt_ref = ref.step()
            dt = d.timestep(0.3)
            assert abs(dt - dt_ref) <= 1e-5 * dt_ref
            d.step(dt_ref)
        S, vR, vp = d.get_state()
    Sr, vRr, vpr = ref.hyd.state()
    assert np.max(np.abs(S - Sr)) <= 2e-3 * np.max(np.abs(Sr - S0))
    vp0 = vpr.mean(axis=1, keepdims=True)
    assert np.max(np.abs(vp - vpr)) <= 5e-2 * np.max(np.abs(vpr - vp0)) + 1e-9
    assert np.max(np.abs(vR - vRr)) <= 5e-2 * np.max(np.abs(vRr))


def test_4096_disk_conservation_and_diagnostics():
    """The large single disk (4096^2, gravity on the 8192 x 4096 padded grid, mixed
    precision) for 300 device steps with the per-step m = 0..8 diagnostic on: one ring row
    per step, C_0 = mass / m_D stays 1, and the FP64 global sums drift by no more than
    round-off (mass) and the scheme's small truncation error (angular momentum; the
    reference's transport is not exactly angular-momentum conserving)."""
    with D.Disk(4096, 4096, eps=0.005, amp=1e-3, precision="mixed") as d:
        d.init_standard()
        d.set_diagnostics(8, 1024)
        m0, L0 = d.conserved()
        d.run_steps(300, 0.3)
        m1, L1 = d.conserved()
        t, C = d.diagnostics()
    assert len(t) == 300 and C.shape == (300, 9)
    assert np.all(np.diff(t) > 0)
    assert np.max(np.abs(C[:, 0] - 1.0)) < 1e-9
    assert abs(C[-1, 2]) > 4e-4  # the m = 2 seed (|C2| = amp / 2 = 5e-4) is carried
    assert abs(m1 - m0) <= 1e-11 * m0, (m1 - m0) / m0
    assert abs(L1 - L0) <= 1e-8 * abs(L0), (L1 - L0) / L0


def test_mixed_requires_multiple_of_128():
    with pytest.raises(D.DiskGPUError) as e:
        D.Disk(96, 128, precision="mixed")
    assert e.value.code == -4


def test_mixed_nonfinite_reported():
    with D.Disk(128, 128, precision="mixed") as d:
        d.init_standard()
        S, vR, vp = d.get_state()
        vR[3, 3] = np.inf
        d.set_state(S, vR, vp)
        with pytest.raises(D.DiskGPUError) as e:
            d.run_steps(3)
        assert e.value.code == -3


@pytest.mark.parametrize("form", ["tile", "packed"])
@pytest.mark.parametrize("N,steps,rec", [(256, 40, False), (1024, 12, False), (128, 30, True), (384, 20, False)])
def test_tiled_hydro_matches_warp_form(N, steps, rec, form, monkeypatch):
    """The tiled hydro kernel, its packed two-column form (DISKGPU_HYDRO32=tile / packed)
    and the warp-marching kernel (DISKGPU_HYDRO32=warp) compute the same step with the same
    expressions; they differ only in how the compiler contracts them into FMAs, which the
    near-cancellation of the radial force amplifies.  States agree to <= 1e-4 of the
    perturbation's size after the given steps (an indexing or halo error shows up at O(1)),
    dt and mode records to 1e-6.  384 is not a multiple of either tile width, so the last
    column of tiles is partial."""
    out = []
    for kind in (form, "warp"):
        monkeypatch.setenv("DISKGPU_HYDRO32", kind)
        with D.Disk(N, N, eps=0.005, amp=1e-2, precision="mixed") as d:
            d.init_standard()
            S0 = d.get_state()[0].mean(axis=1, keepdims=True)
            if rec:
                recs, t, n = d.advance(0.02, dtout=0.005)
            else:
                d.run_steps(steps, 0.3)
                recs = None
            out.append((d.get_state(), d.time(), recs, S0))
    (Sa, vRa, vpa), (ta, na), ra, S0 = out[0]
    (Sb, vRb, vpb), (tb, nb), rb, _ = out[1]
    assert na == nb and ta == pytest.approx(tb, rel=1e-6)
    vp0 = vpb.mean(axis=1, keepdims=True)
    for a, b, scale in ((Sa, Sb, np.max(np.abs(Sb - S0))), (vRa, vRb, np.max(np.abs(vRb))),
                        (vpa, vpb, np.max(np.abs(vpb - vp0)))):
        d = np.abs(a - b)
        where = np.unravel_index(np.argmax(d), d.shape)
        assert d.max() <= 1e-4 * scale + 1e-12, (d.max() / scale, where)
    if rec:
        assert len(ra) == len(rb) and len(ra) >= 3
        np.testing.assert_allclose(ra[:, 1:3], rb[:, 1:3], rtol=1e-6)


def test_autotuner_reports_its_choice(monkeypatch):
    """The autotuner runs at the first state upload, leaves the state and dt untouched, and
    says what it chose; DISKGPU_TUNE=0 keeps the defaults; a second disk of the same grid
    reuses the cached choice."""
    monkeypatch.delenv("DISKGPU_HYDRO32", raising=False)
    with D.Disk(256, 512, eps=0.005, amp=1e-3, precision="mixed") as a:
        a.init_standard()
        info = a.tuning()
        assert "hydro" in info and "gravity" in info and "cached" not in info
        dt_tuned = a.timestep(0.3)
        S_tuned = a.get_state()[0]
    with D.Disk(256, 512, eps=0.005, amp=1e-3, precision="mixed") as b:
        b.init_standard()
        assert b.tuning().endswith("(cached)")
    monkeypatch.setenv("DISKGPU_TUNE", "0")
    with D.Disk(256, 512, eps=0.005, amp=1e-3, precision="mixed") as c:
        c.init_standard()
        assert c.tuning().startswith("tuning off")
        assert c.timestep(0.3) == dt_tuned
        np.testing.assert_array_equal(c.get_state()[0], S_tuned)


def test_row_tile_handover_is_bit_identical(monkeypatch):
    """The row-tile hand-over between a step's hydro kernel and the next step's phi
    transform (on by default at 1024^2) changes only when kernels may start, never what
    they compute: the state after graph-launched steps, a caller-forces step and single
    steps is bit-for-bit the one with the hand-over off (DISKGPU_ROWSYNC=0)."""
    monkeypatch.delenv("DISKGPU_HYDRO32", raising=False)
    out = []
    for rs in ("1", "0"):
        monkeypatch.setenv("DISKGPU_ROWSYNC", rs)
        with D.Disk(1024, 1024, eps=0.005, amp=1e-2, precision="mixed") as d:
            d.init_standard()
            d.run_steps(40, 0.3)
            dt = d.timestep(0.3)
            d.step_forces(dt)        # hydro with the disk's own gravity switched off
            d.step(dt)               # single self-gravity steps right after it
            d.step(dt)
            d.run_steps(24, 0.3)
            out.append((d.get_state(), d.time()))
    (a, ta), (b, tb) = out
    assert ta == tb
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


def test_rowtile_wait_timeout_is_reported_and_handle_recovers(monkeypatch):
    """Failure detection without a GPU fault: DISKGPU_TEST_ROWTILE_STALL=<tile row> makes one
    row-tile counter stay above zero after the first step's hydro finished, so the second
    step's phi transform gives up its bounded wait (~1 s of SM clock; its own TMA copies are
    valid and are drained before it exits) and raises the timeout status.  The host returns
    DG_ERR_TIMEOUT; a new state clears the status and the counters, and the same handle then
    steps bit-identically to a fresh one."""
    import time
    monkeypatch.setenv("DISKGPU_TUNE", "0")
    monkeypatch.delenv("DISKGPU_HYDRO32", raising=False)
    monkeypatch.delenv("DISKGPU_ROWSYNC", raising=False)
    monkeypatch.setenv("DISKGPU_TEST_ROWTILE_STALL", "20")
    with D.Disk(1024, 1024, eps=0.005, amp=1e-3, precision="mixed") as d:
        d.init_standard()
        S, vR, vp = d.get_state()
        t0 = time.time()
        with pytest.raises(D.DiskGPUError) as e:
            d.run_steps(4, 0.3)
        assert e.value.code == -6, e.value
        assert time.time() - t0 < 30
        d.set_state(S, vR, vp)
        d.run_steps(4, 0.3)
        got = d.get_state()
    monkeypatch.delenv("DISKGPU_TEST_ROWTILE_STALL")
    with D.Disk(1024, 1024, eps=0.005, amp=1e-3, precision="mixed") as f:
        f.set_state(S, vR, vp)
        f.run_steps(4, 0.3)
        want = f.get_state()
    for x, y in zip(got, want):
        np.testing.assert_array_equal(x, y)


def test_capture_graph_up_front_changes_nothing(monkeypatch):
    """dg_capture_graph records the 64-step graph without running it: stepping afterwards
    (single steps, then graph launches, with the row-tile hand-over at 1024^2) gives the
    state bit for bit that the same steps give with the graph recorded on first use."""
    monkeypatch.delenv("DISKGPU_ROWSYNC", raising=False)
    out = []
    for pre in (True, False):
        with D.Disk(1024, 1024, eps=0.005, amp=1e-2, precision="mixed") as d:
            d.init_standard()
            if pre:
                d.capture_graph()
            d.run_steps(6, 0.3)
            d.run_steps(128, 0.3)
            d.run_steps(3, 0.3)
            out.append((d.get_state(), d.time()))
    (a, ta), (b, tb) = out
    assert ta == tb
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_advance_with_record_callback_matches_advance(prec):
    """dg_advance_cb hands over the same records, in order, as dg_advance collects: the
    same times and step counts, the records of one run exactly as the callback saw them,
    and those of two runs to 1e-12 (each CTA folds its share of the mode sums with an FP64
    atomic add, so the summation order, and the last bits, vary between runs)."""
    runs = []
    for cb in (False, True):
        seen = []
        with D.Disk(128, 128, eps=0.01, amp=1e-3, precision=prec) as d:
            d.init_standard()
            rec, t, n = d.advance(3.0, on_record=(lambda *r: seen.append(r)) if cb else None)
        runs.append((rec, t, n))
        if cb:
            np.testing.assert_array_equal(np.array(seen), rec)
    np.testing.assert_allclose(runs[0][0], runs[1][0], rtol=1e-10, atol=1e-13)
    assert runs[0][1:] == runs[1][1:]
