"""dg_timestep_static: the CFL time step for callers that must not allocate device memory
(a memory pool or framework owns the device, or a fixed-budget loop must stay out of the
allocator).  It must agree with dg_timestep on the same state, on two calls in a row, with
nothing of its own allocated (its scratch is a static per-device array): the device's free
memory is the same before and after those calls.  The first call on a device may load the
library's device code and looks up the scratch address, so the free-memory check starts
after it.  Collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

import diskgpu as D

pytestmark = pytest.mark.gpu


def _call_static(dev_arrays, p, cfl, dt_dev, stream):
    S, vR, vp = dev_arrays
    rc = D.lib().dg_timestep_static(S.data_ptr(), vR.data_ptr(), vp.data_ptr(), p.Nu, p.Nphi, p.Rin, p.Rout,
                                    p.Kpoly, p.gamma_gas, cfl, dt_dev.data_ptr(), C.c_void_p(stream))
    assert rc == 0, D.lib().dg_status_string(rc)


def test_static_timestep_matches_dg_timestep_twice():
    import torch

    with D.Disk(96, 80, eps=0.01, amp=0.05) as d:
        d.init_standard()
        dt_dev = torch.zeros(1, dtype=torch.float64, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        S, vR, vp = d.get_state()
        warm = [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (S, vR, vp)]
        _call_static(warm, d.p, 0.3, dt_dev, stream)  # set-up call (scratch address lookup)
        torch.cuda.synchronize()
        for call in range(2):
            S, vR, vp = d.get_state()
            dev = [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (S, vR, vp)]
            torch.cuda.synchronize()
            free0 = torch.cuda.mem_get_info()[0]
            _call_static(dev, d.p, 0.3, dt_dev, stream)
            torch.cuda.synchronize()
            assert torch.cuda.mem_get_info()[0] == free0, "the call changed the device's free memory"
            got = float(dt_dev.item())
            want = d.timestep(0.3)
            assert got == pytest.approx(want, rel=1e-12), (call, got, want)
            d.step(want)  # a different state for the second call


def test_static_timestep_rejects_too_many_rows():
    import torch

    x = torch.zeros(8193 * 2, dtype=torch.float64, device="cuda")
    rc = D.lib().dg_timestep_static(x.data_ptr(), x.data_ptr(), x.data_ptr(), 8193, 2, 0.25, 1.0, 0.25, 2.0, 0.3,
                                    x.data_ptr(), None)
    assert rc == -4
