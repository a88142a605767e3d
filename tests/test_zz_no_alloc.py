"""how_tstep_noalloc: the CFL time step for callers that cannot allocate GPU
memory (a host application whose memory pool owns the device, or code under
an allocator that forbids cudaMalloc after set-up).  It takes the caller's
device state and a device slot for dt and uses only a fixed array compiled
into the library.  Checked against the context-based how_tstep on the same
state, twice in a row (the shared array keeps the previous call's contents).

Collected last on purpose: a failure here leaves every other test already run.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_DT = 1e-13   # the dt tolerance of the parity tests


def _lib_and_params(hm, n, problem, **kw):
    p = hm.make_parameters(nx=n[0], ny=n[1], nz=n[2], nt=1, tend=1.0, gam=5.0 / 3.0, cour=0.4,
                           problem=problem, **kw)
    lib = hm.lib()
    lib.how_tstep_noalloc.argtypes = [ctypes.c_void_p, ctypes.POINTER(hm.Params), ctypes.c_void_p,
                                      ctypes.c_void_p]
    lib.how_tstep_noalloc.restype = ctypes.c_int
    return lib, p


@pytest.mark.parametrize("n,problem", [((48, 40, 36), "blast3d_b"), ((128, 128, 1), "orszag_tang")])
def test_noalloc_tstep_matches_context_tstep(n, problem):
    import torch
    import how_mhd as hm

    lib, p = _lib_and_params(hm, n, problem)
    # the state after a few steps (non-trivial velocities), through the context path
    with hm.Domain(p) as dom:
        dom.init_problem()
        dom.run(0.0, 3)
        q = dom.get_state(0)
        dt_ctx = dom.tstep()
    q_dev = torch.from_numpy(q).cuda()
    dt_dev = torch.zeros(1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        dt_dev.zero_()
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc = lib.how_tstep_noalloc(ctypes.c_void_p(q_dev.data_ptr()), ctypes.byref(p),
                                   ctypes.c_void_p(dt_dev.data_ptr()), ctypes.c_void_p(stream))
        assert rc == 0, lib.how_last_error().decode()
        torch.cuda.synchronize()
        if call == 1:
            # after the first call on this device (which may place the module
            # and its fixed array), a call takes no device memory
            assert torch.cuda.mem_get_info()[0] == free_before
        dt = float(dt_dev.item())
        assert abs(dt / dt_ctx - 1.0) <= TOL_DT, (dt, dt_ctx)


def test_noalloc_rejects_oversize():
    import how_mhd as hm

    lib, p = _lib_and_params(hm, (1024, 512, 1), "uniform")
    dt = ctypes.c_double()
    rc = lib.how_tstep_noalloc(ctypes.c_void_p(1), ctypes.byref(p), ctypes.byref(dt), None)
    assert rc == -1   # HOW_ERR_ARG
    assert "HOW_NOALLOC_MAX_LINES" in lib.how_last_error().decode()
