"""axj_compute_dt_noalloc: ComputeTimeStep for callers that cannot allocate device memory.

Some hosts own their device memory through something else -- a framework's caching
allocator, or a Fortran driver that passes its own device arrays -- and cannot let the
library call cudaMalloc. For them the library offers this one entry point: it takes
device arrays from the caller and keeps the scratch of its min-reduction in a fixed
array inside the library. This test calls it through the C-ABI on two calls in a row,
each on a different state, and checks the result against the handle-based
axj_compute_dt on the same state.
"""
import ctypes as C

import numpy as np
import pytest

import axisymmetricjet_b200 as axj
from axisymmetricjet_b200 import fixtures

pytestmark = pytest.mark.gpu

REL = 1e-14  # both compute the same per-point values; the minimum is exact


def _fn():
    lib = axj.load_library()
    fn = lib.axj_compute_dt_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                   C.POINTER(axj.AxjParams), C.c_double, C.c_void_p, C.c_void_p]
    return lib, fn


def test_noalloc_dt_matches_handle_dt_twice(oracle_mod):
    import torch

    c = fixtures.nozzle_case(dt_mode=1)  # blanked points; dt from the local temperature
    Nz, Nr = c["Nz"], c["Nr"]
    patches = axj.patches_from_records(c["records"], Nz, Nr)
    dev = axj.AxiJetSolver(c["params"], c["zvec"], c["rvec"], c["ibval"], patches)
    dev.set_state(c["pv"], c["target"])
    # the 1-D metrics (ComputeMetric) from the oracle, a checker-side copy
    ora = oracle_mod.Oracle(c["params"], c["zvec"], c["rvec"], c["ibval"], patches)
    dxidz, detadr, _, _ = ora.metrics()
    lib, fn = _fn()
    cuda = torch.device("cuda", 0)
    d_dxidz = torch.tensor(np.ascontiguousarray(dxidz[0, :]), dtype=torch.float64, device=cuda)
    d_detadr = torch.tensor(np.ascontiguousarray(detadr[:, 0]), dtype=torch.float64, device=cuda)
    d_ib = torch.tensor(c["ibval"], dtype=torch.float64, device=cuda)
    d_dt = torch.full((1,), -1.0, dtype=torch.float64, device=cuda)
    for call in range(2):
        d_pv = torch.tensor(dev.get_state(), dtype=torch.float64, device=cuda)
        torch.cuda.synchronize()
        rc = fn(d_pv.data_ptr(), Nz, Nz, Nr, d_dxidz.data_ptr(), d_detadr.data_ptr(), d_ib.data_ptr(),
                C.byref(c["params"]), 0.0, d_dt.data_ptr(), None)
        assert rc == 0, lib.axj_last_error(None)
        torch.cuda.synchronize()
        got = float(d_dt.item())
        want = dev.compute_time_step()
        assert abs(got - want) <= REL * abs(want), (call, got, want)
        dev.rk4(want)  # the second call sees the next state
    dev.close()


def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch

    lib, fn = _fn()
    small = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = axj.default_params()
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = fn(small.data_ptr(), 5000, 5000, 5000, small.data_ptr(), small.data_ptr(), None, C.byref(p), 0.0,
            out.data_ptr(), None)
    assert rc == 1  # AXJ_ERR_ARG, before any device work
    assert b"scratch limit" in lib.axj_last_error(None)
