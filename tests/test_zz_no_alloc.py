"""axj_compute_dt_noalloc: ComputeTimeStep for callers that cannot allocate device memory.

Some hosts own their device memory through something else -- a framework's caching
allocator, or a Fortran driver that passes its own device arrays -- and cannot let the
library call cudaMalloc. For them the library offers this one entry point: it takes
device arrays from the caller and keeps the scratch of its min-reduction in a fixed
array inside the library. These tests call it through the C-ABI and check it against the
handle-based axj_compute_dt on the same state: two calls in a row on successive states
(row-pitched arrays), the reference dt mode with the stale scalar T, an all-blanked grid
(dt = 100) and non-finite inputs (NaN).
"""
import ctypes as C

import numpy as np
import pytest

import axisymmetricjet_b200 as axj
from axisymmetricjet_b200 import fixtures

pytestmark = pytest.mark.gpu

REL = 1e-14  # the same per-point formulas (the handle's kernel multiplies by 1/Re where this one
             # divides: an ulp at most); the minimum is exact
PAD = 24     # caller arrays with a row pitch of Nz + PAD


def _fn():
    lib = axj.load_library()
    fn = lib.axj_compute_dt_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                   C.POINTER(axj.AxjParams), C.c_double, C.c_void_p, C.c_void_p]
    return lib, fn


class Caller:
    """Device arrays a caller owns (torch here), in pitched rows, and the call."""

    def __init__(self, c, oracle_mod, patches):
        import torch
        self.torch = torch
        self.Nz, self.Nr = c["Nz"], c["Nr"]
        self.pitch = self.Nz + PAD
        self.cuda = torch.device("cuda", 0)
        # the 1-D metrics (ComputeMetric) from the oracle, a checker-side copy
        ora = oracle_mod.Oracle(c["params"], c["zvec"], c["rvec"], c["ibval"], patches)
        dxidz, detadr, _, _ = ora.metrics()
        ora.close()
        self.dxidz = torch.tensor(np.ascontiguousarray(dxidz[0, :]), dtype=torch.float64, device=self.cuda)
        self.detadr = torch.tensor(np.ascontiguousarray(detadr[:, 0]), dtype=torch.float64, device=self.cuda)
        self.dt = torch.full((1,), -1.0, dtype=torch.float64, device=self.cuda)
        self.lib, self.fn = _fn()

    def pitched(self, a):
        a = np.asarray(a, dtype=np.float64)
        out = np.full(a.shape[:-1] + (self.pitch,), 7.5)  # padding the kernel must not read
        out[..., :self.Nz] = a
        return self.torch.tensor(out, dtype=self.torch.float64, device=self.cuda)

    def __call__(self, pv, ibval, params, stale_T=0.0):
        d_pv = self.pitched(pv)
        d_ib = self.pitched(ibval) if ibval is not None else None
        self.torch.cuda.synchronize()
        rc = self.fn(d_pv.data_ptr(), self.pitch, self.Nz, self.Nr, self.dxidz.data_ptr(), self.detadr.data_ptr(),
                     d_ib.data_ptr() if d_ib is not None else None, C.byref(params), float(stale_T),
                     self.dt.data_ptr(), None)
        assert rc == 0, self.lib.axj_last_error(None)
        self.torch.cuda.synchronize()
        return float(self.dt.item())


def _setup(c, oracle_mod):
    patches = axj.patches_from_records(c["records"], c["Nz"], c["Nr"])
    dev = axj.AxiJetSolver(c["params"], c["zvec"], c["rvec"], c["ibval"], patches)
    dev.set_state(c["pv"], c["target"])
    return dev, Caller(c, oracle_mod, patches), patches


def test_noalloc_dt_matches_handle_dt_twice(oracle_mod):
    c = fixtures.nozzle_case(dt_mode=1)  # blanked points; dt from the local temperature
    dev, call, _ = _setup(c, oracle_mod)
    for k in range(2):
        got = call(dev.get_state(), c["ibval"], c["params"])
        want = dev.compute_time_step()
        assert abs(got - want) <= REL * abs(want), (k, got, want)
        dev.rk4(want)  # the second call sees the next state
    dev.close()


def test_noalloc_reference_dt_with_stale_T(oracle_mod):
    """dt_mode = AXJ_DT_REFERENCE: the sound-speed term uses the stale module scalar T the
    caller passes (ModInputOutput.f90:405). After one step the handle holds the T of the
    last face point of stage 4; the oracle, stepped alike, gives the caller that value."""
    c = fixtures.nozzle_case(sc=True, Mj=1.5, Re=5000.0)
    dev, call, patches = _setup(c, oracle_mod)
    ora = oracle_mod.Oracle(c["params"], c["zvec"], c["rvec"], c["ibval"], patches)
    ora.set_state(c["pv"], c["target"])
    # first step: the stale T is still 0
    got = call(dev.get_state(), c["ibval"], c["params"], stale_T=0.0)
    want = dev.compute_time_step()
    assert abs(got - want) <= REL * abs(want), (got, want)
    dev.rk4(want)
    ora.rk4(want)
    stale = ora.stale_T()
    assert stale > 0.0
    got = call(dev.get_state(), c["ibval"], c["params"], stale_T=stale)
    want = dev.compute_time_step()
    assert abs(got - want) <= REL * abs(want), (got, want)
    ora.close()
    dev.close()


def test_noalloc_all_blanked_and_nonfinite(oracle_mod):
    c = fixtures.case("jet96x64", dt_mode=1)
    dev, call, _ = _setup(c, oracle_mod)
    pv = dev.get_state()
    assert call(pv, np.zeros_like(c["ibval"]), c["params"]) == 100.0
    bad = pv.copy()
    bad[4, 10, 20] = np.nan
    assert np.isnan(call(bad, c["ibval"], c["params"]))
    bad = pv.copy()
    bad[3, 30, 40] = np.inf
    assert np.isnan(call(bad, c["ibval"], c["params"]))
    # a non-finite value at a blanked point is not looked at
    ib = c["ibval"].copy()
    ib[10, 20] = 0.0
    bad = pv.copy()
    bad[4, 10, 20] = np.nan
    got = call(bad, ib, c["params"])
    assert np.isfinite(got)
    # and the scratch left by those calls does not leak into the next one
    assert call(pv, c["ibval"], c["params"]) == call(pv, None, c["params"])
    dev.close()


def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch

    lib, fn = _fn()
    small = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = axj.default_params()
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    for nz, nr in ((5000, 5000), (1 << 40, 1 << 40), (1, 1 << 62)):
        rc = fn(small.data_ptr(), nz, nz, nr, small.data_ptr(), small.data_ptr(), None, C.byref(p), 0.0,
                out.data_ptr(), None)
        assert rc == 1  # AXJ_ERR_ARG, before any device work
        assert b"scratch limit" in lib.axj_last_error(None)
