"""Failure detection through the C-ABI (ModInputOutput.f90:424-429 stops the reference on a
time-step blow-up; the library returns a status instead and never stops the process).

Every failure here is made on the host or by a wait limit, never by a device fault:
* a NaN written into the host state before axj_set_state: the dt kernel or the last
  stage's finiteness check reports AXJ_ERR_NONFINITE;
* a grid whose every point is blanked: ComputeTimeStep's minimum stays at its initial 100,
  which the reference stops on ("Time step blow up"), reported as AXJ_ERR_DT_BLOWUP;
* the kernels' bounded TMA waits given a limit of zero polls: every wait gives up, the
  kernels wait (bounded) for their transfers in flight, flag the timeout and return; the
  step reports AXJ_ERR_TIMEOUT, and the same handle, given its state again with the
  default limit, steps exactly as a fresh handle does (the context stays usable).
"""
import numpy as np
import pytest

import axisymmetricjet_b200 as axj
from axisymmetricjet_b200 import fixtures

pytestmark = pytest.mark.gpu

NONFINITE, DT_BLOWUP, TIMEOUT = 3, 4, 5


def solver(c):
    patches = axj.patches_from_records(c["records"], c["Nz"], c["Nr"])
    return axj.AxiJetSolver(c["params"], c["zvec"], c["rvec"], c["ibval"], patches)


def test_nan_temperature_is_reported_by_the_time_step():
    c = fixtures.case("jet96x64sc")
    pv = c["pv"].copy()
    pv[4, 20, 30] = np.nan
    with solver(c) as s:
        s.set_state(pv, c["target"])
        with pytest.raises(axj.AxjError) as e:
            s.compute_time_step()
        assert e.value.code == NONFINITE


def test_nan_swirl_is_reported_by_the_step():
    """V_theta does not enter ComputeTimeStep: the step's finiteness check catches it."""
    c = fixtures.case("jet96x64sc")
    pv = c["pv"].copy()
    pv[2, 20, 30] = np.nan
    with solver(c) as s:
        s.set_state(pv, c["target"])
        dt = s.compute_time_step()
        assert np.isfinite(dt)
        with pytest.raises(axj.AxjError) as e:
            s.rk4(dt)
        assert e.value.code == NONFINITE
        # a finite state clears the flags
        s.set_state(c["pv"], c["target"])
        s.rk4(s.compute_time_step())
        assert np.isfinite(s.get_state()).all()


def test_all_blanked_grid_is_a_time_step_blow_up(oracle_mod):
    c = fixtures.case("jet96x64")
    c["ibval"] = np.zeros_like(c["ibval"])
    with solver(c) as s:
        s.set_state(c["pv"], c["target"])
        with pytest.raises(axj.AxjError) as e:
            s.compute_time_step()
        assert e.value.code == DT_BLOWUP
    o = oracle_mod.Oracle(c["params"], c["zvec"], c["rvec"], c["ibval"],
                          oracle_mod.patches_from_records(c["records"], c["Nz"], c["Nr"]))
    o.set_state(c["pv"], c["target"])
    with pytest.raises(RuntimeError):
        o.compute_time_step()


@pytest.mark.parametrize("name", ["jet96x64sc", "nozzle_sc"])
def test_wait_timeout_is_reported_and_the_context_stays_usable(name):
    """Physical dt, so that the restarted handle's dt does not depend on the stale scalar T
    a step may have left behind."""
    if name == "jet96x64sc":
        c = fixtures.case("jet96x64sc", dt_mode=1)
    else:
        c = fixtures.nozzle_case(sc=True, Mj=1.5, Re=5000.0, dt_mode=1)
    fresh = solver(c)
    fresh.set_state(c["pv"], c["target"])
    dt = fresh.compute_time_step()
    fresh.rk4(dt)
    want = fresh.get_state()
    fresh.close()
    with solver(c) as s:
        s.set_state(c["pv"], c["target"])
        assert s.compute_time_step() == dt
        s.set_wait_limit(0)
        try:
            with pytest.raises(axj.AxjError) as e:
                s.rk4(dt)
            assert e.value.code == TIMEOUT
        finally:
            s.set_wait_limit(-1)
        s.set_state(c["pv"], c["target"])
        assert s.compute_time_step() == dt
        s.rk4(dt)
        np.testing.assert_array_equal(s.get_state(), want)


def test_batch_wait_timeout_is_reported_and_the_batch_recovers():
    """The batched kernels share the bounded waits: with the limit at zero a batch step
    reports AXJ_ERR_TIMEOUT; with the default limit and the states set again, the batch steps
    as the same instances do one by one (physical dt, FP64)."""
    cases = fixtures.batch_instances(3, seed=5, nz_range=(256, 384), nr_range=(96, 128), dt_mode=1)
    singles, batched = [], []
    for c in cases:
        for lst in (singles, batched):
            s = solver(c)
            s.set_state(c["pv"], c["target"])
            lst.append(s)
    b = axj.AxjBatch(batched)
    batched[0].set_wait_limit(0)
    try:
        with pytest.raises(axj.AxjError) as e:
            b.run(1)
        assert e.value.code == TIMEOUT
    finally:
        batched[0].set_wait_limit(-1)
    for s, c in zip(batched, cases):
        s.set_state(c["pv"], c["target"])
    b.run(2)
    for s in singles:
        s.run(2)
    for s, t in zip(singles, batched):
        a, r = t.get_state(), s.get_state()
        errs = [np.abs(a[f] - r[f]).max() / max(np.abs(r[f]).max(), 1e-300) for f in range(5)]
        assert max(errs) <= 1e-12, errs
    b.close()
    for s in singles + batched:
        s.close()
