"""The C oracle's ComputeRHS (with the sensor, the bc loop and the sponges) and one RK4
step against the plain-Python restatement in tests/restatement.py, written from
ModRHS.f90, ModBC.f90, ModAxis.f90 and ModRungeKutta.f90: bit for bit."""
import numpy as np
import pytest
import restatement as rs

import axisymmetricjet_b200 as axj
from axisymmetricjet_b200 import fixtures
from axisymmetricjet_b200._ffi import NSCBC_NOSLIP_WALL, SAT_NOSLIP_WALL


def _nozzle(wall, **kw):
    return fixtures.nozzle_case(Nz=48, Nr=36, iw=12, jb=14, jt=18, wall=wall, **kw)


CASES = {
    "jet": lambda: fixtures.make_case(48, 36, 30.0, 15.0, 0.9, 1000.0),
    "jet_sc": lambda: fixtures.make_case(48, 36, 30.0, 15.0, 1.5, 5000.0, sc=True),
    "nozzle_nscbc_wall": lambda: _nozzle(NSCBC_NOSLIP_WALL),
    "nozzle_sat_wall_sc": lambda: _nozzle(SAT_NOSLIP_WALL, sc=True, Mj=1.5, Re=5000.0),
    # the reference generator's case: stretched grid, blanked lip, wall outflow (250 x 50)
    "writemesh_sc": lambda: fixtures.writemesh_case(sc=True, Re=5000.0),
    "jet_forcing": lambda: fixtures.make_case(
        48, 36, 30.0, 15.0, 0.9, 1000.0, control_forcing=1, forcing_z0=3.0, forcing_r0=0.5, forcing_lz=1.0,
        forcing_lr=0.3, forcing_mat=np.arange(25.0).reshape(5, 5) * 1e-3),
}


def _setup(oracle_mod, c):
    patches = axj.patches_from_records(c["records"], c["Nz"], c["Nr"])
    maps = axj.point_maps(patches, c["Nz"], c["Nr"], c["ibval"])
    o = oracle_mod.Oracle(c["params"], c["zvec"], c["rvec"], c["ibval"],
                          oracle_mod.patches_from_records(c["records"], c["Nz"], c["Nr"]))
    o.set_state(c["pv"], c["target"])
    args = (axj.operator_tables(), maps, o.metrics(), c["z"], c["r"], c["params"], patches)
    return o, args


def _state(c):
    """The case's state with a smooth wave on top (every term of the right-hand side
    non-trivial, the sensor active)."""
    pv = c["pv"].copy()
    zz, rr = np.meshgrid(c["z"], c["r"])
    pv[3] += 0.05 * np.sin(zz) * np.exp(-rr)
    pv[1] += 0.02 * np.cos(0.7 * zz) * rr * np.exp(-rr)
    pv[2] += 0.01 * np.sin(0.5 * zz) * rr * np.exp(-rr)
    pv[4] *= 1.0 + 0.01 * np.cos(0.3 * zz)
    return pv


@pytest.mark.parametrize("name", list(CASES))
def test_rhs_equals_the_oracle_bit_for_bit(oracle_mod, name):
    c = CASES[name]()
    o, args = _setup(oracle_mod, c)
    pv = _state(c)
    got = rs.rhs(pv, c["target"], *args)
    want = o.compute_rhs(pv)
    for e in range(5):
        bad = np.argwhere(got[e] != want[e])
        assert len(bad) == 0, (e, len(bad), [(tuple(b), got[e][tuple(b)], want[e][tuple(b)]) for b in bad[:3]])
    assert np.abs(want).max() > 0


@pytest.mark.parametrize("name", ["jet_sc", "nozzle_sat_wall_sc"])
def test_rk4_step_equals_the_oracle_bit_for_bit(oracle_mod, name):
    c = CASES[name]()
    pv = _state(c)
    c["pv"] = pv
    o, args = _setup(oracle_mod, c)
    dt = o.compute_time_step()
    o.rk4(dt)
    got = rs.rk4(pv, c["target"], dt, *args)
    assert np.array_equal(got, o.get_state())


@pytest.mark.parametrize("dt_mode", [0, 1])
def test_time_step_equals_the_oracle_bit_for_bit(oracle_mod, dt_mode):
    """Reference mode: the stale module scalar T (0 before the first right-hand side,
    then the oracle's tracked value); physical mode: the local T."""
    c = _nozzle(SAT_NOSLIP_WALL, sc=True, Mj=1.5, Re=5000.0, dt_mode=dt_mode)
    o, args = _setup(oracle_mod, c)
    blank = args[1]["blank"] == 1
    for _ in range(2):
        stale = None if dt_mode == 1 else o.stale_T()
        want = o.compute_time_step()
        assert rs.compute_time_step(o.get_state(), blank, args[2], c["params"], stale) == want
        o.rk4(want)


@pytest.mark.parametrize("name", ["jet", "nozzle_nscbc_wall"])
def test_metrics_equal_the_oracle_bit_for_bit(oracle_mod, name):
    """ComputeMetric of the coordinates and of the inverted first metrics."""
    c = CASES[name]()
    o, _ = _setup(oracle_mod, c)
    got = rs.metrics(axj.operator_tables()[0], c["z"], c["r"])
    for g, w in zip(got, o.metrics()):
        assert np.array_equal(g, w)


def test_restated_pipeline_with_restated_metrics(oracle_mod):
    """The whole second restatement with its own metrics: one RK4 step of the
    shock-capturing nozzle equals the oracle's."""
    c = CASES["nozzle_sat_wall_sc"]()
    c["pv"] = _state(c)
    o, args = _setup(oracle_mod, c)
    own = rs.metrics(args[0][0], c["z"], c["r"])
    dt = o.compute_time_step()
    o.rk4(dt)
    got = rs.rk4(c["pv"], c["target"], dt, args[0], args[1], own, *args[3:])
    assert np.array_equal(got, o.get_state())


def test_patch_creation_equals_the_library():
    """PatchCreation of the library (axj_patches_from_records) against the restatement, on
    the reference's nozzle bc file and the fixtures' layouts."""
    import os
    rec = axj.read_bc_file(os.path.join(os.path.dirname(__file__), "golden", "bc_4400x640_nozzle.dat"))
    layouts = [(rec, 4400, 640), (rec, 640, 200), (fixtures.JET_RECORDS, 96, 64),
               (fixtures.nozzle_records(20, 24, 28), 96, 64), (fixtures.writemesh_case()["records"], 250, 50)]
    for records, Nz, Nr in layouts:
        assert axj.patches_from_records(records, Nz, Nr) == rs.create_patches(records, Nz, Nr)
