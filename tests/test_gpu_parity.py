"""Parity of the CUDA path (libaxj.so through the C-ABI) against the CPU oracle.

Tolerances: the FP64 device path differs from the oracle only by FMA contraction and
libm ulps, so per-routine, per-RHS and per-RK4-step results must agree to 1e-12
relative (max error over a field divided by the field's max magnitude; the three
velocity components share one scale, the largest of their magnitudes: V_r and V_theta
start at zero, so their right-hand sides are differences of terms of the V_z equation's
size, and the oracle built with and without FMA contraction differs by 6.6e-12 of the
V_r right-hand side's own maximum on the generator's case, 1.1e-14 on the shared scale).
"""
import os

import numpy as np
import pytest

import axisymmetricjet_b200 as axj
from axisymmetricjet_b200 import fixtures
from axisymmetricjet_b200._ffi import NSCBC_NOSLIP_WALL, SAT_NOSLIP_WALL

pytestmark = pytest.mark.gpu

REL = 1e-12


def relerr(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    scale = np.abs(b).max()
    return np.abs(a - b).max() / (scale if scale > 0 else 1.0)


def field_relerr(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    vscale = max(np.abs(b[k]).max() for k in (1, 2, 3))
    out = []
    for k in range(a.shape[0]):
        scale = vscale if k in (1, 2, 3) else np.abs(b[k]).max()
        out.append(np.abs(a[k] - b[k]).max() / (scale if scale > 0 else 1.0))
    return out


CASES = {
    "jet": lambda: fixtures.case("jet96x64"),
    "jet_sc": lambda: fixtures.case("jet96x64sc"),
    "nozzle_nscbc_wall": lambda: fixtures.nozzle_case(wall=NSCBC_NOSLIP_WALL),
    "nozzle_sat_wall_sc": lambda: fixtures.nozzle_case(wall=SAT_NOSLIP_WALL, sc=True, Mj=1.5, Re=5000.0),
    "jet_forcing_physdt": lambda: fixtures.case(
        "jet96x64", control_forcing=1, forcing_z0=3.0, forcing_r0=0.5, forcing_lz=1.0, forcing_lr=0.3,
        forcing_mat=np.arange(25.0).reshape(5, 5) * 1e-3, dt_mode=1),
    "jet_ragged": lambda: fixtures.make_case(77, 45, 30.0, 15.0, 0.9, 1000.0),
    # the reference generator's case: stretched z and r, blanked lip, NSCBC wall outflow
    "writemesh": lambda: fixtures.writemesh_case(),
    "writemesh_sc": lambda: fixtures.writemesh_case(sc=True, Re=5000.0),
    # harmonic inflow forcing (control_forcing = 2), the batched instances' forcing
    "jet_harmonic": lambda: fixtures.case(
        "jet96x64", control_forcing=2, forcing_z0=1.0, forcing_r0=0.5, forcing_lz=0.5, forcing_lr=0.2,
        harmonic_amp=0.018, harmonic_st=0.4, harmonic_uj=0.9),
}


def pair(c, oracle_mod):
    gp = axj.patches_from_records(c["records"], c["Nz"], c["Nr"])
    op = oracle_mod.patches_from_records(c["records"], c["Nz"], c["Nr"])
    assert gp == op
    dev = axj.AxiJetSolver(c["params"], c["zvec"], c["rvec"], c["ibval"], gp)
    ora = oracle_mod.Oracle(c["params"], c["zvec"], c["rvec"], c["ibval"], op)
    dev.set_state(c["pv"], c["target"])
    ora.set_state(c["pv"], c["target"])
    return dev, ora


@pytest.mark.parametrize("name", ["nozzle_nscbc_wall", "jet_ragged", "writemesh"])
def test_operators(oracle_mod, name):
    c = CASES[name]()
    dev, ora = pair(c, oracle_mod)
    rng = np.random.default_rng(7)
    var = rng.standard_normal((c["Nr"], c["Nz"]))
    first = rng.standard_normal((c["Nr"], c["Nz"]))
    for dirn in (1, 2):
        assert relerr(dev.deriv1(var, dirn), ora.deriv1(var, dirn)) < REL
        assert relerr(dev.deriv2(var, dirn, first), ora.deriv2(var, dirn, first)) < REL
        prior = rng.standard_normal((c["Nr"], c["Nz"]))
        assert relerr(dev.tgfilter(var, dirn, prior), ora.tgfilter(var, dirn, prior)) < REL
    prior = rng.standard_normal((c["Nr"], c["Nz"]))
    assert relerr(dev.tgfilter(None, 1, prior, inplace=True), ora.tgfilter(None, 1, prior, inplace=True)) < REL


@pytest.mark.parametrize("name", list(CASES))
def test_rhs(oracle_mod, name):
    c = CASES[name]()
    dev, ora = pair(c, oracle_mod)
    rd = dev.compute_rhs(c["pv"])
    ro = ora.compute_rhs(c["pv"])
    errs = field_relerr(rd, ro)
    assert max(errs) < REL, errs


# The sensor's outputs are fourth differences of smooth fields: sums that cancel to a
# small remainder, and the interior tiles form them as one 9-point stencil (the square
# of the centred SBP2 row) rather than two 5-point passes. On the generator's case, whose
# initial field is smooth everywhere, the oracle built with and without FMA contraction
# already differs by 1.6e-12 of the largest output (1e-14 on the jet), so its tolerance
# is ten times wider; a wrong stencil row or closure shows as an O(1) error.
SENSOR_REL = {"jet_sc": 1e-11, "nozzle_sat_wall_sc": 1e-11, "writemesh_sc": 1e-10}


@pytest.mark.parametrize("name", list(SENSOR_REL))
def test_sensor(oracle_mod, name):
    c = CASES[name]()
    dev, ora = pair(c, oracle_mod)
    errs = [relerr(a, b) for a, b in zip(dev.sensor(c["pv"]), ora.sensor(c["pv"]))]
    assert max(errs) < SENSOR_REL[name], errs


@pytest.mark.parametrize("name", list(CASES))
def test_rk4_steps(oracle_mod, name):
    c = CASES[name]()
    dev, ora = pair(c, oracle_mod)
    for step in range(3):
        dd = dev.compute_time_step()
        do = ora.compute_time_step()
        assert abs(dd - do) <= 1e-14 * abs(do), (step, dd, do)
        dev.rk4(do)
        ora.rk4(do)
        errs = field_relerr(dev.get_state(), ora.get_state())
        assert max(errs) < REL, (step, errs)
    assert dev.get_time()[0] == ora.get_time()[0] == 3
    assert abs(dev.get_time()[1] - ora.get_time()[1]) <= 1e-15


@pytest.mark.parametrize("name", ["jet_sc", "jet_harmonic"])
def test_graph_run_equals_stepping(oracle_mod, name):
    c = CASES[name]()
    dev, ora = pair(c, oracle_mod)
    dev2, _ = pair(c, oracle_mod)
    dlast = dev.run(5)
    for _ in range(5):
        d = dev2.compute_time_step()
        dev2.rk4(d)
    assert dlast == d
    np.testing.assert_array_equal(dev.get_state(), dev2.get_state())
    it, t = dev.get_time()
    it2, t2 = dev2.get_time()
    assert it == it2 == 5 and t == t2


def test_run_output_callback(oracle_mod):
    c = CASES["jet"]()
    dev, _ = pair(c, oracle_mod)
    seen = []
    dev.run(6, out_every=2, callback=lambda it, t, pv: seen.append((it, t, pv[0, 3, 3])))
    assert [s[0] for s in seen] == [2, 4, 6]
    assert seen[-1][1] == dev.get_time()[1]


def test_run_outputs_equal_the_stepped_states():
    """The outputs of axj_run (device snapshot, copy on a second stream while the next
    steps run, callback one output later) are the states of those iterations exactly."""
    c = CASES["jet_sc"]()
    patches = axj.patches_from_records(c["records"], c["Nz"], c["Nr"])
    a = axj.AxiJetSolver(c["params"], c["zvec"], c["rvec"], c["ibval"], patches)
    b = axj.AxiJetSolver(c["params"], c["zvec"], c["rvec"], c["ibval"], patches)
    a.set_state(c["pv"], c["target"])
    b.set_state(c["pv"], c["target"])
    seen = []
    a.run(9, out_every=3, callback=lambda it, t, pv: seen.append((it, t, pv)))
    assert [s[0] for s in seen] == [3, 6, 9]
    for it, t, pv in seen:
        b.run(3)
        assert b.get_time() == (it, t)
        assert np.array_equal(pv, b.get_state())
    a.close()
    b.close()


def test_restart_round_trip():
    """Restart (ModSolver.f90:103-106): a run continued from a written state, its
    iteration and time equals the uninterrupted run. With the physical dt the step
    depends on nothing else (the stale-T dt of the reference restarts from T = 0, as
    the reference's module scalar does)."""
    c = CASES["jet_forcing_physdt"]()
    patches = axj.patches_from_records(c["records"], c["Nz"], c["Nr"])
    full = axj.AxiJetSolver(c["params"], c["zvec"], c["rvec"], c["ibval"], patches)
    full.set_state(c["pv"], c["target"])
    saved = []
    full.run(8, out_every=4, callback=lambda it, t, pv: saved.append((it, t, pv)))
    it4, t4, pv4 = saved[0]
    rest = axj.AxiJetSolver(c["params"], c["zvec"], c["rvec"], c["ibval"], patches)
    rest.set_state(pv4, c["target"], iteration=it4, time=t4)
    rest.run(4)
    assert rest.get_time() == full.get_time()
    assert np.array_equal(rest.get_state(), full.get_state())
    full.close()
    rest.close()


def test_multistep_jet512x128(oracle_mod):
    """The small plain jet (512 x 128): 100 RK4 steps, relative L2 error per field."""
    c = fixtures.case("jet512x128")
    dev, ora = pair(c, oracle_mod)
    dev.run(100)
    ora.run(100)
    a, b = dev.get_state(), ora.get_state()
    for k in (0, 1, 3, 4):
        l2 = np.linalg.norm(a[k] - b[k]) / np.linalg.norm(b[k])
        assert l2 < 1e-11, (k, l2)


def test_multistep_writemesh(oracle_mod):
    """The reference generator's case with shock capturing: 60 RK4 steps (graph-run on
    the device), relative L2 error per field."""
    c = CASES["writemesh_sc"]()
    dev, ora = pair(c, oracle_mod)
    dev.run(60)
    ora.run(60)
    a, b = dev.get_state(), ora.get_state()
    for k in (0, 1, 3, 4):
        l2 = np.linalg.norm(a[k] - b[k]) / np.linalg.norm(b[k])
        assert l2 < 1e-11, (k, l2)
    (itd, td), (ito, to) = dev.get_time(), ora.get_time()
    assert itd == ito == 60 and abs(td - to) <= 1e-12 * to


GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def reference_nozzle_4400x640():
    """The reference's own bc file (bc_4400x640_nozzle.dat: SAT inflow below and above the
    lip, NSCBC no-slip walls around the lip up to i = 597 between rows 150 and 169, a
    non-reflecting top and outflow, the axis) on the production grid and flow, with the
    points inside the lip blanked (rows 151..168, columns 1..596, 1-based) as the
    reference's generator blanks its lip (WriteMeshAndSoln/write_soln_file.f90:204-213)."""
    rec = axj.read_bc_file(os.path.join(GOLDEN, "bc_4400x640_nozzle.dat"))
    c = fixtures.case("jet4400x640", records=rec)
    ib = np.ones((c["Nr"], c["Nz"]))
    ib[150:168, :596] = 0.0
    c["ibval"] = ib
    return c


PRODUCTION = {
    # the benchmarked configuration: 4400 x 640, Mach 1.5, Re 5000, shock capturing, reference dt
    "jet4400x640": lambda: fixtures.case("jet4400x640"),
    "reference_nozzle_4400x640": reference_nozzle_4400x640,
}


@pytest.mark.parametrize("name", list(PRODUCTION))
def test_rk4_steps_production_size(oracle_mod, name):
    """Three RK4 steps at the production size against the oracle, <= 1e-12 per field per
    step, with every path computing its own dt (the stale-T reference dt)."""
    c = PRODUCTION[name]()
    dev, ora = pair(c, oracle_mod)
    if name.startswith("reference_nozzle"):
        blank = np.asarray(c["ibval"]) == 0
        assert blank.sum() == 18 * 596
    for step in range(3):
        dd = dev.compute_time_step()
        do = ora.compute_time_step()
        assert abs(dd - do) <= 1e-14 * abs(do), (step, dd, do)
        dev.rk4(do)
        ora.rk4(do)
        errs = field_relerr(dev.get_state(), ora.get_state())
        assert max(errs) < REL, (step, errs)
    dev.close()
    ora.close()


@pytest.mark.parametrize("name", ["jet_sc", "jet", "nozzle_sat_wall_sc", "writemesh_sc"])
@pytest.mark.parametrize("precision", [0, 1])
def test_half_tile_stage_kernel_equals_whole_tiles(name, precision):
    """Interior tiles as two CTAs of 8 rows (stage_rows 8) and as one CTA of 16 rows
    (stage_rows 16) run the same per-point code (separate compilations, so FMA contraction
    may differ in the last bit): equal to 1e-13 of each field's scale after 4 steps; a half
    tile in the wrong place or a missed half is an O(1) difference."""
    c = CASES[name]()
    c["params"].precision = precision
    patches = axj.patches_from_records(c["records"], c["Nz"], c["Nr"])
    out = []
    for rows in (8, 16):
        c["params"].stage_rows = rows
        s = axj.AxiJetSolver(c["params"], c["zvec"], c["rvec"], c["ibval"], patches)
        s.set_state(c["pv"], c["target"])
        s.run(4)
        out.append(s.get_state())
        s.close()
    errs = field_relerr(out[0], out[1])
    assert max(errs) < 1e-13, errs


def test_half_tile_stage_kernel_production_size():
    c = fixtures.case("jet4400x640")
    patches = axj.patches_from_records(c["records"], c["Nz"], c["Nr"])
    out = []
    for rows in (8, 16):
        c["params"].stage_rows = rows
        s = axj.AxiJetSolver(c["params"], c["zvec"], c["rvec"], c["ibval"], patches)
        s.set_state(c["pv"], c["target"])
        s.run(3)
        out.append(s.get_state())
        s.close()
    errs = field_relerr(out[0], out[1])
    assert max(errs) < 1e-13, errs
