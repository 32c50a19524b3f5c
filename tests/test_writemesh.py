"""The case of the reference's own generator (WriteMeshAndSoln/write_soln_file.f90):
the restated grid, blanking, bc file and initial condition, on the host and the oracle.
The device parity of the case is in test_gpu_parity.py ("writemesh", "writemesh_sc")."""
import numpy as np

import axisymmetricjet_b200 as axj
from axisymmetricjet_b200 import fixtures
from axisymmetricjet_b200._ffi import AXIS, NSCBC_NONREFLECTING, NSCBC_NOSLIP_WALL, SAT_FARFIELD


def test_grid_shape_and_stretching():
    z, r, ib = fixtures.writemesh_grid()
    assert z.shape == (250,) and r.shape == (50,) and ib.shape == (50, 250)
    assert np.all(np.diff(z) > 0) and np.all(np.diff(r) > 0)
    # the first stretching stops at the first column beyond z = 11 (ipos2 = 127, 1-based);
    # the second starts there, just above 11, and ends short of 15
    assert z[125] <= 11.0 < z[126] < z[127]
    assert 14.8 < z[-1] < 15.0 and 14.99 < r[-1] < 15.0
    assert 0.0 < z[0] < 0.2 and 0.0 < r[0] < 0.2  # xi starts at 1/n: no point on z = 0 or r = 0


def test_blanked_lip_and_bc_rows_agree():
    z, r, ib = fixtures.writemesh_grid()
    rec = fixtures.writemesh_records(z, r)
    (_, _, _, _, _, jbottom), (_, _, _, iright, _, _), (_, _, _, _, _, jtop) = rec[0], rec[1], rec[2]
    assert (jbottom, jtop, iright) == (19, 25, 70)
    # blanked: rows strictly between the lip walls, columns left of the lip's right face
    blank = np.argwhere(ib == 0.0)
    assert blank[:, 0].min() == jbottom and blank[:, 0].max() == jtop - 2
    assert blank[:, 1].min() == 0 and blank[:, 1].max() == iright - 2
    assert len(blank) == (jtop - jbottom - 1) * (iright - 1)
    assert rec[6] == (NSCBC_NOSLIP_WALL, -1, -1, -1, 1, -1)  # the generator's outflow row
    assert [x[0] for x in rec] == [SAT_FARFIELD, NSCBC_NOSLIP_WALL, NSCBC_NOSLIP_WALL, NSCBC_NOSLIP_WALL,
                                   SAT_FARFIELD, NSCBC_NONREFLECTING, NSCBC_NOSLIP_WALL, AXIS]


def test_bc_file_round_trip(tmp_path, oracle_mod):
    c = fixtures.writemesh_case()
    path = str(tmp_path / "bc.dat")
    fixtures.write_bc_file(path, c["records"])
    assert axj.read_bc_file(path) == c["records"]
    assert open(path).readline() == "1  91  1  1  1  1  19  1  1  \n"
    gp = axj.patches_from_records(c["records"], c["Nz"], c["Nr"])
    assert gp == oracle_mod.patches_from_records(c["records"], c["Nz"], c["Nr"])


def test_initial_condition():
    c = fixtures.writemesh_case()
    pv, r, z = c["pv"], c["r"], c["z"]
    Uj = 0.8 * 0.6 ** 0.5
    # p = rho T = 1; no radial or swirl velocity; still fluid beyond r = 1
    np.testing.assert_allclose(pv[0] * pv[4], 1.0, rtol=1e-15)
    assert not pv[1].any() and not pv[2].any()
    assert not pv[3][r > 1.0].any()
    # the core runs at U_j up to z = 6 and decays as (z - 5)**-1.5 beyond
    near = z <= 6.0
    assert abs(pv[3][0, near].max() - Uj) < 1e-6 * Uj
    far = np.nonzero(z > 6.0)[0][5]
    np.testing.assert_allclose(pv[3][0, far], pv[3][0, 0] / (z[far] - 5.0) ** 1.5, rtol=1e-14)
    # the core is at the jet temperature T_j / T_inf = 0.6, the ambient at 1
    np.testing.assert_allclose(pv[4][0, 0], 0.6, rtol=1e-6)
    assert np.all(pv[4][r > 1.0] == 1.0)
    assert np.array_equal(c["target"], pv)


def test_oracle_steps_the_case(oracle_mod):
    for sc in (False, True):
        c = fixtures.writemesh_case(sc=sc)
        ora = oracle_mod.Oracle(c["params"], c["zvec"], c["rvec"], c["ibval"],
                                oracle_mod.patches_from_records(c["records"], c["Nz"], c["Nr"]))
        ora.set_state(c["pv"], c["target"])
        for _ in range(10):
            ora.rk4(ora.compute_time_step())
        st = ora.get_state()
        assert np.isfinite(st).all()
        # blanked points are never updated (ModRungeKutta.f90:139)
        blank = c["ibval"] == 0.0
        assert np.array_equal(st[:, blank], c["pv"][:, blank])
