"""The C oracle's artificial-diffusivity sensor (ComputeArtTransCoeffs,
ModShockCapturing.f90:5-101: dilatation, strain-rate magnitude, fourth differences, the
three quantities, the in-place z filter, the r filter, scaling and z ramp) against a
second restatement in plain Python (tests/restatement.py), bit for bit."""
import numpy as np
import pytest
from restatement import sensor

import axisymmetricjet_b200 as axj
from axisymmetricjet_b200 import fixtures
from axisymmetricjet_b200._ffi import SAT_NOSLIP_WALL

CASES = {
    "jet_sc": lambda: fixtures.case("jet96x64sc"),
    "nozzle_sat_sc": lambda: fixtures.nozzle_case(Nz=48, Nr=36, iw=12, jb=14, jt=18, wall=SAT_NOSLIP_WALL, sc=True,
                                                  Mj=1.5, Re=5000.0),
}


@pytest.mark.parametrize("name", list(CASES))
def test_sensor_equals_the_oracle_bit_for_bit(oracle_mod, name):
    c = CASES[name]()
    patches = axj.patches_from_records(c["records"], c["Nz"], c["Nr"])
    maps = axj.point_maps(patches, c["Nz"], c["Nr"], c["ibval"])
    o = oracle_mod.Oracle(c["params"], c["zvec"], c["rvec"], c["ibval"],
                          oracle_mod.patches_from_records(c["records"], c["Nz"], c["Nr"]))
    # a state with compressions and expansions: the jet plus a smooth wave
    pv = c["pv"].copy()
    zz, rr = np.meshgrid(c["z"], c["r"])
    pv[3] += 0.05 * np.sin(zz) * np.exp(-rr)
    pv[1] += 0.02 * np.cos(0.7 * zz) * rr * np.exp(-rr)
    got = sensor(pv, axj.operator_tables(), maps, o.metrics(), c["z"], c["r"], c["params"])
    want = o.sensor(pv)
    for g, w, name_ in zip(got, want, ("mu*", "beta*", "kappa*")):
        assert np.abs(w).max() > 0, name_
        bad = np.argwhere(g != w)
        assert len(bad) == 0, (name_, len(bad), [(tuple(b), g[tuple(b)], w[tuple(b)]) for b in bad[:3]])
