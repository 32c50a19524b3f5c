"""A second, independent restatement of the reference's patch-driven operators in plain
Python, written from ModDeriv.f90 and ModTGfilter.f90 directly, against the C oracle:
Compute1stDerivative (ModDeriv.f90:5-120), Compute2ndDerivative (:123-238) and
PerformTGfilter (ModTGfilter.f90:5-95), including the in-place z filter (the recurrence
ModShockCapturing.f90:63 runs). Both sum DOT_PRODUCT left to right from 0 over the full
row, so they must agree bit for bit. The stencil rows per point come from
axj_point_maps, which equals the oracle's own selection (test_point_maps.py)."""
import numpy as np
import pytest
from restatement import stencil, tg_inplace_z

import axisymmetricjet_b200 as axj
from axisymmetricjet_b200 import fixtures
from axisymmetricjet_b200._ffi import NSCBC_NOSLIP_WALL, SAT_NOSLIP_WALL


def _case(wall):
    Nz, Nr, iw, jb, jt = 48, 36, 12, 14, 18
    ib = np.ones((Nr, Nz))
    ib[jb:jt - 1, :iw - 1] = 0.0
    return fixtures.make_case(Nz, Nr, 30.0, 15.0, 0.9, 1000.0, records=fixtures.nozzle_records(iw, jb, jt, wall),
                              ibval=ib)


@pytest.mark.parametrize("wall", [NSCBC_NOSLIP_WALL, SAT_NOSLIP_WALL])
def test_operators_equal_the_oracle_bit_for_bit(oracle_mod, wall):
    c = _case(wall)
    patches = axj.patches_from_records(c["records"], c["Nz"], c["Nr"])
    maps = axj.point_maps(patches, c["Nz"], c["Nr"], c["ibval"])
    o = oracle_mod.Oracle(c["params"], c["zvec"], c["rvec"], c["ibval"],
                          oracle_mod.patches_from_records(c["records"], c["Nz"], c["Nr"]))
    s1, s2, tg = axj.operator_tables()
    dxidz, detadr, ddxidxidz, ddetadetadr = o.metrics()
    rng = np.random.default_rng(11)
    var = rng.standard_normal((c["Nr"], c["Nz"]))
    first = rng.standard_normal((c["Nr"], c["Nz"]))
    blank = maps["blank"] == 1
    for dirn, rows, met, met2 in ((1, maps["zrow"], dxidz, ddxidxidz), (2, maps["rrow"], detadr, ddetadetadr)):
        d1 = stencil(s1, var, rows, blank, dirn, 6, 5) * met  # :57 / :108, every point
        assert np.array_equal(d1, o.deriv1(var, dirn)), dirn
        d2 = stencil(s2, var, rows, blank, dirn, 6, 5)
        d2 = d2 * (met * met) + first * met2  # :175 / :227
        assert np.array_equal(d2, o.deriv2(var, dirn, first)), dirn
        prior = rng.standard_normal((c["Nr"], c["Nz"]))
        f = stencil(tg, var, rows, blank, dirn, 11, 9)
        want = np.where(blank, prior, f)  # no zeroing: blanked points keep out's values
        assert np.array_equal(want, o.tgfilter(var, dirn, prior)), dirn
    prior = rng.standard_normal((c["Nr"], c["Nz"]))
    assert np.array_equal(tg_inplace_z(tg, prior, maps["zrow"], blank), o.tgfilter(None, 1, prior, inplace=True))
