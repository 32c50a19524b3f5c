"""A second, independent restatement of the reference's patch-driven operators in plain
Python, written from ModDeriv.f90 and ModTGfilter.f90 directly, against the C oracle:
Compute1stDerivative (ModDeriv.f90:5-120), Compute2ndDerivative (:123-238) and
PerformTGfilter (ModTGfilter.f90:5-95), including the in-place z filter (the recurrence
ModShockCapturing.f90:63 runs). Both sum DOT_PRODUCT left to right from 0 over the full
row, so they must agree bit for bit. The stencil rows per point come from
axj_point_maps, which equals the oracle's own selection (test_point_maps.py)."""
import numpy as np
import pytest

import axisymmetricjet_b200 as axj
from axisymmetricjet_b200 import fixtures
from axisymmetricjet_b200._ffi import NSCBC_NOSLIP_WALL, SAT_NOSLIP_WALL


def _case(wall):
    Nz, Nr, iw, jb, jt = 48, 36, 12, 14, 18
    ib = np.ones((Nr, Nz))
    ib[jb:jt - 1, :iw - 1] = 0.0
    return fixtures.make_case(Nz, Nr, 30.0, 15.0, 0.9, 1000.0, records=fixtures.nozzle_records(iw, jb, jt, wall),
                              ibval=ib)


def _window(row, i, width):
    """First index of the DOT_PRODUCT window of SBP row `row` at point i (0-based):
    rows 0-3 start at the strip's first point i - row, rows 5-8 end at its last point
    i + 8 - row, row 4 is centred."""
    if row == 4:
        return i - (width - 1) // 2, width
    if row < 4:
        return i - row, width
    return i + 8 - row - (width - 1), width


def _dot(coef, line, w0, n):
    s = 0.0
    for m in range(n):
        q = w0 + m
        v = line[q] if 0 <= q < len(line) else 0.0  # never-written halo cells are 0
        s = s + coef[m] * v
    return s


def _stencil(table, var, rows, blank, dirn, wide, interior_width):
    """out = 0; per non-blanked point the row's DOT_PRODUCT along dirn (1: z, 2: r)."""
    Nr, Nz = var.shape
    out = np.zeros_like(var)
    for j in range(Nr):
        for i in range(Nz):
            if blank[j, i]:
                continue
            row = int(rows[j, i])
            pos, line = (i, var[j, :]) if dirn == 1 else (j, var[:, i])
            if row == 4:
                w0, n = _window(4, pos, interior_width)
            else:
                w0, n = _window(row, pos, wide)
            out[j, i] = _dot(table[row], line, w0, n)
    return out


def _tg_inplace_z(table, var, rows, blank):
    """PerformTGfilter(q, 1, q): point i reads the already filtered points before it."""
    q = var.copy()
    Nr, Nz = q.shape
    for i in range(Nz):
        for j in range(Nr):
            if blank[j, i]:
                continue
            row = int(rows[j, i])
            w0, n = _window(row, i, 9 if row == 4 else 11)
            q[j, i] = _dot(table[row], q[j, :], w0, n)
    return q


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
        d1 = _stencil(s1, var, rows, blank, dirn, 6, 5) * met  # :57 / :108, every point
        assert np.array_equal(d1, o.deriv1(var, dirn)), dirn
        d2 = _stencil(s2, var, rows, blank, dirn, 6, 5)
        d2 = d2 * (met * met) + first * met2  # :175 / :227
        assert np.array_equal(d2, o.deriv2(var, dirn, first)), dirn
        prior = rng.standard_normal((c["Nr"], c["Nz"]))
        f = _stencil(tg, var, rows, blank, dirn, 11, 9)
        want = np.where(blank, prior, f)  # no zeroing: blanked points keep out's values
        assert np.array_equal(want, o.tgfilter(var, dirn, prior)), dirn
    prior = rng.standard_normal((c["Nr"], c["Nz"]))
    assert np.array_equal(_tg_inplace_z(tg, prior, maps["zrow"], blank), o.tgfilter(None, 1, prior, inplace=True))
