"""Known-answer tests that pin the CPU oracle (no GPU needed).

The reference ships no tests or golden vectors, so the oracle's restatement of
ModOperator / ModDeriv / ModPatch is pinned by properties of the reference's own
tables and fixture: polynomial exactness of the SBP rows (ModOperator.f90:25-78),
unit sums of the truncated-Gaussian rows (:93-112), constant metrics on uniform
grids (ModDeriv.f90:241-382), the shipped bc file (bc_4400x640_nozzle.dat) and
free-stream preservation of the full right-hand side.
"""
import os
from fractions import Fraction

import numpy as np
import pytest

from axisymmetricjet_b200 import fixtures
from axisymmetricjet_b200._ffi import default_params

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _tables(oracle_mod):
    c = fixtures.case("jet96x64")
    o = oracle_mod.Oracle(c["params"], c["zvec"], c["rvec"], c["ibval"],
                          oracle_mod.patches_from_records(c["records"], c["Nz"], c["Nr"]))
    return o.tables()


def _window(row, width):
    """offsets of the window of SBP row `row` relative to the point (ModDeriv.f90:25-46)"""
    if row == 4:
        return list(range(-2, 3)) if width == 6 else list(range(-4, 5))
    if row < 4:
        return [-row + m for m in range(width)]
    end = 8 - row
    return [end - (width - 1) + m for m in range(width)]


def _exact_degree(coef, offs, order):
    deg = -1
    for k in range(0, 8):
        lhs = sum(Fraction(c) * Fraction(o) ** k for c, o in zip(coef, offs))
        if order == 1:
            rhs = Fraction(k) * Fraction(0) ** (k - 1) if k >= 1 else Fraction(0)
        else:
            rhs = Fraction(k * (k - 1)) * Fraction(0) ** (k - 2) if k >= 2 else Fraction(0)
        if abs(float(lhs - rhs)) > 1e-12:
            break
        deg = k
    return deg


def test_sbp1_rows(oracle_mod):
    s1, _, _ = _tables(oracle_mod)
    for row in range(9):
        n = 5 if row == 4 else 6
        coef = s1[row, :n]
        assert abs(coef.sum()) < 1e-15, row
        deg = _exact_degree(coef, _window(row, 6)[:n], 1)
        assert deg >= (4 if row == 4 else 2), (row, deg)
    # bottom block is the negated mirror of the top block (ModOperator.f90:32-38)
    np.testing.assert_array_equal(s1[5:9], -s1[3::-1, ::-1])


def test_sbp2_rows(oracle_mod):
    _, s2, _ = _tables(oracle_mod)
    for row in range(9):
        n = 5 if row == 4 else 6
        coef = s2[row, :n]
        assert abs(coef.sum()) < 1e-14, row
        deg = _exact_degree(coef, _window(row, 6)[:n], 2)
        assert deg >= (3 if row == 4 else 1), (row, deg)
    np.testing.assert_array_equal(s2[5:9], s2[3::-1, ::-1])


def test_tg_rows(oracle_mod):
    _, _, tg = _tables(oracle_mod)
    assert tg[0, 0] == 1.0 and np.all(tg[0, 1:] == 0.0)
    # interior 9-point row sums to exactly 1 in rational arithmetic (:111-112)
    interior = [Fraction(107, 103680), Fraction(149, 12960), Fraction(1997, 25920), Fraction(3091, 12960),
                Fraction(3565, 10368)]
    assert sum(interior) * 2 - interior[-1] == 1
    assert abs(tg[4, :9].sum() - 1.0) < 1e-15
    # boundary rows are single-precision literals in the reference: sums are 1 to float accuracy
    for row in (1, 2, 3):
        assert abs(tg[row].sum() - 1.0) < 1e-6
        assert all(float(np.float32(v)) == v for v in tg[row])
    np.testing.assert_array_equal(tg[5:9], tg[3::-1, ::-1])


def test_uniform_metrics(oracle_mod):
    c = fixtures.make_case(48, 32, 30.0, 15.0, 0.9, 1000.0)
    z = np.linspace(0.0, 4.7, 48)
    r = np.linspace(0.0, 3.1, 32)
    zvec = np.ascontiguousarray(np.broadcast_to(z[None, :], (32, 48)))
    rvec = np.ascontiguousarray(np.broadcast_to(r[:, None], (32, 48)))
    o = oracle_mod.Oracle(c["params"], zvec, rvec, c["ibval"],
                          oracle_mod.patches_from_records(c["records"], 48, 32))
    dxidz, detadr, ddxi, ddeta = o.metrics()
    np.testing.assert_allclose(dxidz, 47 / 4.7, rtol=1e-13)
    np.testing.assert_allclose(detadr, 31 / 3.1, rtol=1e-13)
    assert np.abs(ddxi).max() < 1e-9 and np.abs(ddeta).max() < 1e-9


def test_reference_bc_fixture(oracle_mod):
    """bc_4400x640_nozzle.dat (the reference's only input fixture) -> the 4-wide strips
    that CreateAllPatches/PatchCreation produce (ModPatch.f90:117-309)."""
    rows = []
    with open(os.path.join(GOLDEN, "bc_4400x640_nozzle.dat")) as f:
        for line in f:
            v = [int(x) for x in line.split()]
            if v:
                rows.append(tuple(v[1:7]))
    assert len(rows) == 8
    got = oracle_mod.patches_from_records(rows, 4400, 640)
    expect = [
        (1, 4, 1, 150, 91, 1),
        (1, 597, 147, 150, 94, -2),
        (597, 600, 150, 169, 94, 1),
        (1, 597, 169, 172, 94, 2),
        (1, 4, 169, 640, 91, 1),
        (1, 4400, 637, 640, 92, -2),
        (4397, 4400, 1, 640, 92, -1),
        (1, 4400, 1, 4, 90, 2),
    ]
    assert got == expect


def _uniform_case():
    Nz, Nr = 40, 32
    z, r, zvec, rvec = fixtures.grid(Nz, Nr, 30.0, 15.0)
    pv = np.zeros((5, Nr, Nz))
    pv[0], pv[3], pv[4] = 1.25, 0.4, 0.8
    return Nz, Nr, zvec, rvec, pv


@pytest.mark.parametrize("sc", [0, 1])
def test_free_stream_preservation(oracle_mod, sc):
    """A uniform state equal to its target has a zero right-hand side everywhere."""
    Nz, Nr, zvec, rvec, pv = _uniform_case()
    params = default_params(shock_capturing=sc, C_mu=0.002, C_beta=1.75, C_kappa=0.01)
    o = oracle_mod.Oracle(params, zvec, rvec, np.ones((Nr, Nz)),
                          oracle_mod.patches_from_records(fixtures.JET_RECORDS, Nz, Nr))
    o.set_state(pv, pv)
    rhs = o.compute_rhs(pv)
    assert np.abs(rhs).max() < 1e-11
