"""The operator tables and default constants of the oracle and of the library against
the reference's own source text (tests/golden/reference_constants.json, written by
tests/golden/make_reference_constants.py from ModOperator.f90 and ModuleVariables.f90 with
Fortran's literal kinds: the truncated-Gaussian boundary rows are single-precision
literals). Every value must be equal exactly (a signed zero of a mirrored row equals 0)."""
import json
import os

import numpy as np
import pytest

import axisymmetricjet_b200 as axj
from axisymmetricjet_b200 import _ffi, fixtures

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_constants.json")


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        d = json.load(f)
    d["arrays"] = {k: np.array([[float.fromhex(x) for x in row] for row in v]) for k, v in d["tables"].items()}
    return d


def _assert_exact(got, want, what):
    bad = np.argwhere(got != want)
    assert len(bad) == 0, (what, [(tuple(i), got[tuple(i)], want[tuple(i)]) for i in bad[:5]])


def test_library_tables_equal_the_reference_source(golden):
    s1, s2, tg = axj.operator_tables()
    _assert_exact(s1, golden["arrays"]["SBP1"], "SBP1")
    _assert_exact(s2, golden["arrays"]["SBP2"], "SBP2")
    _assert_exact(tg, golden["arrays"]["TGFILT"], "TGfilt")


def test_oracle_tables_equal_the_reference_source(golden, oracle_mod):
    c = fixtures.case("jet96x64")
    o = oracle_mod.Oracle(c["params"], c["zvec"], c["rvec"], c["ibval"],
                          oracle_mod.patches_from_records(c["records"], c["Nz"], c["Nr"]))
    s1, s2, tg = o.tables()
    _assert_exact(s1, golden["arrays"]["SBP1"], "SBP1")
    _assert_exact(s2, golden["arrays"]["SBP2"], "SBP2")
    _assert_exact(tg, golden["arrays"]["TGFILT"], "TGfilt")


def test_boundary_filter_rows_are_single_precision(golden):
    """TGfilt rows 1-3 (and their mirrors) hold default-REAL literals: every value is a
    float32 (ModOperator.f90:94-97), the interior row is double precision (:113-114)."""
    tg = golden["arrays"]["TGFILT"]
    for row in (1, 2, 3, 5, 6, 7):
        assert np.array_equal(tg[row].astype(np.float32).astype(np.float64), tg[row]), row
    assert not np.array_equal(tg[4].astype(np.float32).astype(np.float64), tg[4])


def test_default_params_equal_the_reference_source(golden):
    p = _ffi.default_params()
    r = {k: float.fromhex(v["value"]) for k, v in golden["reals"].items()}
    i = golden["integers"]
    for name in ("gam", "Re", "Pr", "CFL", "sponge_start_top", "sponge_A_top", "sponge_end_left", "sponge_A_left",
                 "C_mu", "C_beta", "C_kappa"):
        assert getattr(p, name) == r[name], name
    assert p.forcing_alpha == r["alpha"]
    assert p.do_viscous_terms == i["do_viscous_terms"]
    assert p.shock_capturing == i["ShockCapturing"]
    assert p.control_forcing == i["ControlForcing"]


def test_bc_codes_equal_the_reference_source(golden):
    i = golden["integers"]
    for name in ("AXIS", "SAT_FARFIELD", "NSCBC_NONREFLECTING", "SAT_NOSLIP_WALL", "NSCBC_NOSLIP_WALL", "SPONGE"):
        assert getattr(_ffi, name) == i[name], name
