"""The per-point stencil rows and face operations that axj_create encodes in the device
descriptors (axj_point_maps) against the ones the oracle's operators select and its
bc loop actually applies (recorded during one pass), point for point, on every patch
layout the tests use and on the reference's own nozzle bc file. No GPU needed."""
import os

import numpy as np
import pytest

import axisymmetricjet_b200 as axj
from axisymmetricjet_b200 import fixtures
from axisymmetricjet_b200._ffi import NSCBC_NOSLIP_WALL, SAT_NOSLIP_WALL

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _reference_nozzle_case():
    """bc_4400x640_nozzle.dat on a 640 x 200 grid (its indices reach i = 597, j = 169),
    with the lip between its wall rows blanked as the generator blanks it."""
    rec = axj.read_bc_file(os.path.join(GOLDEN, "bc_4400x640_nozzle.dat"))
    c = fixtures.make_case(640, 200, 60.0, 15.0, 1.5, 5000.0, records=rec)
    ib = np.ones((200, 640))
    ib[150:168, :596] = 0.0  # rows 151..168, columns 1..596 (1-based) inside the lip
    c["ibval"] = ib
    return c


CASES = {
    "jet": lambda: fixtures.case("jet96x64"),
    "ragged": lambda: fixtures.make_case(77, 45, 30.0, 15.0, 0.9, 1000.0),
    "nozzle_nscbc": lambda: fixtures.nozzle_case(wall=NSCBC_NOSLIP_WALL),
    "nozzle_sat": lambda: fixtures.nozzle_case(wall=SAT_NOSLIP_WALL),
    "writemesh": lambda: fixtures.writemesh_case(),
    "reference_nozzle_bc": _reference_nozzle_case,
    # later patches of the same direction overlapping earlier strips win their points:
    # a -1 wall face at i = 4 over the inflow strip (rows 5..8 there instead of 0..3), and
    # a -2 wall inside the domain
    "overlap": lambda: fixtures.make_case(96, 64, 30.0, 15.0, 0.9, 1000.0, records=fixtures.JET_RECORDS + [
        (NSCBC_NOSLIP_WALL, -1, 4, 4, 10, 20), (SAT_NOSLIP_WALL, -2, 30, 60, 40, 40)]),
}


@pytest.mark.parametrize("name", list(CASES))
def test_point_maps_equal_the_oracle(oracle_mod, name):
    c = CASES[name]()
    patches = axj.patches_from_records(c["records"], c["Nz"], c["Nr"])
    lib = axj.point_maps(patches, c["Nz"], c["Nr"], c["ibval"])
    o = oracle_mod.Oracle(c["params"], c["zvec"], c["rvec"], c["ibval"],
                          oracle_mod.patches_from_records(c["records"], c["Nz"], c["Nr"]))
    o.set_state(c["pv"], c["target"])
    ora = o.point_maps()
    for k in ("zrow", "rrow", "blank", "nfaceops", "faceop_ids"):
        bad = np.argwhere(lib[k] != ora[k])
        assert len(bad) == 0, (k, [(tuple(b), lib[k][tuple(b)], ora[k][tuple(b)]) for b in bad[:5]])
    assert lib["nfaceops"].sum() > 0
    if name == "overlap":
        assert (lib["zrow"][9:20, 0:4] == np.array([5, 6, 7, 8])).all()
        assert (lib["zrow"][0:9, 0:4] == np.array([0, 1, 2, 3])).all()
        # i = 4, j = 10..20: the -1 wall acts there; the inflow face is at i = 1
        assert (lib["faceop_ids"][9:20, 3] == 5).all()
        assert (lib["faceop_ids"][9:20, 0] == 1).all()


def test_point_maps_rejects_bad_patches():
    with pytest.raises(axj.AxjError) as e:
        axj.point_maps([(1, 4, 1, 64, 91, 3)], 64, 64, np.ones((64, 64)))
    assert e.value.code == 6
