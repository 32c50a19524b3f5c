"""The device path of the patch preprocessing (axj_prep.cuh: one thread per grid row for
the descriptors, codes and face list, one per tile for the tile classes) against the host
path axj_create uses by default, with the device path's per-row and per-tile functions run
on the host: descriptors, face list, the four tile lists and the stale-T point must be
identical. Algorithm 2 (the same functions launched on the device) is compared in the GPU
suite."""
import os

import numpy as np
import pytest

import axisymmetricjet_b200 as axj
from axisymmetricjet_b200 import fixtures
from axisymmetricjet_b200._ffi import NSCBC_NOSLIP_WALL, SAT_NOSLIP_WALL

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _reference_nozzle():
    rec = axj.read_bc_file(os.path.join(GOLDEN, "bc_4400x640_nozzle.dat"))
    ib = np.ones((200, 640))
    ib[150:168, :596] = 0.0
    return rec, 640, 200, ib


LAYOUTS = {
    "jet": lambda: (fixtures.JET_RECORDS, 96, 64, np.ones((64, 96))),
    "jet4400x640": lambda: (fixtures.JET_RECORDS, 4400, 640, np.ones((640, 4400))),
    "ragged": lambda: (fixtures.JET_RECORDS, 77, 45, np.ones((45, 77))),
    "nozzle_nscbc": lambda: (lambda c: (c["records"], 96, 64, c["ibval"]))(fixtures.nozzle_case(wall=NSCBC_NOSLIP_WALL)),
    "nozzle_sat": lambda: (lambda c: (c["records"], 96, 64, c["ibval"]))(fixtures.nozzle_case(wall=SAT_NOSLIP_WALL)),
    "writemesh": lambda: (lambda c: (c["records"], 250, 50, c["ibval"]))(fixtures.writemesh_case()),
    "reference_nozzle_bc": _reference_nozzle,
    "overlap": lambda: (fixtures.JET_RECORDS + [(NSCBC_NOSLIP_WALL, -1, 4, 4, 10, 20),
                                                (SAT_NOSLIP_WALL, -2, 30, 60, 40, 40)], 96, 64, np.ones((64, 96))),
}


def _assert_same(a, b):
    assert np.array_equal(a["desc"], b["desc"])
    assert np.array_equal(a["faces"], b["faces"])
    for x, y in zip(a["tiles"], b["tiles"]):
        assert np.array_equal(x, y)
    assert a["stale"] == b["stale"]


@pytest.mark.parametrize("name", list(LAYOUTS))
def test_device_algorithm_equals_host_path(name):
    records, Nz, Nr, ib = LAYOUTS[name]()
    patches = axj.patches_from_records(records, Nz, Nr)
    host = axj.prep_maps(patches, Nz, Nr, ib, algorithm=0)
    dev = axj.prep_maps(patches, Nz, Nr, ib, algorithm=1)
    _assert_same(host, dev)
    assert sum(len(t) for t in host["tiles"][:2]) == sum(len(t) for t in host["tiles"][2:])
    if name == "jet4400x640":
        assert len(host["tiles"][0]) > 0.8 * (len(host["tiles"][0]) + len(host["tiles"][1]))


def test_point_maps_agree_with_prep_maps():
    records, Nz, Nr, ib = LAYOUTS["nozzle_sat"]()
    patches = axj.patches_from_records(records, Nz, Nr)
    m = axj.point_maps(patches, Nz, Nr, ib)
    d = axj.prep_maps(patches, Nz, Nr, ib)["desc"][:, :Nz]
    assert np.array_equal(m["zrow"], d & 15)
    assert np.array_equal(m["rrow"], (d >> 4) & 15)
    assert np.array_equal(m["blank"], (d >> 8) & 1)
    assert np.array_equal(m["nfaceops"] > 0, (d >> 12) > 0)


def test_patch_prep_parameter_is_checked():
    c = fixtures.case("jet96x64", patch_prep=2)
    patches = axj.patches_from_records(c["records"], c["Nz"], c["Nr"])
    with pytest.raises(axj.AxjError) as e:
        axj.AxiJetSolver(c["params"], c["zvec"], c["rvec"], c["ibval"], patches)
    assert e.value.code == 1


@pytest.mark.gpu
def test_device_path_on_the_device_equals_host_path():
    """Algorithm 2: the kernels of axj_prep.cu on the device; and a handle built with
    patch_prep = 1 steps exactly as one built on the host."""
    for name in ("jet", "nozzle_sat", "writemesh", "reference_nozzle_bc", "overlap", "jet4400x640"):
        records, Nz, Nr, ib = LAYOUTS[name]()
        patches = axj.patches_from_records(records, Nz, Nr)
        _assert_same(axj.prep_maps(patches, Nz, Nr, ib, algorithm=0), axj.prep_maps(patches, Nz, Nr, ib, algorithm=2))
    states = []
    for prep in (0, 1):
        c = fixtures.nozzle_case(wall=SAT_NOSLIP_WALL, sc=True, Mj=1.5, Re=5000.0, patch_prep=prep)
        s = axj.AxiJetSolver(c["params"], c["zvec"], c["rvec"], c["ibval"],
                             axj.patches_from_records(c["records"], c["Nz"], c["Nr"]))
        s.set_state(c["pv"], c["target"])
        s.run(3)
        states.append(s.get_state())
        s.close()
    assert np.array_equal(states[0], states[1])
