"""Host-side checks of the C-ABI library (no device work)."""
import ctypes as C
import os
import re

import pytest

import axisymmetricjet_b200 as axj
from axisymmetricjet_b200 import fixtures

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "axj.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(axj_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = axj.load_library()
    names = declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert lib.axj_version().decode().startswith("axj")


def test_default_params_match_c():
    lib = axj.load_library()
    p = axj.AxjParams()
    lib.axj_default_params(C.byref(p))
    q = axj.default_params()
    assert bytes(p) == bytes(q)


@pytest.mark.parametrize("records", [fixtures.JET_RECORDS, fixtures.nozzle_records(20, 24, 28)])
def test_patches_library_equals_oracle(oracle_mod, records):
    for Nz, Nr in ((96, 64), (4400, 640)):
        assert axj.patches_from_records(records, Nz, Nr) == oracle_mod.patches_from_records(records, Nz, Nr)


def test_read_reference_bc_file(oracle_mod):
    rec = axj.read_bc_file(os.path.join(GOLDEN, "bc_4400x640_nozzle.dat"))
    assert rec[0] == (91, 1, 1, 1, 1, 150)
    assert rec[-1] == (90, 2, 1, -1, 1, 1)
    assert axj.patches_from_records(rec, 4400, 640) == oracle_mod.patches_from_records(rec, 4400, 640)


def test_bc_file_parsing(tmp_path):
    """Records of 9 integers (ModPatch.f90:30-63); blank lines are skipped as list-directed
    input skips them; a missing file or a short record is an error."""
    with pytest.raises(axj.AxjError) as e:
        axj.read_bc_file(str(tmp_path / "missing.dat"))
    assert e.value.code == 1
    p = tmp_path / "bc.dat"
    p.write_text("\n1 91 1 1 1 1 5 1 1\n\n1 90 2 1 -1 1 1 1 1\n\n")
    assert axj.read_bc_file(str(p)) == [(91, 1, 1, 1, 1, 5), (90, 2, 1, -1, 1, 1)]
    for short in ("1 91 1 1 1 1 5 1\n", "1 91 1 1 1 x 5 1 1\n"):
        p.write_text(short)
        with pytest.raises(axj.AxjError) as e:
            axj.read_bc_file(str(p))
        assert e.value.code == 6


def test_bad_bc_record_rejected():
    with pytest.raises(axj.AxjError) as e:
        axj.patches_from_records([(91, 3, 1, 1, 1, -1)], 64, 64)
    assert e.value.code == 6


def test_create_rejects_bad_input_before_touching_a_device():
    c = fixtures.case("jet96x64")
    # grid too small
    with pytest.raises(axj.AxjError) as e:
        axj.AxiJetSolver(c["params"], c["zvec"][:8, :8], c["rvec"][:8, :8], c["ibval"][:8, :8], [])
    assert e.value.code == 7
    # non-tensor-product grid
    z = c["zvec"].copy()
    z[5, 7] += 1e-3
    patches = axj.patches_from_records(c["records"], c["Nz"], c["Nr"])
    with pytest.raises(axj.AxjError) as e:
        axj.AxiJetSolver(c["params"], z, c["rvec"], c["ibval"], patches)
    assert e.value.code in (7, 9)  # 9 when no device is present (checked first)
