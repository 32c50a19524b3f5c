"""The error measures of axisymmetricjet_b200.accuracy on constructed fields (no GPU)."""
import numpy as np

from axisymmetricjet_b200 import accuracy


def _state(rng, Nr=6, Nz=10):
    pv = np.empty((5, Nr, Nz))
    pv[0] = 1.0 + 0.1 * rng.random((Nr, Nz))
    pv[1] = 0.0
    pv[2] = 0.0
    pv[3] = rng.random((Nr, Nz))
    pv[4] = 1.0 + 0.1 * rng.random((Nr, Nz))
    return pv


def test_pressure_is_the_reference_pvec():
    pv = _state(np.random.default_rng(1))
    assert np.array_equal(accuracy.pressure(pv), pv[0] * pv[4])  # ModAssign.f90:19


def test_relative_errors():
    rng = np.random.default_rng(2)
    ref = _state(rng)
    got = ref.copy()
    got[0] *= 1.0 + 1e-6
    got[1, 2, 3] = 1e-9  # a perturbation of a zero field
    e = accuracy.field_errors(got, ref)
    assert abs(e["rho"]["rel_l2"] - 1e-6) < 1e-12
    assert abs(e["rho"]["rel_max"] - 1e-6) < 1e-12
    # V_r is zero in the reference: its own relative error is the raw norm, its error
    # relative to the velocity vector is small
    assert e["Vr"]["rel_l2"] == 1e-9
    assert e["Vr"]["rel_max_vel"] == 1e-9 / np.abs(ref[3]).max()
    assert e["p"]["rel_l2"] == accuracy.rel_l2(got[0] * got[4], ref[0] * ref[4])
    assert e["T"]["rel_l2"] == 0.0


def test_farfield_probe_row_and_measures():
    rng = np.random.default_rng(3)
    ref = _state(rng)
    target = ref.copy()
    target[0] = 1.0
    target[4] = 1.0
    r = np.linspace(0.0, 5.0, ref.shape[1])
    f = accuracy.farfield_pressure(ref, ref, target, r, 2.1)
    assert f["row"] == int(np.argmin(np.abs(r - 2.1)))
    assert f["prms"] == f["prms_ref"] > 0
    assert f["prms_rel_err"] == 0.0 and f["diff_rms_rel"] == 0.0 and f["diff_rms_over_p_inf"] == 0.0
    got = ref.copy()
    got[0, f["row"]] += 1e-3
    g = accuracy.farfield_pressure(got, ref, target, r, 2.1)
    d = 1e-3 * ref[4, f["row"]]
    assert abs(g["diff_rms_over_p_inf"] - np.sqrt(np.mean(d * d))) < 1e-15
