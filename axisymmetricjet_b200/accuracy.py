"""Error measures of a solution against a reference solution of the same grid.

Fields are the solver's primitive planes (rho, V_r, V_theta, V_z, T), each (Nr, Nz) with
z fastest. Pressure is the reference's pvec = rho*T (ModAssign.f90:19; the momentum
equations divide its gradient by gam*rho, ModRHS.f90:92-96). Every measure here is
relative, so the scale of p does not enter.
"""
import numpy as np

FIELDS = ("rho", "Vr", "Vt", "Vz", "T")


def pressure(pv, gam=1.4):
    """pvec = rho*T (ModAssign.f90:19); gam is accepted for the callers' signatures."""
    return pv[0] * pv[4]


def rel_l2(a, b):
    d = np.linalg.norm((a - b).ravel())
    n = np.linalg.norm(b.ravel())
    return float(d / n) if n > 0 else float(d)


def rel_max(a, b):
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / (s if s > 0 else 1.0))


def field_errors(pv, ref, gam=1.4):
    """Relative L2 and max errors per field and for the pressure. The velocity
    components also get errors relative to the velocity vector's norm and largest
    magnitude ("rel_l2_vel", "rel_max_vel"): V_r and V_theta can be zero or small
    perturbations, whose own norm says nothing about the accuracy of the solution."""
    out = {}
    vnorm = float(np.sqrt(sum(np.linalg.norm(ref[k].ravel()) ** 2 for k in (1, 2, 3))))
    vmax = float(max(np.abs(ref[k]).max() for k in (1, 2, 3)))
    for k, name in enumerate(FIELDS):
        out[name] = {"rel_l2": rel_l2(pv[k], ref[k]), "rel_max": rel_max(pv[k], ref[k])}
        if k in (1, 2, 3):
            d = pv[k] - ref[k]
            out[name]["rel_l2_vel"] = float(np.linalg.norm(d.ravel()) / vnorm) if vnorm > 0 else 0.0
            out[name]["rel_max_vel"] = float(np.abs(d).max() / vmax) if vmax > 0 else 0.0
    p, pr = pressure(pv, gam), pressure(ref, gam)
    out["p"] = {"rel_l2": rel_l2(p, pr), "rel_max": rel_max(p, pr)}
    return out


def farfield_pressure(pv, ref, target, r, r_probe, gam=1.4):
    """Pressure fluctuation p' = p - p_target along the grid row nearest r = r_probe.

    Returns the row index, the RMS of p' in both solutions, the relative error of the
    RMS, the RMS of the pointwise difference relative to the reference RMS and relative
    to the ambient pressure (the measure that stays defined where the reference p' is
    still zero: no wave has reached the row yet).
    """
    j = int(np.argmin(np.abs(np.asarray(r) - r_probe)))
    p0 = pressure(target, gam)[j]
    a = pressure(pv, gam)[j] - p0
    b = pressure(ref, gam)[j] - p0
    rms_a = float(np.sqrt(np.mean(a * a)))
    rms_b = float(np.sqrt(np.mean(b * b)))
    d = float(np.sqrt(np.mean((a - b) ** 2)))
    return {
        "row": j,
        "r": float(np.asarray(r)[j]),
        "prms": rms_a,
        "prms_ref": rms_b,
        "prms_rel_err": abs(rms_a - rms_b) / rms_b if rms_b > 0 else None,
        "diff_rms_rel": d / rms_b if rms_b > 0 else None,
        "diff_rms_over_p_inf": d / float(np.abs(p0).mean()),
    }
