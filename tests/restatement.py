"""A plain-Python restatement of the reference's patch-driven operators and of its
artificial-diffusivity sensor, written from the Fortran directly (ModDeriv.f90,
ModTGfilter.f90, ModShockCapturing.f90) as a second, independent check of the C oracle.
Test infrastructure only: slow (Python loops), for grids of a few thousand points. Every
DOT_PRODUCT is summed left to right from 0 over the full row, every expression in the
Fortran's operand order, transcendental functions through libm (math module)."""
import math

import numpy as np


def window(row, i, width):
    """First index of the DOT_PRODUCT window of SBP row `row` at point i (0-based):
    rows 0-3 start at the strip's first point i - row, rows 5-8 end at its last point
    i + 8 - row, row 4 is centred."""
    if row == 4:
        return i - (width - 1) // 2, width
    if row < 4:
        return i - row, width
    return i + 8 - row - (width - 1), width


def dot(coef, line, w0, n):
    s = 0.0
    for m in range(n):
        q = w0 + m
        v = line[q] if 0 <= q < len(line) else 0.0  # never-written halo cells are 0
        s = s + coef[m] * v
    return s


def stencil(table, var, rows, blank, dirn, wide, interior_width):
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
                w0, n = window(4, pos, interior_width)
            else:
                w0, n = window(row, pos, wide)
            out[j, i] = dot(table[row], line, w0, n)
    return out


def tg_inplace_z(table, var, rows, blank):
    """PerformTGfilter(q, 1, q): point i reads the already filtered points before it."""
    q = var.copy()
    Nr, Nz = q.shape
    for i in range(Nz):
        for j in range(Nr):
            if blank[j, i]:
                continue
            row = int(rows[j, i])
            w0, n = window(row, i, 9 if row == 4 else 11)
            q[j, i] = dot(table[row], q[j, :], w0, n)
    return q


def sensor(pv, tables, maps, metrics, z, r, params):
    """ComputeArtTransCoeffs (ModShockCapturing.f90:5-101) on the state pv[5, Nr, Nz] of a
    single block: mu*, beta*, kappa* after the scaling and the z ramp, before
    UpdateTransportCoeffs. tables = (SBP1, SBP2, TGfilt); maps = axj_point_maps; metrics =
    (dxidz, detadr, ddxidxidz, ddetadetadr) per point; z, r the coordinate lines."""
    s1, s2, tg = tables
    dxidz, detadr = metrics[0], metrics[1]
    blank = maps["blank"] == 1
    zr, rr = maps["zrow"], maps["rrow"]
    Nr, Nz = pv.shape[1:]
    rho, Vr, Vz, T = pv[0], pv[1], pv[3], pv[4]
    # Compute1stDerivative of V_r and V_z (ModRHS.f90:30-39)
    dVrdz = stencil(s1, Vr, zr, blank, 1, 6, 5) * dxidz
    dVzdz = stencil(s1, Vz, zr, blank, 1, 6, 5) * dxidz
    dVrdr = stencil(s1, Vr, rr, blank, 2, 6, 5) * detadr
    dVzdr = stencil(s1, Vz, rr, blank, 2, 6, 5) * detadr
    rr2 = np.broadcast_to(r[:, None], (Nr, Nz))
    third = 1.0 / 3.0
    # ComputeDilatation (:106-124), ComputeMgnStrRate (:127-158); row 1 (r = 0) takes the
    # axis forms, so its V_r/r is never used
    with np.errstate(divide="ignore", invalid="ignore"):
        vr_r = Vr / rr2
    dil = dVrdr + vr_r + dVzdz
    dil[0] = 2.0 * dVrdr[0] + dVzdz[0]
    S11 = dVrdr - third * dil
    S13 = 0.5 * (dVrdz + dVzdr)
    S33 = dVzdz - third * dil
    S22 = vr_r - third * dil
    S22[0] = dVrdr[0] - third * dil[0]
    zero = np.zeros_like(S11)
    S = np.sqrt(S11 * S11 + zero * zero + S13 * S13 + zero * zero + S22 * S22 + zero * zero + S13 * S13 + zero * zero
                + S33 * S33)
    # fourth derivatives in computational coordinates (:27-51)
    def d4(f, dirn):
        rows = zr if dirn == 1 else rr
        return stencil(s2, stencil(s2, f, rows, blank, dirn, 6, 5), rows, blank, dirn, 6, 5)
    d4Sz, d4Sr, d4Tz, d4Tr, d4Dz, d4Dr = d4(S, 1), d4(S, 2), d4(T, 1), d4(T, 2), d4(dil, 1), d4(dil, 2)
    # ComputeTobeFilteredQuantities (:160-222)
    dz = np.empty(Nz)
    dz[1:-1] = (z[2:] - z[:-2]) / 2.0
    dz[0] = z[1] - z[0]
    dz[-1] = z[-1] - z[-2]
    dr = np.empty(Nr)
    dr[1:-1] = (r[2:] - r[:-2]) / 2.0
    dr[0] = r[1] - r[0]
    dr[-1] = r[-1] - r[-2]
    DZ = np.broadcast_to(dz[None, :], (Nr, Nz))
    DR = np.broadcast_to(dr[:, None], (Nr, Nz))
    vort = np.abs(dVrdz - dVzdr)
    H = np.where(-1.0 * dil < 0.0, 0.0, 1.0)
    eps = float(np.float32(1e-15))  # a default-REAL literal (:202)
    fsw = H * (dil * dil) / (dil * dil + vort * vort + eps)
    gam = params.gam
    q_mu = rho * np.abs(d4Sz * (DZ * DZ) + d4Sr * (DR * DR))
    q_beta = rho * fsw * np.abs(d4Dz * (DZ * DZ) + d4Dr * (DR * DR))
    q_kappa = rho / (gam * np.sqrt(T)) * np.abs(d4Tz * DZ + d4Tr * DR)
    # the filters (:63-77): in place along z, then along r into the star fields (zero
    # before: a fresh block), the scaling (:79-81) and the z ramp (:83-92)
    Re, Pr = params.Re, params.Pr
    out = []
    for q, c in ((q_mu, params.C_mu * Re), (q_beta, params.C_beta * Re), (q_kappa, params.C_kappa * Re * Pr)):
        qz = tg_inplace_z(tg, q, zr, blank)
        star = np.where(blank, 0.0, stencil(tg, qz, rr, blank, 2, 11, 9))
        out.append(c * star)
    ramp = np.array([(1.0 + math.tanh(5.0 * (zi - 10.0))) / 2.0 for zi in z])
    return [o * ramp[None, :] for o in out]
