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


# ---------------------------------------------------------------------------
# AssignValues, ComputeRHS with the bc loop and sponges, axis_conditions, RK4
# ---------------------------------------------------------------------------
AXIS, SAT_FARFIELD, NSCBC_NONREFLECTING, SAT_NOSLIP_WALL, NSCBC_NOSLIP_WALL = 90, 91, 92, 93, 94


def assign_values(pv):
    """AssignValues (ModAssign.f90:5-29): primitives, p = rho T, mu = kappa = T**0.666,
    beta = (3/5) mu, lambda = beta - (2/3) mu (libm pow per value)."""
    rho, Vr, Vt, Vz, T = (pv[k].copy() for k in range(5))
    mu = np.vectorize(lambda t: math.pow(t, 0.666))(T)
    beta = (3.0 / 5.0) * mu
    return dict(rho=rho, Vr=Vr, Vt=Vt, Vz=Vz, T=T, p=rho * T, mu=mu, kappa=mu.copy(), beta=beta,
                lam=beta - (2.0 / 3.0) * mu)


def _eigen(rho, U, T, gam, rdir):
    """eigen_matrices_in_z_direction (ModBC.f90:280-357, U = V_z) or _in_r_direction
    (:359-437, U = V_r): the diagonal of lam, T_mat and T_mat_inv, 0-based."""
    sT = math.sqrt(T)
    lam = [U, U, U, U - sT, U + sT]
    t_p = rho / ((gam - 1.0) * T)
    t_m = -1.0 / ((gam - 1.0) * sT)
    t_q = 1.0 / ((gam - 1.0) * sT)
    i1 = -1.0 * (gam - 1.0) * T / (gam * rho)
    i4 = (gam - 1.0) * T / (2.0 * gam * rho)
    c_m = -1.0 * (gam - 1.0) * sT / 2.0
    c_p = (gam - 1.0) * sT / 2.0
    c5 = (gam - 1.0) / (2.0 * gam)
    if not rdir:
        Tm = [[-1.0 * rho / T, 0.0, 0.0, t_p, t_p],
              [0.0, 0.0, 1.0, 0.0, 0.0],
              [0.0, 1.0, 0.0, 0.0, 0.0],
              [0.0, 0.0, 0.0, t_m, t_q],
              [1.0, 0.0, 0.0, 1.0, 1.0]]
        Ti = [[i1, 0.0, 0.0, 0.0, 1.0 / gam],
              [0.0, 0.0, 1.0, 0.0, 0.0],
              [0.0, 1.0, 0.0, 0.0, 0.0],
              [i4, 0.0, 0.0, c_m, c5],
              [i4, 0.0, 0.0, c_p, c5]]
    else:
        Tm = [[-1.0 * rho / T, 0.0, 0.0, t_p, t_p],
              [0.0, 0.0, 0.0, t_m, t_q],
              [0.0, 0.0, 1.0, 0.0, 0.0],
              [0.0, 1.0, 0.0, 0.0, 0.0],
              [1.0, 0.0, 0.0, 1.0, 1.0]]
        Ti = [[i1, 0.0, 0.0, 0.0, 1.0 / gam],
              [0.0, 0.0, 0.0, 1.0, 0.0],
              [0.0, 0.0, 1.0, 0.0, 0.0],
              [i4, c_m, 0.0, 0.0, c5],
              [i4, c_p, 0.0, 0.0, c5]]
    return lam, Tm, Ti


def _matvec(A, v):
    out = []
    for r_ in range(5):
        s = 0.0
        for c in range(5):
            s = s + A[r_][c] * v[c]
        out.append(s)
    return out


def _t_lam_w(Tm, lam, w):
    """MATMUL(MATMUL(T_mat, lam), w) with lam diagonal: the inner product's off-diagonal
    terms are exact zeros."""
    TL = [[0.0] * 5 for _ in range(5)]
    for r_ in range(5):
        for c in range(5):
            s = 0.0
            for k in range(5):
                s = s + Tm[r_][k] * (lam[k] if k == c else 0.0)
            TL[r_][c] = s
    return _matvec(TL, w)


def rhs(pv, tgt, tables, maps, metrics, z, r, params, patches):
    """ComputeRHS (ModRHS.f90:5-258) of a single block on the state pv: the derivatives,
    the sensor when shock capturing is on, the inviscid and viscous terms, the bc loop
    (ModBC.f90:13-277) and the sponges (:548-617). Returns rhs[5, Nr, Nz]."""
    s1, s2, tg = tables
    dxidz, detadr, ddxidxidz, ddetadetadr = metrics
    blank = maps["blank"] == 1
    zr, rr = maps["zrow"], maps["rrow"]
    gam, Re, Pr = params.gam, params.Re, params.Pr
    Nr, Nz = pv.shape[1:]
    q = assign_values(pv)
    d1z = {k: stencil(s1, q[k], zr, blank, 1, 6, 5) * dxidz for k in ("rho", "Vr", "Vt", "Vz", "T", "p")}
    d1r = {k: stencil(s1, q[k], rr, blank, 2, 6, 5) * detadr for k in ("rho", "Vr", "Vt", "Vz", "T", "p")}
    sc = params.shock_capturing == 1
    if sc:
        ms, bs, ks = sensor(pv, tables, maps, metrics, z, r, params)
        q["mu"] = q["mu"] + ms
        q["beta"] = q["beta"] + bs
        q["lam"] = q["beta"] - (2.0 / 3.0) * q["mu"]
        q["kappa"] = q["kappa"] + ks
    out = np.zeros((5, Nr, Nz))
    R = np.broadcast_to(r[:, None], (Nr, Nz))
    rho, Vr, Vt, Vz, T = q["rho"], q["Vr"], q["Vt"], q["Vz"], q["T"]
    js = slice(1, Nr)  # the axis row is skipped
    with np.errstate(divide="ignore", invalid="ignore"):
        out[0, js] = (Vr * d1r["rho"] + Vz * d1z["rho"] + rho * (d1r["Vr"] + Vr / R + d1z["Vz"]))[js]
        out[1, js] = (Vr * d1r["Vr"] + Vz * d1z["Vr"] + 1.0 / (gam * rho) * d1r["p"])[js]
        out[2, js] = (Vr * d1r["Vt"] + Vr * Vt / R + Vz * d1z["Vt"])[js]
        out[3, js] = (Vr * d1r["Vz"] + Vz * d1z["Vz"] + 1.0 / (gam * rho) * d1z["p"])[js]
        out[4, js] = (Vr * d1r["T"] + Vz * d1z["T"] + (gam - 1.0) * T * (d1r["Vr"] + Vr / R + d1z["Vz"]))[js]
    out = -1.0 * out
    if params.do_viscous_terms == 1:
        def d2(k, dirn):
            rows, met, met2, first = (zr, dxidz, ddxidxidz, d1z[k]) if dirn == 1 else (rr, detadr, ddetadetadr, d1r[k])
            return stencil(s2, q[k], rows, blank, dirn, 6, 5) * (met * met) + first * met2
        d2z = {k: d2(k, 1) for k in ("Vr", "Vt", "Vz", "T")}
        d2r = {k: d2(k, 2) for k in ("Vr", "Vt", "Vz", "T")}
        dmudz = stencil(s1, q["mu"], zr, blank, 1, 6, 5) * dxidz
        dkapdz = stencil(s1, q["kappa"], zr, blank, 1, 6, 5) * dxidz
        dmudr = stencil(s1, q["mu"], rr, blank, 2, 6, 5) * detadr
        dkapdr = stencil(s1, q["kappa"], rr, blank, 2, 6, 5) * detadr
        d2Vrdzdr = stencil(s1, d1z["Vr"], rr, blank, 2, 6, 5) * detadr
        d2Vzdzdr = stencil(s1, d1z["Vz"], rr, blank, 2, 6, 5) * detadr
        mu, kap = q["mu"], q["kappa"]
        if sc:
            tmp = q["lam"] / mu
            f43, o13, t23 = 2.0 + tmp, 1.0 + tmp, -1.0 * tmp
        else:
            f43, o13, t23 = 29.0 / 15.0, 14.0 / 15.0, 1.0 / 15.0
        with np.errstate(divide="ignore", invalid="ignore"):
            obr = 1.0 / R
        dVrdr, dVzdr, dVtdr, dTdr = d1r["Vr"], d1r["Vz"], d1r["Vt"], d1r["T"]
        dVrdz, dVzdz, dVtdz, dTdz = d1z["Vr"], d1z["Vz"], d1z["Vt"], d1z["T"]
        with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
            c = 1.0 / (Re * rho)
            v2 = c * (mu * (f43 * d2r["Vr"] + f43 * obr * dVrdr + o13 * d2Vzdzdr + d2z["Vr"] - f43 * Vr * (obr * obr))
                      + dmudr * (f43 * dVrdr - t23 * Vr * obr - t23 * dVzdz) + dmudz * (dVrdz + dVzdr))
            v3 = c * (mu * (d2r["Vt"] + d2z["Vt"] + obr * dVtdr - Vt * (obr * obr)) + dmudr * (dVtdr - Vt * obr)
                      + dmudz * dVtdz)
            v4 = c * (mu * (d2r["Vz"] + f43 * d2z["Vz"] + o13 * d2Vrdzdr + obr * dVzdr + o13 * obr * dVrdz)
                      + dmudr * (dVzdr + dVrdz) + dmudz * (f43 * dVzdz - t23 * dVrdr - t23 * Vr * obr))
            x5 = gam / (Re * Pr * rho) * (kap * (d2r["T"] + obr * dTdr + d2z["T"]) + dkapdr * dTdr + dkapdz * dTdz)
            y5 = gam * (gam - 1.0) / Re * mu / rho * (
                dVrdr * (f43 * dVrdr - t23 * Vr * obr - t23 * dVzdz) + (dVtdr - Vt * obr) * (dVtdr - Vr * obr)
                + Vr * obr * (f43 * Vr * obr - t23 * dVrdr - t23 * dVzdz) + dVtdz * dVtdz
                + dVzdz * (f43 * dVzdz - t23 * dVrdr - t23 * Vr * obr) + (dVrdz + dVzdr) * (dVzdr + dVrdz))
        out[1, js] = (out[1] + v2)[js]
        out[2, js] = (out[2] + v3)[js]
        out[3, js] = (out[3] + v4)[js]
        out[4, js] = (out[4] + x5 + y5)[js]
    if params.control_forcing == 1:
        _control_forcing(out, pv, tgt, z, r, params)
    _bc_loop(out, pv, tgt, q, d1z, d1r, dxidz, detadr, gam, patches)
    _sponges(out, pv, tgt, z, r, params)
    return out


def _control_forcing(out, pv, tgt, z, r, params):
    """ControlForcingTerms (ModControlForcing.f90:43-61), with the matrix and the Gaussian
    window from the parameters instead of Vz_Control_Vr_Feedback.dat."""
    F = [params.forcing_mat[q] for q in range(25)]
    Nr, Nz = pv.shape[1:]
    for i in range(Nz):
        for j in range(Nr):
            dz, dr = z[i] - params.forcing_z0, r[j] - params.forcing_r0
            G = math.exp(-((dz * dz) / (params.forcing_lz * params.forcing_lz))
                         - (dr * dr) / (params.forcing_lr * params.forcing_lr))
            for e in range(5):
                for k in range(5):
                    out[e, j, i] = out[e, j, i] + params.forcing_alpha * F[5 * e + k] * G * (pv[k, j, i] - tgt[k, j, i])


def _bc_loop(out, pv, tgt, q, d1z, d1r, dxidz, detadr, gam, patches):
    """BoundaryConditions (ModBC.f90:13-277) for one block: patches in order, the face
    line of each, SAT (compute_SAT_RHS :439-469) and NSCBC (ComputeNSCBCRHS :471-545)."""
    sigma_1 = sigma_2 = -2.0
    one_by_h_44 = 48.0 / 49.0
    Nr, Nz = pv.shape[1:]
    for (i_s, i_e, j_s, j_e, bc, d) in patches:
        if bc == AXIS:
            continue
        if d == 1:
            ii, jj = (i_s, i_s), (j_s, j_e)
        elif d == -1:
            ii, jj = (i_e, i_e), (j_s, j_e)
        elif d == 2:
            ii, jj = (i_s, i_e), (j_s, j_s)
        else:
            ii, jj = (i_s, i_e), (j_e, j_e)
        adir = abs(d)
        for i1 in range(ii[0], ii[1] + 1):
            for j1 in range(jj[0], jj[1] + 1):
                i, j = i1 - 1, j1 - 1
                rho, Vr, Vz, T = q["rho"][j, i], q["Vr"][j, i], q["Vz"][j, i], q["T"][j, i]
                pvl = [pv[e, j, i] for e in range(5)]
                if bc == SAT_FARFIELD:
                    if j1 == 1 or adir != 1:
                        continue
                    lam, Tm, Ti = _eigen(rho, Vz, T, gam, False)
                    lam = [(abs(v) + v) / 2.0 if d > 0 else (abs(v) - v) / 2.0 for v in lam]
                    w = _matvec(Ti, [pvl[e] - tgt[e, j, i] for e in range(5)])
                    sat = _t_lam_w(Tm, lam, w)
                    for e in range(5):
                        out[e, j, i] = out[e, j, i] + sigma_1 * dxidz[j, i] * one_by_h_44 * sat[e]
                elif bc == SAT_NOSLIP_WALL:
                    rd = adir == 2
                    tI = list(pvl)
                    tI[1 if rd else 3] = 0.0
                    lam, Tm, Ti = _eigen(rho, Vr if rd else Vz, T, gam, rd)
                    lam = [(abs(v) + v) / 2.0 if d > 0 else (abs(v) - v) / 2.0 for v in lam]
                    w = _matvec(Ti, [pvl[e] - tI[e] for e in range(5)])
                    sat = _t_lam_w(Tm, lam, w)
                    met = detadr[j, i] if rd else dxidz[j, i]
                    for e in range(5):
                        out[e, j, i] = out[e, j, i] + sigma_1 * met * one_by_h_44 * sat[e]
                    tV = [pvl[0], 0.0, 0.0, 0.0, tgt[4, j, i]]
                    for e in range(5):
                        out[e, j, i] = out[e, j, i] + sigma_2 * met * one_by_h_44 * (pvl[e] - tV[e])
                elif bc == NSCBC_NONREFLECTING:
                    if j1 == 1:
                        continue
                    g = {k: (d1z[k][j, i], d1r[k][j, i]) for k in ("rho", "Vr", "Vt", "Vz", "T", "p")}
                    if adir == 1:
                        add = [Vz * g["rho"][0] + rho * g["Vz"][0], Vz * g["Vr"][0], Vz * g["Vt"][0],
                               Vz * g["Vz"][0] + 1.0 / (gam * rho) * g["p"][0], Vz * g["T"][0] + (gam - 1.0) * T * g["Vz"][0]]
                        lam, Tm, Ti = _eigen(rho, Vz, T, gam, False)
                    else:
                        add = [Vr * g["rho"][1] + rho * g["Vr"][1], Vr * g["Vr"][1] + 1.0 / (gam * rho) * g["p"][1],
                               Vr * g["Vt"][1], Vr * g["Vz"][1], Vr * g["T"][1] + (gam - 1.0) * T * g["Vr"][1]]
                        lam, Tm, Ti = _eigen(rho, Vr, T, gam, True)
                    for e in range(5):
                        out[e, j, i] = out[e, j, i] + add[e]
                    # the non-reflecting face takes z-derivatives in both directions (:487-493)
                    w = _matvec(Ti, [g[k][0] for k in ("rho", "Vr", "Vt", "Vz", "T")])
                    w = [0.0 if ((d > 0 and lam[e] > 0.0) or (d < 0 and lam[e] < 0.0)) else w[e] for e in range(5)]
                    ns = _t_lam_w(Tm, lam, w)
                    for e in range(5):
                        out[e, j, i] = out[e, j, i] - ns[e]
                elif bc == NSCBC_NOSLIP_WALL:
                    rd = adir == 2
                    lam, Tm, Ti = _eigen(rho, Vr if rd else Vz, T, gam, rd)
                    dv = [(d1r if rd else d1z)[k][j, i] for k in ("rho", "Vr", "Vt", "Vz", "T")]
                    w = _matvec(Ti, dv)
                    if d < 0:
                        w[3] = -1.0 * w[4]
                    else:
                        w[4] = -1.0 * w[3]
                    ns = _t_lam_w(Tm, lam, w)
                    if rd:
                        out[0, j, i] = out[0, j, i] + (Vr * d1r["rho"][j, i] + rho * d1r["Vr"][j, i])
                    else:
                        out[0, j, i] = out[0, j, i] + (Vz * d1z["rho"][j, i] + rho * d1z["Vz"][j, i])
                    for e in range(5):
                        out[e, j, i] = out[e, j, i] - ns[e]
                    out[1:, j, i] = 0.0


def _sponges(out, pv, tgt, z, r, params):
    """sponge_bcs (ModBC.f90:548-617): the top sponge on every row, the inflow sponge from
    row 2 (the axis rank), zeta**n_sponge with the real exponent 2.0 (libm pow)."""
    st, At, el, Al = params.sponge_start_top, params.sponge_A_top, params.sponge_end_left, params.sponge_A_left
    Nr, Nz = pv.shape[1:]
    for i in range(Nz):
        for j in range(Nr):
            if r[j] >= st:
                for e in range(5):
                    zeta = (r[j] - st) / (r[Nr - 1] - st)
                    out[e, j, i] = out[e, j, i] - At * math.pow(zeta, 2.0) * (pv[e, j, i] - tgt[e, j, i])
    for i in range(Nz):
        for j in range(1, Nr):
            if z[i] <= el:
                for e in range(5):
                    zeta = (el - z[i]) / el
                    out[e, j, i] = out[e, j, i] - Al * math.pow(zeta, 2.0) * (pv[e, j, i] - tgt[e, j, i])


def axis_conditions(pv, prim, s1):
    """axis_conditions (ModAxis.f90:5-35): row 1 of rho, V_z, T from rows 2..6 of the
    primitives of the previous AssignValues (the stage input), into pv."""
    for k, e in (("rho", 0), ("Vz", 3), ("T", 4)):
        f = prim[k]
        col = np.zeros(f.shape[1])
        for i in range(f.shape[1]):
            d = 0.0
            for m in range(1, 6):
                d = d + s1[0][m] * f[m, i]
            col[i] = -1.0 * d / s1[0][0]
        pv[e, 0, :] = col


def rk4(pv, tgt, delt, tables, maps, metrics, z, r, params, patches):
    """RK4 (ModRungeKutta.f90:5-171): k_s = delt*rhs, stages pv_old + 0.5 k1, + 0.5 k2,
    + k3, each followed by axis_conditions on the stage input's primitives; the final
    update skips blanked points."""
    pv_old = pv.copy()
    cur = pv.copy()
    ks = []
    for s, a in enumerate((0.5, 0.5, 1.0, None)):
        prim = assign_values(cur)
        k = delt * rhs(cur, tgt, tables, maps, metrics, z, r, params, patches)
        ks.append(k)
        if a is not None:
            cur = pv_old + a * k if a != 1.0 else pv_old + k
            axis_conditions(cur, prim, tables[0])
    prim = assign_values(cur)
    new = pv_old + 1.0 / 6.0 * ks[0] + 1.0 / 3.0 * (ks[1] + ks[2]) + 1.0 / 6.0 * ks[3]
    blank = maps["blank"] == 1
    new[:, blank] = cur[:, blank]
    axis_conditions(new, prim, tables[0])
    return new


def compute_time_step(pv, blank, metrics, params, stale_T=None):
    """ComputeTimeStep (ModInputOutput.f90:389-438) of a single block: the CFL step of
    every point (100 at blanked points) with the scalar stale_T, or the local T where
    stale_T is None, and its minimum."""
    q = assign_values(pv)
    dxidz, detadr = metrics[0], metrics[1]
    Re, Pr, CFL = params.Re, params.Pr, params.CFL
    best = math.inf
    Nr, Nz = pv.shape[1:]
    for i in range(Nz):
        for j in range(Nr):
            if blank[j, i]:
                d = 100.0
            else:
                x, y = dxidz[j, i], detadr[j, i]
                Ts = q["T"][j, i] if stale_T is None else stale_T
                inv = abs(q["Vz"][j, i] * x + q["Vr"][j, i] * y) + math.sqrt(Ts) * math.sqrt(x * x + y * y)
                s = abs(x) + abs(y)
                visc = 2.0 * max(q["mu"][j, i] / Re, q["lam"][j, i] / Re, q["kappa"][j, i] / (Re * Pr)) * (s * s)
                d = CFL / (inv + visc)
            best = min(best, d)
    return best


def compute_metric_1d(s1, x):
    """ComputeMetric (ModDeriv.f90:241-382) along one coordinate line of a single block
    (every neighbour is MPI_PROC_NULL): SBP1 closure rows on the 4 points at each end,
    the centred row between."""
    n = len(x)
    out = np.zeros(n)
    for i in range(n):
        if i < 4:
            row, w0, m = i, 0, 6
        elif i >= n - 4:
            row, w0, m = 8 - (n - 1) + i, n - 6, 6
        else:
            row, w0, m = 4, i - 2, 5
        out[i] = dot(s1[row], x, w0, m)
    return out


def metrics(s1, z, r):
    """dxi/dz, deta/dr and their derivatives as ModSolver.f90:56-73 forms them:
    (dxidz, detadr, ddxidxidz, ddetadetadr) on the (Nr, Nz) grid."""
    dxidz = 1.0 / compute_metric_1d(s1, z)
    detadr = 1.0 / compute_metric_1d(s1, r)
    dd_z = compute_metric_1d(s1, dxidz)
    dd_r = compute_metric_1d(s1, detadr)
    Nz, Nr = len(z), len(r)
    b = lambda v, ax: np.broadcast_to(v[None, :] if ax == 1 else v[:, None], (Nr, Nz)).copy()
    return b(dxidz, 1), b(detadr, 2), b(dd_z, 1), b(dd_r, 2)


def create_patches(records, Nz, Nr):
    """CreateAllPatches + PatchCreation (ModPatch.f90:117-309) for a single block holding
    the grid: -1 indices resolved to the grid size, each face widened to its 4-wide strip,
    the strip's first and last points inside the block found in the block's loop order
    (i outer, j inner), a patch kept when any point of the block lies in its strip.
    Returns (i_start, i_end, j_start, j_end, bc, bc_dir) tuples."""
    out = []
    for bc, d, bis, bie, bjs, bje in records:
        bis = Nz if bis == -1 else bis
        bjs = Nr if bjs == -1 else bjs
        bie = Nz if bie == -1 else bie
        bje = Nr if bje == -1 else bje
        if d == 1:
            ps, pe, qs, qe = bis, bis + 3, bjs, bje
        elif d == -1:
            ps, pe, qs, qe = bie - 3, bie, bjs, bje
        elif d == 2:
            ps, pe, qs, qe = bis, bie, bjs, bjs + 3
        else:
            ps, pe, qs, qe = bis, bie, bje - 3, bje
        found = 0
        s_i = s_j = e_i = e_j = 0
        for i in range(1, Nz + 1):
            for j in range(1, Nr + 1):
                if (i - ps) * (i - pe) <= 0 and (j - qs) * (j - qe) <= 0:
                    if not found:
                        s_i, s_j, found = i, j, 1
                    else:
                        e_i, e_j = i, j
        if not found:
            continue
        if d == 1:
            p = (s_i, s_i + 3, s_j, e_j)
        elif d == -1:
            p = (e_i - 3, e_i, s_j, e_j)
        elif d == 2:
            p = (s_i, e_i, s_j, s_j + 3)
        else:
            p = (s_i, e_i, e_j - 3, e_j)
        out.append(p + (bc, d))
    return out
