// axj_point.cuh -- pointwise physics of one grid point: inviscid and viscous
// right-hand side, SAT/NSCBC face operations, sponges, control forcing and the
// CFL time step. Every expression keeps the reference's operand order
// (left-to-right as written in the Fortran source), so the device result
// differs from a CPU evaluation of the same source only by FMA contraction and
// libm ulps.
#pragma once

#include "axj_common.cuh"

namespace axj {

// Primitive state at a point (pv(i,j,1,1:5) = rho, V_r, V_theta, V_z, T) plus the
// transport coefficients after AssignValues / UpdateTransportCoeffs, in arithmetic
// type R (double on the FP64 path; float for the interior of the mixed path).
template <typename R>
struct PrimT {
  R rho, Vr, Vt, Vz, T;
  R mu, kappa, lambda;
};

// The 26 derivative values ComputeRHS forms at a point (ModRHS.f90:29-41, :118-133).
template <typename R>
struct DerivT {
  R drhodz, dVrdz, dVtdz, dVzdz, dTdz, dpdz, dmudz, dkappadz;
  R drhodr, dVrdr, dVtdr, dVzdr, dTdr, dpdr, dmudr, dkappadr;
  R d2Vrdz2, d2Vtdz2, d2Vzdz2, d2Tdz2;
  R d2Vrdr2, d2Vtdr2, d2Vzdr2, d2Tdr2;
  R d2Vrdzdr, d2Vzdzdr;
};
using Prim = PrimT<double>;
using Deriv = DerivT<double>;

template <typename RO, typename RI>
AXJ_HD PrimT<RO> convert(const PrimT<RI>& q) {
  return PrimT<RO>{RO(q.rho), RO(q.Vr), RO(q.Vt), RO(q.Vz), RO(q.T), RO(q.mu), RO(q.kappa), RO(q.lambda)};
}
template <typename RO, typename RI>
AXJ_HD DerivT<RO> convert(const DerivT<RI>& d) {
  return DerivT<RO>{RO(d.drhodz),  RO(d.dVrdz),   RO(d.dVtdz),   RO(d.dVzdz),   RO(d.dTdz),    RO(d.dpdz),
                    RO(d.dmudz),   RO(d.dkappadz), RO(d.drhodr),  RO(d.dVrdr),   RO(d.dVtdr),   RO(d.dVzdr),
                    RO(d.dTdr),    RO(d.dpdr),    RO(d.dmudr),   RO(d.dkappadr), RO(d.d2Vrdz2), RO(d.d2Vtdz2),
                    RO(d.d2Vzdz2), RO(d.d2Tdz2),  RO(d.d2Vrdr2), RO(d.d2Vtdr2), RO(d.d2Vzdr2), RO(d.d2Tdr2),
                    RO(d.d2Vrdzdr), RO(d.d2Vzdzdr)};
}

// Per-point reciprocals and per-run constants of the right-hand side: the reference
// divides by r, rho, gam*rho, Re*rho and Re*Pr*rho at every point (about ten FP64
// divisions); here 1/r comes from a per-row table, 1/rho is formed once and the
// constant factors once per run. The products differ from the quotients by rounding.
template <typename R>
struct RhsConst {
  R gam, inv_gam, gam_m1, inv_Re, gam_RePr, gg1_Re;  // gam, 1/gam, gam-1, 1/Re, gam/(Re Pr), gam(gam-1)/Re
};
template <typename R>
AXJ_HD RhsConst<R> rhs_const(double gam, double Re, double Pr) {
  return RhsConst<R>{R(gam), R(1.0 / gam), R(gam - 1.0), R(1.0 / Re), R(gam / (Re * Pr)), R(gam * (gam - 1.0) / Re)};
}
// The same factors from the values the host formed once per run (Consts), so that no
// division is left in the per-point code.
template <typename R>
AXJ_HD RhsConst<R> rhs_const(const Consts& c) {
  return RhsConst<R>{R(c.gam), R(c.inv_gam), R(c.gam - 1.0), R(c.inv_Re), R(c.gam_RePr), R(c.gg1_Re)};
}

// Inviscid part, already negated (ModRHS.f90:92-96 and :103-113).
template <typename R>
AXJ_HD void rhs_inviscid(const PrimT<R>& q, const DerivT<R>& d, R onebyr, R inv_rho, const RhsConst<R>& k, R rhs[5]) {
  const R mone = R(-1.0);
  const R rho = q.rho, Vr = q.Vr, Vt = q.Vt, Vz = q.Vz, T = q.T;
  const R Vr_r = Vr * onebyr;
  const R igr = k.inv_gam * inv_rho;
  R r1 = Vr * d.drhodr + Vz * d.drhodz + rho * (d.dVrdr + Vr_r + d.dVzdz);
  R r2 = Vr * d.dVrdr + Vz * d.dVrdz + igr * d.dpdr;
  R r3 = Vr * d.dVtdr + Vt * Vr_r + Vz * d.dVtdz;
  R r4 = Vr * d.dVzdr + Vz * d.dVzdz + igr * d.dpdz;
  R r5 = Vr * d.dTdr + Vz * d.dTdz + k.gam_m1 * T * (d.dVrdr + Vr_r + d.dVzdz);
  rhs[0] = mone * r1;
  rhs[1] = mone * r2;
  rhs[2] = mone * r3;
  rhs[3] = mone * r4;
  rhs[4] = mone * r5;
}

// Viscous S_r, S_theta, S_z, S_T (ModRHS.f90:135-209). With shock capturing the
// per-point constants come from lambda/mu (:180-188).
template <typename R>
AXJ_HD void rhs_viscous(const PrimT<R>& q, const DerivT<R>& d, R onebyr, R inv_rho, const RhsConst<R>& k, bool sc,
                        R rhs[5]) {
  const R one = R(1.0);
  R fourby3 = R(29.0 / 15.0), oneby3 = R(14.0 / 15.0), twoby3 = R(1.0 / 15.0);
  const R Vr = q.Vr, Vt = q.Vt, mu = q.mu, kappa = q.kappa;
  if (sc) {
    R tmp = q.lambda / q.mu;
    fourby3 = R(2.0) + tmp;
    oneby3 = one + tmp;
    twoby3 = R(-1.0) * tmp;
  }
  const R iRr = k.inv_Re * inv_rho;  // 1/(Re rho)
  rhs[1] = rhs[1] + iRr *
                        (mu * (fourby3 * d.d2Vrdr2 + fourby3 * onebyr * d.dVrdr + oneby3 * d.d2Vzdzdr + d.d2Vrdz2 -
                               fourby3 * Vr * (onebyr * onebyr)) +
                         d.dmudr * (fourby3 * d.dVrdr - twoby3 * Vr * onebyr - twoby3 * d.dVzdz) +
                         d.dmudz * (d.dVrdz + d.dVzdr));
  rhs[2] = rhs[2] + iRr *
                        (mu * (d.d2Vtdr2 + d.d2Vtdz2 + onebyr * d.dVtdr - Vt * (onebyr * onebyr)) +
                         d.dmudr * (d.dVtdr - Vt * onebyr) + d.dmudz * d.dVtdz);
  rhs[3] = rhs[3] + iRr *
                        (mu * (d.d2Vzdr2 + fourby3 * d.d2Vzdz2 + oneby3 * d.d2Vrdzdr + onebyr * d.dVzdr +
                               oneby3 * onebyr * d.dVrdz) +
                         d.dmudr * (d.dVzdr + d.dVrdz) +
                         d.dmudz * (fourby3 * d.dVzdz - twoby3 * d.dVrdr - twoby3 * Vr * onebyr));
  rhs[4] = rhs[4] +
           k.gam_RePr * inv_rho *
               (kappa * (d.d2Tdr2 + onebyr * d.dTdr + d.d2Tdz2) + d.dkappadr * d.dTdr + d.dkappadz * d.dTdz) +
           k.gg1_Re * mu * inv_rho *
               (d.dVrdr * (fourby3 * d.dVrdr - twoby3 * Vr * onebyr - twoby3 * d.dVzdz) +
                (d.dVtdr - Vt * onebyr) * (d.dVtdr - Vr * onebyr) +
                Vr * onebyr * (fourby3 * Vr * onebyr - twoby3 * d.dVrdr - twoby3 * d.dVzdz) + d.dVtdz * d.dVtdz +
                d.dVzdz * (fourby3 * d.dVzdz - twoby3 * d.dVrdr - twoby3 * Vr * onebyr) +
                (d.dVrdz + d.dVzdr) * (d.dVzdr + d.dVrdz));
}

// mu = T**0.666 (ModAssign.f90:20) as exp2(0.666 log2 T): within a few ulp of pow. The
// FP32 stencils and the allocation-free dt use it; the FP64 kernels use the table-driven
// pow0666 (axj_pow.cuh).
template <typename R>
AXJ_HD R mu_of_T(R T);
template <>
AXJ_HD double mu_of_T<double>(double T) { return exp2(0.666 * log2(T)); }
template <>
AXJ_HD float mu_of_T<float>(float T) { return exp2f(0.666f * log2f(T)); }

// ---------------------------------------------------------------------------
// Characteristic algebra of ModBC.f90:280-545 for primitive variables.
// T_mat, T_mat_inv and Lambda are sparse; each product below is the
// corresponding MATMUL row with its zero terms dropped, the non-zero terms kept
// in column order (adding +-0 to a running sum does not change it).
// ---------------------------------------------------------------------------
struct Eig {
  double lam[5];
  double t11, t14, t15, ta, tb;      // T_mat (1,1),(1,4),(1,5) and the +-1/((g-1)sqrt T) pair
  double i11, i15, i41, i4c, i45;    // T_mat_inv (1,1),(1,5),(4,1),(4,4|2),(4,5)
};

// eigen_matrices_in_z_direction (:280-358) with U = V_z, or _in_r_direction (:360-437)
// with U = V_r; the two differ only in where the entries sit.
AXJ_HD void eigen_matrices(double rho, double U, double T, double gam, Eig& e) {
  e.lam[0] = U;
  e.lam[1] = U;
  e.lam[2] = U;
  e.lam[3] = (U - sqrt(T));
  e.lam[4] = (U + sqrt(T));
  e.t11 = -1.0 * rho / T;
  e.t14 = rho / ((gam - 1.0) * T);
  e.t15 = rho / ((gam - 1.0) * T);
  e.ta = -1.0 / ((gam - 1.0) * sqrt(T));
  e.tb = 1.0 / ((gam - 1.0) * sqrt(T));
  e.i11 = -1.0 * (gam - 1.0) * T / (gam * rho);
  e.i15 = 1.0 / gam;
  e.i41 = (gam - 1.0) * T / (2.0 * gam * rho);
  e.i4c = -1.0 * (gam - 1.0) * sqrt(T) / 2.0;
  e.i45 = (gam - 1.0) / (2.0 * gam);
}

// w = MATMUL(T_mat_inv, v)
AXJ_HD void apply_tinv(bool rdir, const Eig& e, const double v[5], double w[5]) {
  const double i5c = -e.i4c;  // (5,4|2) = (g-1) sqrt(T)/2, the exact negative of (4,4|2)
  const double vc = rdir ? v[1] : v[3];
  double w1 = e.i11 * v[0] + e.i15 * v[4];
  double w2 = rdir ? v[3] : v[2];
  double w3 = rdir ? v[2] : v[1];
  double w4 = e.i41 * v[0] + e.i4c * vc + e.i45 * v[4];
  double w5 = e.i41 * v[0] + i5c * vc + e.i45 * v[4];
  w[0] = w1; w[1] = w2; w[2] = w3; w[3] = w4; w[4] = w5;
}

// out = MATMUL(MATMUL(T_mat, lam), w) with lam = diag(l).
AXJ_HD void apply_tlam(bool rdir, const Eig& e, const double l[5], const double w[5], double out[5]) {
  double o1 = (e.t11 * l[0]) * w[0] + (e.t14 * l[3]) * w[3] + (e.t15 * l[4]) * w[4];
  double oab = (e.ta * l[3]) * w[3] + (e.tb * l[4]) * w[4];
  double o5 = l[0] * w[0] + l[3] * w[3] + l[4] * w[4];
  if (!rdir) {
    out[0] = o1; out[1] = l[2] * w[2]; out[2] = l[1] * w[1]; out[3] = oab; out[4] = o5;
  } else {
    out[0] = o1; out[1] = oab; out[2] = l[2] * w[2]; out[3] = l[1] * w[1]; out[4] = o5;
  }
}

// compute_SAT_RHS (:439-469): rhs_SAT = T Lambda^{+/-} T^{-1} (pv - target).
AXJ_HD void sat_term(bool rdir, int bc_dir, const Eig& e, const double pv[5], const double tg[5], double out[5]) {
  double l[5];
  for (int q = 0; q < 5; ++q)
    l[q] = bc_dir > 0 ? (fabs(e.lam[q]) + e.lam[q]) / 2.0 : (fabs(e.lam[q]) - e.lam[q]) / 2.0;
  double v[5], w[5];
  for (int q = 0; q < 5; ++q) v[q] = pv[q] - tg[q];
  apply_tinv(rdir, e, v, w);
  apply_tlam(rdir, e, l, w, out);
}

// One boundary-patch operation at a face point (BoundaryConditions, ModBC.f90:25-274),
// added to rhs in place. j1 marks the axis row j = 1, which the far-field and
// non-reflecting faces skip (:60-62, :148-150).
AXJ_HD void face_op(int bc, int bc_dir, bool j1, const Prim& q, const Deriv& d, const double tgt[5],
                    double dxidz, double detadr, double gam, double rhs[5]) {
  const double sigma_1 = -2.0, sigma_2 = -2.0, one_by_h_44 = 48.0 / 49.0;
  const int adir = bc_dir < 0 ? -bc_dir : bc_dir;
  const double pv[5] = {q.rho, q.Vr, q.Vt, q.Vz, q.T};
  Eig e;
  double out[5];
  if (bc == 91) {  // SAT_FARFIELD (:54-79), z-faces only
    if (j1 || adir != 1) return;
    eigen_matrices(q.rho, q.Vz, q.T, gam, e);
    sat_term(false, bc_dir, e, pv, tgt, out);
    for (int k = 0; k < 5; ++k) rhs[k] = rhs[k] + sigma_1 * dxidz * one_by_h_44 * out[k];
  } else if (bc == 93) {  // SAT_NOSLIP_WALL (:82-140)
    if (adir != 1 && adir != 2) return;
    const bool rd = adir == 2;
    const double tI[5] = {pv[0], rd ? 0.0 : pv[1], pv[2], rd ? pv[3] : 0.0, pv[4]};
    eigen_matrices(q.rho, rd ? q.Vr : q.Vz, q.T, gam, e);
    sat_term(rd, bc_dir, e, pv, tI, out);
    const double met = rd ? detadr : dxidz;
    for (int k = 0; k < 5; ++k) rhs[k] = rhs[k] + sigma_1 * met * one_by_h_44 * out[k];
    const double tV[5] = {pv[0], 0.0, 0.0, 0.0, tgt[4]};
    for (int k = 0; k < 5; ++k) rhs[k] = rhs[k] + sigma_2 * met * one_by_h_44 * (pv[k] - tV[k]);
  } else if (bc == 92) {  // NSCBC_NONREFLECTING (:142-213)
    if (j1) return;
    const double rho = q.rho, Vr = q.Vr, Vz = q.Vz, T = q.T;
    bool rd;
    if (adir == 1) {
      rhs[0] = rhs[0] + (Vz * d.drhodz + rho * d.dVzdz);
      rhs[1] = rhs[1] + Vz * d.dVrdz;
      rhs[2] = rhs[2] + Vz * d.dVtdz;
      rhs[3] = rhs[3] + (Vz * d.dVzdz + 1.0 / (gam * rho) * d.dpdz);
      rhs[4] = rhs[4] + (Vz * d.dTdz + (gam - 1.0) * T * d.dVzdz);
      rd = false;
      eigen_matrices(rho, Vz, T, gam, e);
    } else if (adir == 2) {
      rhs[0] = rhs[0] + (Vr * d.drhodr + rho * d.dVrdr);
      rhs[1] = rhs[1] + (Vr * d.dVrdr + 1.0 / (gam * rho) * d.dpdr);
      rhs[2] = rhs[2] + Vr * d.dVtdr;
      rhs[3] = rhs[3] + Vr * d.dVzdr;
      rhs[4] = rhs[4] + (Vr * d.dTdr + (gam - 1.0) * T * d.dVrdr);
      rd = true;
      eigen_matrices(rho, Vr, T, gam, e);
    } else {
      return;
    }
    // ComputeNSCBCRHS (:487-511): the non-reflecting face uses the z-derivative
    // vector for both face orientations, as the reference does.
    const double dv[5] = {d.drhodz, d.dVrdz, d.dVtdz, d.dVzdz, d.dTdz};
    double w[5];
    apply_tinv(rd, e, dv, w);
    for (int k = 0; k < 5; ++k) {
      if (bc_dir > 0) { if (e.lam[k] > 0.0) w[k] = 0.0; }
      else if (bc_dir < 0) { if (e.lam[k] < 0.0) w[k] = 0.0; }
    }
    apply_tlam(rd, e, e.lam, w, out);
    for (int k = 0; k < 5; ++k) rhs[k] = rhs[k] - out[k];
  } else if (bc == 94) {  // NSCBC_NOSLIP_WALL (:218-267)
    const double rho = q.rho, Vr = q.Vr, Vz = q.Vz;
    double dv[5];
    bool rd;
    if (adir == 1) {
      rd = false;
      eigen_matrices(rho, Vz, q.T, gam, e);
      dv[0] = d.drhodz; dv[1] = d.dVrdz; dv[2] = d.dVtdz; dv[3] = d.dVzdz; dv[4] = d.dTdz;
    } else if (adir == 2) {
      rd = true;
      eigen_matrices(rho, Vr, q.T, gam, e);
      dv[0] = d.drhodr; dv[1] = d.dVrdr; dv[2] = d.dVtdr; dv[3] = d.dVzdr; dv[4] = d.dTdr;
    } else {
      return;
    }
    double w[5];
    apply_tinv(rd, e, dv, w);
    if (bc_dir < 0) w[3] = -1.0 * w[4];
    else if (bc_dir > 0) w[4] = -1.0 * w[3];
    apply_tlam(rd, e, e.lam, w, out);
    if (!rd) rhs[0] = rhs[0] + (Vz * d.drhodz + rho * d.dVzdz);
    else rhs[0] = rhs[0] + (Vr * d.drhodr + rho * d.dVrdr);
    for (int k = 0; k < 5; ++k) rhs[k] = rhs[k] - out[k];
    rhs[1] = 0.0; rhs[2] = 0.0; rhs[3] = 0.0; rhs[4] = 0.0;
  }
}

// Does face operation (bc, bc_dir) at a point assign the module scalar T?
// (ModBC.f90:156, eigen routines :287, :367.)
AXJ_HD bool face_op_sets_T(int bc, int bc_dir, bool j1) {
  const int adir = bc_dir < 0 ? -bc_dir : bc_dir;
  if (bc == 91) return !j1 && adir == 1;
  if (bc == 93) return adir == 1 || adir == 2;
  if (bc == 92) return !j1;
  if (bc == 94) return adir == 1 || adir == 2;
  return false;
}

// sponge_bcs (ModBC.f90:548-617). zeta**2.0 is evaluated as zeta*zeta.
AXJ_HD void sponge(double z, double r, bool j1, const Consts& c, const double pv[5], const double tg[5],
                   double rhs[5]) {
  if (r >= c.sponge_start_top) {
    double zeta = (r - c.sponge_start_top) / (c.r_top - c.sponge_start_top);
    double f = c.sponge_A_top * (zeta * zeta);
    for (int k = 0; k < 5; ++k) rhs[k] = rhs[k] - f * (pv[k] - tg[k]);
  }
  if (!j1 && z <= c.sponge_end_left) {
    double zeta = (c.sponge_end_left - z) / (c.sponge_end_left);
    double f = c.sponge_A_left * (zeta * zeta);
    for (int k = 0; k < 5; ++k) rhs[k] = rhs[k] - f * (pv[k] - tg[k]);
  }
}

// ControlForcingTerms (ModControlForcing.f90:45-61); F is row-major 5x5.
AXJ_HD void control_forcing(double z, double r, const Consts& c, const double* F, const double pv[5],
                            const double tg[5], double rhs[5]) {
  double dz = z - c.forcing_z0, dr = r - c.forcing_r0;
  double G = exp(-((dz * dz) / (c.forcing_lz * c.forcing_lz)) - (dr * dr) / (c.forcing_lr * c.forcing_lr));
  for (int e = 0; e < 5; ++e)
    for (int k = 0; k < 5; ++k) rhs[e] = rhs[e] + c.forcing_alpha * F[e * 5 + k] * G * (pv[k] - tg[k]);
}

// Harmonic inflow forcing (control_forcing = 2, an extension; the reference's
// ControlForcingTerms is the feedback above): rhs(V_z) += A omega G cos(omega t) in the
// same Gaussian window, a V_z fluctuation of amplitude A G.
// cwt = cos(omega t) of the stage, evaluated once per launch.
AXJ_HD void harmonic_forcing(double z, double r, double cwt, const Consts& c, double rhs[5]) {
  double dz = z - c.forcing_z0, dr = r - c.forcing_r0;
  double G = exp(-((dz * dz) / (c.forcing_lz * c.forcing_lz)) - (dr * dr) / (c.forcing_lr * c.forcing_lr));
  rhs[3] = rhs[3] + c.harm_amp * c.harm_omega * G * cwt;
}

// Per-point dt of ComputeTimeStep (ModInputOutput.f90:395-416).
AXJ_HD double dt_point(double Vz, double Vr, double Ts, double mu, double lambda, double kappa, double dxidz,
                       double detadr, const Consts& c) {
  double inv = fabs(Vz * dxidz + Vr * detadr) + sqrt(Ts) * sqrt(dxidz * dxidz + detadr * detadr);
  double a = mu / c.Re, b = lambda / c.Re, k = kappa / (c.Re * c.Pr);
  double mx = a;
  if (b > mx) mx = b;
  if (k > mx) mx = k;
  double s = fabs(dxidz) + fabs(detadr);
  double visc = 2.0 * mx * (s * s);
  return c.CFL / (inv + visc);
}

}  // namespace axj
