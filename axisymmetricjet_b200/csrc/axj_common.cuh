// axj_common.cuh -- shared definitions of the B200 hot path: operator tables,
// per-point stencil descriptors and launch constants.
#pragma once

#include <cstdint>
#include <cmath>

#if defined(__CUDACC__)
#define AXJ_HD __host__ __device__ __forceinline__
#else
#define AXJ_HD inline
#endif

namespace axj {

// ---------------------------------------------------------------------------
// Tile geometry of the fused stage kernel: TZ points along z (one warp wide, so
// every global row access is a coalesced 256-byte line) by TR points along r.
// ---------------------------------------------------------------------------
constexpr int TZ = 32;
constexpr int TR = 16;
constexpr int STAGE_THREADS = 256;

// Halo of the two tile classes. Interior tiles only use the interior SBP rows
// (reach 2); general tiles (domain edges, patch strips, blanked points, face
// points) use patch-selected closure rows whose windows reach 5 points.
constexpr int H_INT = 2;
constexpr int H_GEN = 5;
// Halo of the strain-rate / temperature / dilatation fields in the sensor kernel:
// two SBP2 reaches (fourth derivative as SBP2 of SBP2).
constexpr int SENS_HS_INT = 2 * H_INT;
constexpr int SENS_HS_GEN = 2 * H_GEN;
// z halo rounded up to an even count so every smem row starts 16-byte aligned
// relative to the global row.
constexpr int hz_of(int h) { return (h + 1) & ~1; }

// ---------------------------------------------------------------------------
// Per-point descriptor (uint32):
//   bits 0-3  : z stencil code 0..8 = SBP row (4 = interior), 9 = no derivative
//   bits 4-7  : r stencil code
//   bit  8    : blanked point (ibval == 0)
//   bits 12-31: index into the face-operation list (0 = no face operation)
// A point whose row code is 9 gets a zero derivative (ModDeriv.f90:14,23: out = 0
// and CYCLE for ibval == 0).
// ---------------------------------------------------------------------------
constexpr uint32_t ROW_NONE = 9u;
AXJ_HD int desc_zrow(uint32_t d) { return (int)(d & 15u); }
AXJ_HD int desc_rrow(uint32_t d) { return (int)((d >> 4) & 15u); }
AXJ_HD bool desc_blank(uint32_t d) { return (d >> 8) & 1u; }
AXJ_HD uint32_t desc_face(uint32_t d) { return d >> 12; }
AXJ_HD uint32_t make_desc(int zr, int rr, bool blank, uint32_t face) {
  return (uint32_t)zr | ((uint32_t)rr << 4) | ((uint32_t)blank << 8) | (face << 12);
}

// Window start offset (relative to the point) of an SBP row of the 6-wide
// derivative operators (ModDeriv.f90:25-46): rows 0-3 start at i_start = i - row,
// rows 5-8 end at i_end = i + (8 - row), row 4 is the centred 5-point stencil.
AXJ_HD int sbp_w0(int row) { return row < 4 ? -row : (row == 4 ? -2 : 3 - row); }
AXJ_HD int sbp_len(int row) { return row == 4 ? 5 : 6; }
// Same for the 11-wide truncated-Gaussian filter (ModTGfilter.f90:19-44).
AXJ_HD int tg_w0(int row) { return row < 4 ? -row : (row == 4 ? -4 : -10 + (8 - row)); }
AXJ_HD int tg_len(int row) { return row == 4 ? 9 : 11; }

constexpr int DT_PHYSICAL = 1;  // axj_dt_mode AXJ_DT_PHYSICAL

// Maximum number of patches and face operations per point.
constexpr int MAX_PATCHES = 64;
constexpr int MAX_FACE_OPS = 8;

// Patch information needed on the device (bc code and direction).
struct PatchDev {
  int bc;
  int dir;
};

// Scalar parameters of one run, passed by value to the kernels.
struct Consts {
  double gam, Re, Pr, CFL;
  double sponge_start_top, sponge_A_top, sponge_end_left, sponge_A_left;
  double C_mu_Re, C_beta_Re, C_kappa_Re_Pr;  // C_mu*Re, C_beta*Re, (C_kappa*Re)*Pr
  double forcing_alpha, forcing_z0, forcing_r0, forcing_lz, forcing_lr;
  double r_top;   // r(i, Nr): sponge normalisation (ModBC.f90:571)
  double harm_amp, harm_omega;  // harmonic forcing (control_forcing == 2): A, 2 pi St U_j
  // per-run factors of the right-hand side, formed once on the host: 1/gam, 1/Re,
  // gam/(Re Pr), gam (gam - 1)/Re
  double inv_gam, inv_Re, gam_RePr, gg1_Re;
  int do_viscous;
  int shock_capturing;
  int control_forcing;  // 0 off, 1 feedback (ControlForcingTerms), 2 harmonic source
  int dt_mode;
  int npatch;
};

}  // namespace axj
