// axj_prep.cuh -- the patch preprocessing of one block (CreateAllPatches,
// ModPatch.f90:214-242; the face lines of the BoundaryConditions loop, ModBC.f90:25-274)
// as per-item functions: one point, one row, one tile. The device path runs them one
// thread per row / per tile (axj_prep.cu); run on the host (axj_prep_maps, algorithm 1),
// the same functions are checked against the host algorithm of axj_create.
#pragma once

#include <cstdint>
#include <vector>

#include "../../include/axj.h"
#include "axj_common.cuh"

namespace axj {

struct PrepArgs {
  const axj_patch* patches;  // PatchCreation output, 1-based inclusive ranges
  int npatch;
  int64_t Nz, Nr, P;         // grid and row pitch of the descriptor planes
  const double* ibval;       // (Nz, Nr), z fastest
};

// The descriptor of point (i, j) (1-based) without its face index, and its face
// operations in patch order (0-based patch indices into ops, at most MAX_FACE_OPS;
// *nops = MAX_FACE_OPS + 1 reports more). The last patch of a direction whose range holds
// the point picks the closure row; a patch acts at the point when the point lies on its
// face line and the bc loop applies an operation there (SAT far field: z faces off the
// axis row; walls: always; NSCBC non-reflecting: off the axis row).
AXJ_HD uint32_t prep_point(const PrepArgs& a, int64_t i, int64_t j, int* nops, int* ops) {
  int wi = -1, wj = -1, n = 0;
  for (int k = 0; k < a.npatch; ++k) {
    const axj_patch& p = a.patches[k];
    const int64_t is = p.i_start < 1 ? 1 : p.i_start, ie = p.i_end > a.Nz ? a.Nz : p.i_end;
    const int64_t js = p.j_start < 1 ? 1 : p.j_start, je = p.j_end > a.Nr ? a.Nr : p.j_end;
    if (i >= is && i <= ie && j >= js && j <= je) {
      if (p.bc_dir == 1 || p.bc_dir == -1) wi = k;
      if (p.bc_dir == 2 || p.bc_dir == -2) wj = k;
    }
    if (p.bc == AXJ_BC_AXIS) continue;
    bool on = false;
    if (p.bc_dir == 1) on = i == p.i_start && j >= p.j_start && j <= p.j_end;
    else if (p.bc_dir == -1) on = i == p.i_end && j >= p.j_start && j <= p.j_end;
    else if (p.bc_dir == 2) on = j == p.j_start && i >= p.i_start && i <= p.i_end;
    else on = j == p.j_end && i >= p.i_start && i <= p.i_end;
    if (!on) continue;
    const bool j1 = (j == 1);
    const int adir = (int)(p.bc_dir < 0 ? -p.bc_dir : p.bc_dir);
    bool active = false;
    if (p.bc == AXJ_BC_SAT_FARFIELD) active = !j1 && adir == 1;
    else if (p.bc == AXJ_BC_SAT_NOSLIP_WALL || p.bc == AXJ_BC_NSCBC_NOSLIP_WALL) active = true;
    else if (p.bc == AXJ_BC_NSCBC_NONREFLECTING) active = !j1;
    if (!active) continue;
    if (n < MAX_FACE_OPS) ops[n] = k;
    ++n;
  }
  *nops = n > MAX_FACE_OPS ? MAX_FACE_OPS + 1 : n;
  int zr = 4, rw = 4;
  if (wi >= 0) {
    const axj_patch& p = a.patches[wi];
    zr = p.bc_dir == 1 ? (int)(i - p.i_start) : (int)(8 + i - p.i_end);
  }
  if (wj >= 0) {
    const axj_patch& p = a.patches[wj];
    rw = p.bc_dir == 2 ? (int)(j - p.j_start) : (int)(8 + j - p.j_end);
  }
  return make_desc(zr, rw, a.ibval[(i - 1) + (j - 1) * a.Nz] == 0.0, 0);
}

// The number of face-list entries of row j (1-based): 1 + count per face point; -1 if a
// point has more than MAX_FACE_OPS operations.
AXJ_HD int64_t prep_row_size(const PrepArgs& a, int64_t j) {
  int ops[MAX_FACE_OPS];
  int64_t s = 0;
  for (int64_t i = 1; i <= a.Nz; ++i) {
    int n = 0;
    prep_point(a, i, j, &n, ops);
    if (n > MAX_FACE_OPS) return -1;
    if (n) s += 1 + n;
  }
  return s;
}

// Row j (1-based): descriptors (with face indices from off on), z / r codes (9 where
// blanked) and face entries (count, then patch indices) of every point, and the
// no-operation descriptor in the pitch padding.
AXJ_HD void prep_row(const PrepArgs& a, int64_t j, int64_t off, uint32_t* desc, unsigned char* zcode,
                     unsigned char* rcode, int* faces) {
  int ops[MAX_FACE_OPS];
  const int64_t base = (j - 1) * a.P;
  for (int64_t i = 1; i <= a.P; ++i) {
    uint32_t d = make_desc(ROW_NONE, ROW_NONE, false, 0);
    if (i <= a.Nz) {
      int n = 0;
      d = prep_point(a, i, j, &n, ops);
      if (n > 0 && n <= MAX_FACE_OPS) {
        d = make_desc(desc_zrow(d), desc_rrow(d), desc_blank(d), (uint32_t)off);
        faces[off] = n;
        for (int k = 0; k < n; ++k) faces[off + 1 + k] = ops[k];
        off += 1 + n;
      }
    }
    desc[base + i - 1] = d;
    zcode[base + i - 1] = (unsigned char)(desc_blank(d) ? ROW_NONE : (uint32_t)desc_zrow(d));
    rcode[base + i - 1] = (unsigned char)(desc_blank(d) ? ROW_NONE : (uint32_t)desc_rrow(d));
  }
}

// Classes of the tile at (i0, j0) with brows rows in its band (0-based): bit 0 = interior
// stage tile (centred rows, no blanked or face point on the tile; centred rows and no
// blanking on its r halo columns and, for the r rows, on its z halo), bit 1 = interior
// sensor tile (centred rows and no blanking within SENS_HS_INT of the tile, the V region
// of reach SENS_HS_INT + H_INT inside the grid).
AXJ_HD int prep_tile_flags(const uint32_t* desc, int64_t P, int64_t Nz, int64_t Nr, int64_t i0, int64_t j0,
                           int64_t brows) {
  auto dsc = [&](int64_t i, int64_t j) { return desc[j * P + i]; };
  bool interior = brows == TR && i0 - H_INT >= 0 && i0 + TZ + H_INT <= Nz && j0 - H_INT >= 0 && j0 + TR + H_INT <= Nr;
  // the tile's own points, its r halo on the tile columns, its z halo on the tile rows
  for (int64_t j = j0 - H_INT; interior && j < j0 + TR + H_INT; ++j) {
    const bool own = j >= j0 && j < j0 + TR;
    for (int64_t i = i0 - (own ? H_INT : 0); interior && i < i0 + TZ + (own ? H_INT : 0); ++i) {
      const uint32_t d = dsc(i, j);
      const bool col = i >= i0 && i < i0 + TZ;
      if (own && col) {
        if (desc_zrow(d) != 4 || desc_rrow(d) != 4 || desc_blank(d) || desc_face(d) != 0) interior = false;
      } else if (col) {
        if (desc_zrow(d) != 4 || desc_rrow(d) != 4 || desc_blank(d)) interior = false;
      } else {
        if (desc_rrow(d) != 4 || desc_blank(d)) interior = false;
      }
    }
  }
  const int64_t hv = SENS_HS_INT + H_INT, hs = SENS_HS_INT, hzv = (hv + 1) & ~(int64_t)1;
  bool sint = brows == TR && i0 - hzv >= 0 && i0 + TZ + hzv <= Nz && j0 - hv >= 0 && j0 + TR + hv <= Nr;
  for (int64_t j = j0 - hs; sint && j < j0 + TR + hs; ++j)
    for (int64_t i = i0 - hs; sint && i < i0 + TZ + hs; ++i) {
      const uint32_t d = dsc(i, j);
      if (desc_zrow(d) != 4 || desc_rrow(d) != 4 || desc_blank(d)) sint = false;
    }
  return (interior ? 1 : 0) | (sint ? 2 : 0);
}

// The device path: rows and tiles one thread each. cands holds (i0, j0, brows) of every
// tile in the host's order; flags gets prep_tile_flags of each. Outputs are host vectors
// (desc, zcode, rcode with pitch P; faces with the leading 0 entry).
int prep_on_device(const PrepArgs& host_args, const int64_t* cands, int64_t ncand, uint32_t* desc,
                   unsigned char* zcode, unsigned char* rcode, std::vector<int>& faces, unsigned char* flags,
                   char* msg, int msglen);

}  // namespace axj
