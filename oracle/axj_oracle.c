/*
 * axj_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY) for the per-step hot path of
 * nataraj2/AxisymmetricJet.
 *
 * This is a line-faithful C restatement of the reference Fortran for one block that
 * holds the whole grid (all MPI neighbours are MPI_PROC_NULL, so nbrs(:) < 0 and
 * ProcessorCommunication is a no-op). It is used only by tests/, by the smoke check and
 * by bench.py's CPU baseline, as the checker. The product (libaxj.so) never calls it.
 *
 * Decomposition replica (axo_set_decomposition): the numerics of the reference run on a
 * dims_z x dims_r process grid (ModDecomp.f90:5-105), on the same global arrays. Every
 * operator reads halo cells that ProcessorCommunication refreshed just before it
 * (ModRHS.f90:20-51, ModShockCapturing.f90:23-76, ModSolver.f90:56-73), so a
 * decomposed run equals the single block except where a rank's own loops use its local
 * extent or its own module state:
 *  - the in-place z filter restarts at every block start from the neighbour's
 *    unfiltered values (exchanged at ModShockCapturing.f90:58-60, filtered at :63);
 *  - the stale scalar T is per rank (ModRHS.f90:76,145 set it at the block's last
 *    point, the rank's face loops override it) and dt is the MIN over ranks
 *    (ModInputOutput.f90:405-422);
 *  - the top sponge divides by r at the block's last row (ModBC.f90:571);
 *  - deltaz / deltar are one-sided at the block's edges (ModShockCapturing.f90:169-186);
 *  - the block's first row takes the axis form of the dilatation and of S22
 *    (ModShockCapturing.f90:114-118, :146-150, :188-192).
 *
 * PARITY STATUS: unpinned against reference outputs. The reference ships no tests or
 * golden vectors and its Fortran cannot be compiled in this image (no gfortran/flang).
 * The restatement is pinned instead by operator known-answer tests (polynomial
 * exactness of SBP1/SBP2, TG row sums), the operator tables and default constants as the
 * reference's source text states them (tests/golden/reference_constants.json, equal bit
 * for bit), the shipped bc fixture (bc_4400x640_nozzle.dat), free-stream
 * preservation, and a second restatement in plain Python (tests/restatement.py: the
 * operators, the sensor, the right-hand side with the bc loop and sponges, RK4), equal
 * to this one bit for bit, all in tests/.
 *
 * Restatement rules:
 *  - Same arithmetic and evaluation order as the Fortran source (left-to-right,
 *    DOT_PRODUCT and MATMUL as sequential sums starting from 0); build with
 *    -ffp-contract=off and no fast-math. libm pow/tanh/exp/sqrt as gfortran calls them.
 *  - Single-precision literals of the reference stay single precision
 *    (TGfilt boundary rows, ModOperator.f90:94-97; the 1e-15 of ModShockCapturing.f90:202).
 *  - Loops that carry no cross-point dependence may run in any order (OpenMP over
 *    columns); the in-place z filter (a recurrence along i) and the stale module scalar T
 *    are evaluated in the reference's order.
 *  - Halo cells of the (-3:Nz+4,-3:Nr+4) arrays that the reference never writes are 0.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/axj.h"

typedef int64_t I8;

typedef struct axo {
  I8 Nz, Nr, LZ, LR;
  axj_params p;
  double SBP1[9][6], SBP2[9][6], TG[9][11];
  /* halo-padded fields (-3:Nz+4, -3:Nr+4) */
  double *zvec, *rvec, *dxidz, *detadr, *dzdxi, *drdeta, *ddxidxidz, *ddetadetadr;
  double *rhovec, *Vrvec, *Vtvec, *Vzvec, *Tvec, *pvec, *muvec, *kappavec, *lambdavec, *betavec;
  double *drhodz, *dVrdz, *dVtdz, *dVzdz, *dTdz, *dpdz, *dmudz, *dkappadz;
  double *drhodr, *dVrdr, *dVtdr, *dVzdr, *dTdr, *dpdr, *dmudr, *dkappadr;
  double *d2Vrdz2, *d2Vtdz2, *d2Vzdz2, *d2Tdz2, *d2Vrdr2, *d2Vtdr2, *d2Vzdr2, *d2Tdr2;
  double *d2Vrdzdr, *d2Vzdzdr;
  /* shock capturing */
  double *MgnStrRate, *d2Sdxi2, *d2Sdeta2, *d4Sdxi4, *d4Sdeta4;
  double *d2Tdxi2, *d2Tdeta2, *d4Tdxi4, *d4Tdeta4;
  double *dilvec, *d2dildxi2, *d2dildeta2, *d4dildxi4, *d4dildeta4;
  double *mustarQ, *mustar, *betastarQ, *betastar, *kappastarQ, *kappastar;
  /* interior fields (Nz, Nr) and solutions (Nz, Nr, 5) */
  double *ibval, *deltvec;
  double *pv, *pv_old, *pv_target, *pv_targetI, *pv_targetV, *k1, *k2, *k3, *k4, *rhs;
  I8 *is_it_i_patch, *which_i_patch, *is_it_j_patch, *which_j_patch;
  axj_patch* patch;
  I8 no_bcs;
  /* decomposition replica: blocks along z and r, block of each i and j, block ranges
     (1-based, inclusive), and each block's module scalar T (ModuleVariables.f90:53) */
  I8 nbz, nbr;
  I8 *bz, *br, *zlo, *zhi, *rlo, *rhi;
  double* Tb;
  /* when set: every face operation the bc loop applies is recorded per point (count and
     1-based patch numbers, one per byte) */
  uint8_t* rec_n;
  uint64_t* rec_ids;
  double delt, time;
  double t_stage;  /* time of the current RHS evaluation (harmonic forcing) */
  I8 iteration;
} axo;

#define HIX(o, i, j) ((size_t)((i) + 3) + (size_t)((j) + 3) * (size_t)(o)->LZ)
#define BLK(o, i, j) ((o)->bz[i] + (o)->nbz * (o)->br[j])
#define H(o, a, i, j) ((o)->a[HIX(o, i, j)])
#define IIX(o, i, j) ((size_t)((i)-1) + (size_t)((j)-1) * (size_t)(o)->Nz)
#define S5(o, a, i, j, e) ((o)->a[IIX(o, i, j) + (size_t)((e)-1) * (size_t)(o)->Nz * (size_t)(o)->Nr])

static double* halloc(axo* o) { return (double*)calloc((size_t)o->LZ * (size_t)o->LR, sizeof(double)); }
static double* ialloc(axo* o, int n) { return (double*)calloc((size_t)o->Nz * (size_t)o->Nr * (size_t)n, sizeof(double)); }

/* ---------------- SBP_operator (ModOperator.f90:5-121) ---------------- */
static void sbp_operator(axo* o) {
  memset(o->SBP1, 0, sizeof(o->SBP1));
  memset(o->SBP2, 0, sizeof(o->SBP2));
  memset(o->TG, 0, sizeof(o->TG));
  double (*S1)[6] = o->SBP1, (*S2)[6] = o->SBP2, (*G)[11] = o->TG;
  /* :25-28 */
  S1[0][0] = -24.0 / 17.0; S1[0][1] = 59.0 / 34.0; S1[0][2] = -4.0 / 17.0; S1[0][3] = -3.0 / 34.0;
  S1[1][0] = -1.0 / 2.0; S1[1][1] = 0.0; S1[1][2] = 1.0 / 2.0;
  S1[2][0] = 4.0 / 43.0; S1[2][1] = -59.0 / 86.0; S1[2][2] = 0.0; S1[2][3] = 59.0 / 86.0; S1[2][4] = -4.0 / 43.0;
  S1[3][0] = 3.0 / 98.0; S1[3][1] = 0.0; S1[3][2] = -59.0 / 98.0; S1[3][3] = 0.0; S1[3][4] = 32.0 / 49.0;
  S1[3][5] = -4.0 / 49.0;
  /* :32-38 bottom = -mirror */
  for (int i = 9; i >= 6; --i)
    for (int j = 6; j >= 1; --j) S1[i - 1][j - 1] = -1.0 * S1[10 - i - 1][7 - j - 1];
  /* :42 */
  S1[4][0] = 1.0 / 12.0; S1[4][1] = -2.0 / 3.0; S1[4][2] = 0.0; S1[4][3] = 2.0 / 3.0; S1[4][4] = -1.0 / 12.0;
  /* :61-64 */
  S2[0][0] = 2.0; S2[0][1] = -5.0; S2[0][2] = 4.0; S2[0][3] = -1.0;
  S2[1][0] = 1.0; S2[1][1] = -2.0; S2[1][2] = 1.0;
  S2[2][0] = -4.0 / 43.0; S2[2][1] = 59.0 / 43.0; S2[2][2] = -110.0 / 43.0; S2[2][3] = 59.0 / 43.0;
  S2[2][4] = -4.0 / 43.0;
  S2[3][0] = -1.0 / 49.0; S2[3][1] = 0.0; S2[3][2] = 59.0 / 49.0; S2[3][3] = -118.0 / 49.0;
  S2[3][4] = 64.0 / 49.0; S2[3][5] = -4.0 / 49.0;
  /* :68-74 bottom = +mirror */
  for (int i = 9; i >= 6; --i)
    for (int j = 6; j >= 1; --j) S2[i - 1][j - 1] = 1.0 * S2[10 - i - 1][7 - j - 1];
  /* :78 */
  S2[4][0] = -1.0 / 12.0; S2[4][1] = 4.0 / 3.0; S2[4][2] = -5.0 / 2.0; S2[4][3] = 4.0 / 3.0; S2[4][4] = -1.0 / 12.0;
  /* TG filter :93-97; the boundary-row literals are default (single-precision) reals */
  G[0][0] = 1.0;
  const float r1[7] = {0.085777408970000f, 0.722371828476000f, 0.356848072173000f, -0.223119093072000f,
                       0.057347064865000f, 0.000747264596000f, 0.000027453993000f};
  const float r2[7] = {-0.032649010764000f, 0.143339502575000f, 0.726678822020000f, 0.294622121167000f,
                       -0.186711738069000f, 0.062038376258000f, -0.007318073189000f};
  const float r3[11] = {0.000054596010000f, -0.042124772446000f, 0.173103107841000f, 0.700384128648000f,
                        0.276543612935000f, -0.131223506571000f, 0.023424966418000f, -0.013937561779000f,
                        0.024565095706000f, -0.013098287852000f, 0.002308621090000f};
  for (int m = 0; m < 7; ++m) { G[1][m] = (double)r1[m]; G[2][m] = (double)r2[m]; }
  for (int m = 0; m < 11; ++m) G[3][m] = (double)r3[m];
  /* :101-107 */
  for (int i = 9; i >= 6; --i)
    for (int j = 11; j >= 1; --j) G[i - 1][j - 1] = 1.0 * G[10 - i - 1][12 - j - 1];
  /* :111-112 */
  G[4][0] = 107.0 / 103680.0; G[4][1] = 149.0 / 12960.0; G[4][2] = 1997.0 / 25920.0;
  G[4][3] = 3091.0 / 12960.0; G[4][4] = 3565.0 / 10368.0; G[4][5] = 3091.0 / 12960.0;
  G[4][6] = 1997.0 / 25920.0; G[4][7] = 149.0 / 12960.0; G[4][8] = 107.0 / 103680.0;
}

/* DOT_PRODUCT(row(0:n-1), var(start:start+n-1)) along z (stride 1) or r (stride LZ). */
static inline double dotz(const double* row, int n, const axo* o, const double* var, I8 i0, I8 j) {
  double s = 0.0;
  for (int m = 0; m < n; ++m) s = s + row[m] * var[HIX(o, i0 + m, j)];
  return s;
}
static inline double dotr(const double* row, int n, const axo* o, const double* var, I8 i, I8 j0) {
  double s = 0.0;
  for (int m = 0; m < n; ++m) s = s + row[m] * var[HIX(o, i, j0 + m)];
  return s;
}

/* Patch-driven stencil row selection shared by ModDeriv and ModTGfilter.
 * Returns 1 and sets (row, window start) if a closure row applies, 0 for interior. */
static inline int zrow(const axo* o, I8 i, I8 j, int* row, I8* w0, int halfwide) {
  if (o->is_it_i_patch[IIX(o, i, j)] == 1) {
    const axj_patch* pt = &o->patch[o->which_i_patch[IIX(o, i, j)] - 1];
    if (pt->bc_dir == 1) { *row = (int)(i - pt->i_start); *w0 = pt->i_start; return 1; }
    if (pt->bc_dir == -1) { *row = (int)(8 + i - pt->i_end); *w0 = pt->i_end - halfwide; return 1; }
    return 2; /* unreachable for consistent maps: no assignment */
  }
  return 0;
}
static inline int rrow(const axo* o, I8 i, I8 j, int* row, I8* w0, int halfwide) {
  if (o->is_it_j_patch[IIX(o, i, j)] == 1) {
    const axj_patch* pt = &o->patch[o->which_j_patch[IIX(o, i, j)] - 1];
    if (pt->bc_dir == 2) { *row = (int)(j - pt->j_start); *w0 = pt->j_start; return 1; }
    if (pt->bc_dir == -2) { *row = (int)(8 + j - pt->j_end); *w0 = pt->j_end - halfwide; return 1; }
    return 2;
  }
  return 0;
}

/* Stencil core of Compute1stDerivative / Compute2ndDerivative /
 * Compute2ndDerivativeComputational (ModDeriv.f90:5-120, :123-238, :387-481). */
static void stencil_pass(const axo* o, double (*OP)[6], const double* var, int dirn, double* out) {
  memset(out, 0, sizeof(double) * (size_t)o->LZ * (size_t)o->LR); /* out = 0.0D0 */
  if (dirn == 1) {
#pragma omp parallel for schedule(static)
    for (I8 j = 1; j <= o->Nr; ++j)
      for (I8 i = 1; i <= o->Nz; ++i) {
        if (o->ibval[IIX(o, i, j)] == 0.0) continue;
        int row; I8 w0;
        int c = zrow(o, i, j, &row, &w0, 5);
        if (c == 1) out[HIX(o, i, j)] = dotz(OP[row], 6, o, var, w0, j);
        else if (c == 0) out[HIX(o, i, j)] = dotz(OP[4], 5, o, var, i - 2, j);
      }
  } else {
#pragma omp parallel for schedule(static)
    for (I8 j = 1; j <= o->Nr; ++j)
      for (I8 i = 1; i <= o->Nz; ++i) {
        if (o->ibval[IIX(o, i, j)] == 0.0) continue;
        int row; I8 w0;
        int c = rrow(o, i, j, &row, &w0, 5);
        if (c == 1) out[HIX(o, i, j)] = dotr(OP[row], 6, o, var, i, w0);
        else if (c == 0) out[HIX(o, i, j)] = dotr(OP[4], 5, o, var, i, j - 2);
      }
  }
}

/* Compute1stDerivative (ModDeriv.f90:5-120) */
static void deriv1(axo* o, const double* var, int dirn, double* out) {
  stencil_pass(o, o->SBP1, var, dirn, out);
  const double* met = dirn == 1 ? o->dxidz : o->detadr;
#pragma omp parallel for schedule(static)
  for (I8 j = 1; j <= o->Nr; ++j)
    for (I8 i = 1; i <= o->Nz; ++i) out[HIX(o, i, j)] = out[HIX(o, i, j)] * met[HIX(o, i, j)];
}

/* Compute2ndDerivative (ModDeriv.f90:123-238) */
static void deriv2(axo* o, const double* var, int dirn, const double* first, double* out) {
  stencil_pass(o, o->SBP2, var, dirn, out);
  const double* met = dirn == 1 ? o->dxidz : o->detadr;
  const double* met2 = dirn == 1 ? o->ddxidxidz : o->ddetadetadr;
#pragma omp parallel for schedule(static)
  for (I8 j = 1; j <= o->Nr; ++j)
    for (I8 i = 1; i <= o->Nz; ++i) {
      size_t x = HIX(o, i, j);
      double m = met[x];
      out[x] = out[x] * (m * m) + first[x] * met2[x];
    }
}

/* Compute2ndDerivativeComputational (ModDeriv.f90:387-481) */
static void deriv2comp(axo* o, const double* var, int dirn, double* out) {
  stencil_pass(o, o->SBP2, var, dirn, out);
}

/* ComputeMetric (ModDeriv.f90:241-382) with nbrs(:) < 0 (domain-edge closures). */
static void compute_metric(axo* o, const double* var, int dirn, double* out) {
  memset(out, 0, sizeof(double) * (size_t)o->LZ * (size_t)o->LR);
  I8 Nz = o->Nz, Nr = o->Nr;
  if (dirn == 1) {
    for (I8 i = 5; i <= Nz - 4; ++i)
      for (I8 j = 1; j <= Nr; ++j) out[HIX(o, i, j)] = dotz(o->SBP1[4], 5, o, var, i - 2, j);
    for (I8 i = 1; i <= 4; ++i)
      for (I8 j = 1; j <= Nr; ++j) out[HIX(o, i, j)] = dotz(o->SBP1[i - 1], 6, o, var, 1, j);
    for (I8 i = Nz - 3; i <= Nz; ++i)
      for (I8 j = 1; j <= Nr; ++j) out[HIX(o, i, j)] = dotz(o->SBP1[8 - Nz + i], 6, o, var, Nz - 5, j);
  } else {
    for (I8 i = 1; i <= Nz; ++i)
      for (I8 j = 5; j <= Nr - 4; ++j) out[HIX(o, i, j)] = dotr(o->SBP1[4], 5, o, var, i, j - 2);
    for (I8 i = 1; i <= Nz; ++i)
      for (I8 j = 1; j <= 4; ++j) out[HIX(o, i, j)] = dotr(o->SBP1[j - 1], 6, o, var, i, 1);
    for (I8 i = 1; i <= Nz; ++i)
      for (I8 j = Nr - 3; j <= Nr; ++j) out[HIX(o, i, j)] = dotr(o->SBP1[8 - Nr + j], 6, o, var, i, Nr - 5);
  }
}

/* PerformTGfilter (ModTGfilter.f90:5-95). out is not zeroed. When var == out the
 * z pass is the in-place recurrence of ModShockCapturing.f90:63 and runs in the
 * reference's loop order (i outer, j inner); rows j are independent of each other. */
static void tgfilter(axo* o, const double* var, int dirn, double* out) {
  if (dirn == 1 && var == out && o->nbz > 1) {
    /* decomposed in-place z filter: a block reads its left neighbour's unfiltered values */
    const size_t nh = (size_t)o->LZ * (size_t)o->LR;
    double* pre = (double*)malloc(nh * sizeof(double));
    memcpy(pre, var, nh * sizeof(double));
#pragma omp parallel for schedule(static)
    for (I8 j = 1; j <= o->Nr; ++j)
      for (I8 i = 1; i <= o->Nz; ++i) {
        if (o->ibval[IIX(o, i, j)] == 0.0) continue;
        int row; I8 w0;
        int c = zrow(o, i, j, &row, &w0, 10);
        const double* tr;
        int n;
        if (c == 1) { tr = o->TG[row]; n = 11; }
        else if (c == 0) { tr = o->TG[4]; n = 9; w0 = i - 4; }
        else continue;
        const I8 lo = o->zlo[o->bz[i]];
        double sum = 0.0;
        for (int m = 0; m < n; ++m) {
          const I8 q = w0 + m;
          sum = sum + tr[m] * (q < lo ? pre : out)[HIX(o, q, j)];
        }
        out[HIX(o, i, j)] = sum;
      }
    free(pre);
    return;
  }
  if (dirn == 1) {
#pragma omp parallel for schedule(static)
    for (I8 j = 1; j <= o->Nr; ++j)
      for (I8 i = 1; i <= o->Nz; ++i) {
        if (o->ibval[IIX(o, i, j)] == 0.0) continue;
        int row; I8 w0;
        int c = zrow(o, i, j, &row, &w0, 10);
        double v;
        if (c == 1) v = dotz(o->TG[row], 11, o, var, w0, j);
        else if (c == 0) v = dotz(o->TG[4], 9, o, var, i - 4, j);
        else continue;
        out[HIX(o, i, j)] = v;
      }
  } else {
    if (var == out) {
      /* never used by the reference; keep the sequential order */
      for (I8 i = 1; i <= o->Nz; ++i)
        for (I8 j = 1; j <= o->Nr; ++j) {
          if (o->ibval[IIX(o, i, j)] == 0.0) continue;
          int row; I8 w0;
          int c = rrow(o, i, j, &row, &w0, 10);
          if (c == 1) out[HIX(o, i, j)] = dotr(o->TG[row], 11, o, var, i, w0);
          else if (c == 0) out[HIX(o, i, j)] = dotr(o->TG[4], 9, o, var, i, j - 4);
        }
      return;
    }
#pragma omp parallel for schedule(static)
    for (I8 j = 1; j <= o->Nr; ++j)
      for (I8 i = 1; i <= o->Nz; ++i) {
        if (o->ibval[IIX(o, i, j)] == 0.0) continue;
        int row; I8 w0;
        int c = rrow(o, i, j, &row, &w0, 10);
        if (c == 1) out[HIX(o, i, j)] = dotr(o->TG[row], 11, o, var, i, w0);
        else if (c == 0) out[HIX(o, i, j)] = dotr(o->TG[4], 9, o, var, i, j - 4);
      }
  }
}

/* AssignValues (ModAssign.f90:5-29) */
static void assign_values(axo* o) {
#pragma omp parallel for schedule(static)
  for (I8 j = 1; j <= o->Nr; ++j)
    for (I8 i = 1; i <= o->Nz; ++i) {
      size_t x = HIX(o, i, j);
      o->rhovec[x] = S5(o, pv, i, j, 1);
      o->Vrvec[x] = S5(o, pv, i, j, 2);
      o->Vtvec[x] = S5(o, pv, i, j, 3);
      o->Vzvec[x] = S5(o, pv, i, j, 4);
      o->Tvec[x] = S5(o, pv, i, j, 5);
      o->pvec[x] = o->rhovec[x] * o->Tvec[x];
      o->muvec[x] = pow(o->Tvec[x], 0.666);
      o->kappavec[x] = o->muvec[x];
      o->betavec[x] = (3.0 / 5.0) * o->muvec[x];
      o->lambdavec[x] = o->betavec[x] - (2.0 / 3.0) * o->muvec[x];
    }
}

/* ---------------- ModShockCapturing (ModShockCapturing.f90:5-258) ---------------- */
static void shock_capturing(axo* o) {
  I8 Nz = o->Nz, Nr = o->Nr;
  /* ComputeDilatation :108-126, ComputeMgnStrRate :129-159 */
#pragma omp parallel for schedule(static)
  for (I8 j = 1; j <= Nr; ++j)
    for (I8 i = 1; i <= Nz; ++i) {
      size_t x = HIX(o, i, j);
      if (j == o->rlo[o->br[j]]) o->dilvec[x] = 2.0 * o->dVrdr[x] + o->dVzdz[x];
      else o->dilvec[x] = o->dVrdr[x] + o->Vrvec[x] / o->rvec[x] + o->dVzdz[x];
    }
#pragma omp parallel for schedule(static)
  for (I8 j = 1; j <= Nr; ++j)
    for (I8 i = 1; i <= Nz; ++i) {
      size_t x = HIX(o, i, j);
      double S11 = o->dVrdr[x] - (1.0 / 3.0) * o->dilvec[x];
      double S12 = 0.0;
      double S13 = 0.5 * (o->dVrdz[x] + o->dVzdr[x]);
      double S21 = 0.0, S23 = 0.0;
      double S31 = S13, S32 = 0.0;
      double S33 = o->dVzdz[x] - (1.0 / 3.0) * o->dilvec[x];
      double S22;
      if (j == o->rlo[o->br[j]]) S22 = o->dVrdr[x] - (1.0 / 3.0) * o->dilvec[x];
      else S22 = o->Vrvec[x] / o->rvec[x] - (1.0 / 3.0) * o->dilvec[x];
      o->MgnStrRate[x] = sqrt(S11 * S11 + S12 * S12 + S13 * S13 + S21 * S21 + S22 * S22 + S23 * S23 +
                              S31 * S31 + S32 * S32 + S33 * S33);
    }
  /* :27-51 */
  deriv2comp(o, o->MgnStrRate, 1, o->d2Sdxi2);
  deriv2comp(o, o->Tvec, 1, o->d2Tdxi2);
  deriv2comp(o, o->dilvec, 1, o->d2dildxi2);
  deriv2comp(o, o->MgnStrRate, 2, o->d2Sdeta2);
  deriv2comp(o, o->Tvec, 2, o->d2Tdeta2);
  deriv2comp(o, o->dilvec, 2, o->d2dildeta2);
  deriv2comp(o, o->d2Sdxi2, 1, o->d4Sdxi4);
  deriv2comp(o, o->d2Tdxi2, 1, o->d4Tdxi4);
  deriv2comp(o, o->d2dildxi2, 1, o->d4dildxi4);
  deriv2comp(o, o->d2Sdeta2, 2, o->d4Sdeta4);
  deriv2comp(o, o->d2Tdeta2, 2, o->d4Tdeta4);
  deriv2comp(o, o->d2dildeta2, 2, o->d4dildeta4);
  /* ComputeTobeFilteredQuantities :162-222 */
  const double eps = (double)1e-15f; /* single-precision literal 1e-15 (:202) */
  const double gam = o->p.gam;
#pragma omp parallel for schedule(static)
  for (I8 j = 1; j <= Nr; ++j)
    for (I8 i = 1; i <= Nz; ++i) {
      size_t x = HIX(o, i, j);
      /* the rank's own extent: i1..i2, j1..j2 (1..Nz, 1..Nr for one block) */
      const I8 i1 = o->zlo[o->bz[i]], i2 = o->zhi[o->bz[i]], j1 = o->rlo[o->br[j]], j2 = o->rhi[o->br[j]];
      double deltaz = 0.0, deltar = 0.0;
      if (i >= i1 + 1 && i <= i2 - 1) deltaz = (H(o, zvec, i + 1, j) - H(o, zvec, i - 1, j)) / 2.0;
      if (i == i1) deltaz = H(o, zvec, i1 + 1, j) - H(o, zvec, i1, j);
      if (i == i2) deltaz = H(o, zvec, i2, j) - H(o, zvec, i2 - 1, j);
      if (j >= j1 + 1 && j <= j2 - 1) deltar = (H(o, rvec, i, j + 1) - H(o, rvec, i, j - 1)) / 2.0;
      if (j == j1) deltar = H(o, rvec, i, j1 + 1) - H(o, rvec, i, j1);
      if (j == j2) deltar = H(o, rvec, i, j2) - H(o, rvec, i, j2 - 1);
      double dil;
      if (j == j1) dil = 2.0 * o->dVrdr[x] + o->dVzdz[x];
      else dil = o->dVrdr[x] + o->Vrvec[x] / o->rvec[x] + o->dVzdz[x];
      double vort = fabs(o->dVrdz[x] - o->dVzdr[x]);
      double mdil = -1.0 * dil;
      double Hm = (mdil < 0.0) ? 0.0 : 1.0; /* Heaviside :224-236 */
      double fsw = Hm * (dil * dil) / (dil * dil + vort * vort + eps);
      o->mustarQ[x] = o->rhovec[x] * fabs((o->d4Sdxi4[x] * (deltaz * deltaz) + o->d4Sdeta4[x] * (deltar * deltar)));
      o->betastarQ[x] =
          o->rhovec[x] * fsw * fabs((o->d4dildxi4[x] * (deltaz * deltaz) + o->d4dildeta4[x] * (deltar * deltar)));
      o->kappastarQ[x] = o->rhovec[x] / (gam * sqrt(o->Tvec[x])) *
                         fabs((o->d4Tdxi4[x] * deltaz + o->d4Tdeta4[x] * deltar));
    }
  /* :63-79 */
  const double Re = o->p.Re, Pr = o->p.Pr;
  tgfilter(o, o->mustarQ, 1, o->mustarQ);
  tgfilter(o, o->mustarQ, 2, o->mustar);
  tgfilter(o, o->betastarQ, 1, o->betastarQ);
  tgfilter(o, o->betastarQ, 2, o->betastar);
  tgfilter(o, o->kappastarQ, 1, o->kappastarQ);
  tgfilter(o, o->kappastarQ, 2, o->kappastar);
  const size_t nh = (size_t)o->LZ * (size_t)o->LR;
  for (size_t x = 0; x < nh; ++x) {
    o->mustar[x] = o->p.C_mu * Re * o->mustar[x];
    o->betastar[x] = o->p.C_beta * Re * o->betastar[x];
    o->kappastar[x] = o->p.C_kappa * Re * Pr * o->kappastar[x];
  }
  /* :81-92 */
#pragma omp parallel for schedule(static)
  for (I8 j = 1; j <= Nr; ++j)
    for (I8 i = 1; i <= Nz; ++i) {
      size_t x = HIX(o, i, j);
      double tmp = (1.0 + tanh(5.0 * (o->zvec[x] - 10.0))) / 2.0;
      o->mustar[x] = o->mustar[x] * tmp;
      o->betastar[x] = o->betastar[x] * tmp;
      o->kappastar[x] = o->kappastar[x] * tmp;
    }
  /* UpdateTransportCoeffs :238-258 */
#pragma omp parallel for schedule(static)
  for (I8 j = 1; j <= Nr; ++j)
    for (I8 i = 1; i <= Nz; ++i) {
      size_t x = HIX(o, i, j);
      o->muvec[x] = o->muvec[x] + o->mustar[x];
      o->betavec[x] = o->betavec[x] + o->betastar[x];
      o->lambdavec[x] = o->betavec[x] - (2.0 / 3.0) * o->muvec[x];
      o->kappavec[x] = o->kappavec[x] + o->kappastar[x];
    }
}

/* ---------------- ModBC (ModBC.f90) ---------------- */
typedef struct {
  double lam[5][5], Tm[5][5], Ti[5][5];
} eig_t;

/* eigen_matrices_in_z_direction (:280-358) / _r_direction (:360-437); lam is a
 * module array that BoundaryConditions zeroes once (:23); only its diagonal is set. */
static void eigen_matrices(int rdir, double rho, double U, double T, double gam, eig_t* e) {
  memset(e->Tm, 0, sizeof(e->Tm));
  memset(e->Ti, 0, sizeof(e->Ti));
  e->lam[0][0] = U;
  e->lam[1][1] = U;
  e->lam[2][2] = U;
  e->lam[3][3] = (U - sqrt(T));
  e->lam[4][4] = (U + sqrt(T));
  e->Tm[0][0] = -1.0 * rho / T;
  e->Tm[0][3] = rho / ((gam - 1.0) * T);
  e->Tm[0][4] = rho / ((gam - 1.0) * T);
  if (!rdir) {
    e->Tm[1][2] = 1.0;
    e->Tm[2][1] = 1.0;
    e->Tm[3][3] = -1.0 / ((gam - 1.0) * sqrt(T));
    e->Tm[3][4] = 1.0 / ((gam - 1.0) * sqrt(T));
  } else {
    e->Tm[1][3] = -1.0 / ((gam - 1.0) * sqrt(T));
    e->Tm[1][4] = 1.0 / ((gam - 1.0) * sqrt(T));
    e->Tm[2][2] = 1.0;
    e->Tm[3][1] = 1.0;
  }
  e->Tm[4][0] = 1.0;
  e->Tm[4][3] = 1.0;
  e->Tm[4][4] = 1.0;
  e->Ti[0][0] = -1.0 * (gam - 1.0) * T / (gam * rho);
  e->Ti[0][4] = 1.0 / gam;
  if (!rdir) {
    e->Ti[1][2] = 1.0;
    e->Ti[2][1] = 1.0;
    e->Ti[3][0] = (gam - 1.0) * T / (2.0 * gam * rho);
    e->Ti[3][3] = -1.0 * (gam - 1.0) * sqrt(T) / 2.0;
    e->Ti[3][4] = (gam - 1.0) / (2.0 * gam);
    e->Ti[4][0] = (gam - 1.0) * T / (2.0 * gam * rho);
    e->Ti[4][3] = (gam - 1.0) * sqrt(T) / 2.0;
    e->Ti[4][4] = (gam - 1.0) / (2.0 * gam);
  } else {
    e->Ti[1][3] = 1.0;
    e->Ti[2][2] = 1.0;
    e->Ti[3][0] = (gam - 1.0) * T / (2.0 * gam * rho);
    e->Ti[3][1] = -1.0 * (gam - 1.0) * sqrt(T) / 2.0;
    e->Ti[3][4] = (gam - 1.0) / (2.0 * gam);
    e->Ti[4][0] = (gam - 1.0) * T / (2.0 * gam * rho);
    e->Ti[4][1] = (gam - 1.0) * sqrt(T) / 2.0;
    e->Ti[4][4] = (gam - 1.0) / (2.0 * gam);
  }
}

/* MATMUL(A(5,5), v(5)) as a sequential sum over k. */
static void matvec(double A[5][5], const double* v, double* out) {
  double t[5];
  for (int r = 0; r < 5; ++r) {
    double s = 0.0;
    for (int k = 0; k < 5; ++k) s = s + A[r][k] * v[k];
    t[r] = s;
  }
  memcpy(out, t, sizeof(t));
}
/* MATMUL(MATMUL(Tm, lam), w) */
static void tlam_w(double Tm[5][5], double lam[5][5], const double* w, double* out) {
  double M[5][5];
  for (int r = 0; r < 5; ++r)
    for (int c = 0; c < 5; ++c) {
      double s = 0.0;
      for (int k = 0; k < 5; ++k) s = s + Tm[r][k] * lam[k][c];
      M[r][c] = s;
    }
  matvec(M, w, out);
}

/* BoundaryConditions (:16-277) + sponge_bcs (:548-617). Sequential: sets the module
   scalar T of the block of every face point it visits. */
static inline void rec_op(axo* o, I8 pn, I8 i, I8 j) {
  if (!o->rec_n) return;
  const size_t x = IIX(o, i, j);
  const uint8_t n = o->rec_n[x];
  if (n < 8) o->rec_ids[x] |= (uint64_t)pn << (8 * n);
  o->rec_n[x] = (uint8_t)(n + 1);
}

static void boundary_conditions(axo* o) {
  const double gam = o->p.gam;
  const double sigma_1 = -2.0, sigma_2 = -2.0, one_by_h_44 = 48.0 / 49.0;
  eig_t e;
  memset(&e, 0, sizeof(e)); /* lam = 0.0D0 (:23) */
  for (I8 pn = 1; pn <= o->no_bcs; ++pn) {
    const axj_patch* pt = &o->patch[pn - 1];
    if (pt->bc == AXJ_BC_AXIS) continue;
    I8 is = 0, ie = -1, js = 0, je = -1;
    if (pt->bc_dir == 1) { is = pt->i_start; ie = pt->i_start; js = pt->j_start; je = pt->j_end; }
    else if (pt->bc_dir == -1) { is = pt->i_end; ie = pt->i_end; js = pt->j_start; je = pt->j_end; }
    else if (pt->bc_dir == 2) { is = pt->i_start; ie = pt->i_end; js = pt->j_start; je = pt->j_start; }
    else if (pt->bc_dir == -2) { is = pt->i_start; ie = pt->i_end; js = pt->j_end; je = pt->j_end; }
    const int adir = (int)(pt->bc_dir < 0 ? -pt->bc_dir : pt->bc_dir);
    for (I8 i = is; i <= ie; ++i)
      for (I8 j = js; j <= je; ++j) {
        size_t x = HIX(o, i, j);
        double pvl[5], tgt[5], w[5], out[5];
        for (int q = 0; q < 5; ++q) { pvl[q] = S5(o, pv, i, j, q + 1); tgt[q] = S5(o, pv_target, i, j, q + 1); }
        double rho = o->rhovec[x], Vr = o->Vrvec[x], Vz = o->Vzvec[x], T = o->Tvec[x];
        if (pt->bc == AXJ_BC_SAT_FARFIELD) {
          if (j == 1) continue;
          if (adir == 1) {
            rec_op(o, pn, i, j);
            eigen_matrices(0, rho, Vz, T, gam, &e);
            o->Tb[BLK(o, i, j)] = T;
            /* compute_SAT_RHS :439-469 */
            for (int q = 0; q < 5; ++q)
              e.lam[q][q] = pt->bc_dir > 0 ? (fabs(e.lam[q][q]) + e.lam[q][q]) / 2.0
                                           : (fabs(e.lam[q][q]) - e.lam[q][q]) / 2.0;
            for (int q = 0; q < 5; ++q) w[q] = pvl[q] - tgt[q];
            matvec(e.Ti, w, w);
            tlam_w(e.Tm, e.lam, w, out);
            for (int q = 0; q < 5; ++q)
              S5(o, rhs, i, j, q + 1) = S5(o, rhs, i, j, q + 1) + sigma_1 * o->dxidz[x] * one_by_h_44 * out[q];
          }
        } else if (pt->bc == AXJ_BC_SAT_NOSLIP_WALL) {
          if (adir == 1 || adir == 2) {
            rec_op(o, pn, i, j);
            int rd = adir == 2;
            double tI[5];
            tI[0] = pvl[0];
            tI[1] = rd ? 0.0 : pvl[1];
            tI[2] = pvl[2];
            tI[3] = rd ? pvl[3] : 0.0;
            tI[4] = pvl[4];
            for (int q = 0; q < 5; ++q) S5(o, pv_targetI, i, j, q + 1) = tI[q];
            eigen_matrices(rd, rho, rd ? Vr : Vz, T, gam, &e);
            o->Tb[BLK(o, i, j)] = T;
            for (int q = 0; q < 5; ++q)
              e.lam[q][q] = pt->bc_dir > 0 ? (fabs(e.lam[q][q]) + e.lam[q][q]) / 2.0
                                           : (fabs(e.lam[q][q]) - e.lam[q][q]) / 2.0;
            for (int q = 0; q < 5; ++q) w[q] = pvl[q] - tI[q];
            matvec(e.Ti, w, w);
            tlam_w(e.Tm, e.lam, w, out);
            const double met = rd ? o->detadr[x] : o->dxidz[x];
            for (int q = 0; q < 5; ++q)
              S5(o, rhs, i, j, q + 1) = S5(o, rhs, i, j, q + 1) + sigma_1 * met * one_by_h_44 * out[q];
            double tV[5] = {pvl[0], 0.0, 0.0, 0.0, tgt[4]};
            for (int q = 0; q < 5; ++q) S5(o, pv_targetV, i, j, q + 1) = tV[q];
            for (int q = 0; q < 5; ++q)
              S5(o, rhs, i, j, q + 1) =
                  S5(o, rhs, i, j, q + 1) + sigma_2 * met * one_by_h_44 * (pvl[q] - tV[q]);
          }
        } else if (pt->bc == AXJ_BC_NSCBC_NONREFLECTING) {
          if (j == 1) continue;
          double Vt = o->Vtvec[x];
          o->Tb[BLK(o, i, j)] = T;
          double drhodr = o->drhodr[x], dVrdr = o->dVrdr[x], dVtdr = o->dVtdr[x], dVzdr = o->dVzdr[x];
          double dTdr = o->dTdr[x], dpdr = o->dpdr[x];
          double drhodz = o->drhodz[x], dVrdz = o->dVrdz[x], dVtdz = o->dVtdz[x], dVzdz = o->dVzdz[x];
          double dTdz = o->dTdz[x], dpdz = o->dpdz[x];
          (void)Vt;
          if (adir == 1) {
            S5(o, rhs, i, j, 1) = S5(o, rhs, i, j, 1) + (Vz * drhodz + rho * dVzdz);
            S5(o, rhs, i, j, 2) = S5(o, rhs, i, j, 2) + Vz * dVrdz;
            S5(o, rhs, i, j, 3) = S5(o, rhs, i, j, 3) + Vz * dVtdz;
            S5(o, rhs, i, j, 4) = S5(o, rhs, i, j, 4) + (Vz * dVzdz + 1.0 / (gam * rho) * dpdz);
            S5(o, rhs, i, j, 5) = S5(o, rhs, i, j, 5) + (Vz * dTdz + (gam - 1.0) * T * dVzdz);
            eigen_matrices(0, rho, Vz, T, gam, &e);
          } else if (adir == 2) {
            S5(o, rhs, i, j, 1) = S5(o, rhs, i, j, 1) + (Vr * drhodr + rho * dVrdr);
            S5(o, rhs, i, j, 2) = S5(o, rhs, i, j, 2) + (Vr * dVrdr + 1.0 / (gam * rho) * dpdr);
            S5(o, rhs, i, j, 3) = S5(o, rhs, i, j, 3) + Vr * dVtdr;
            S5(o, rhs, i, j, 4) = S5(o, rhs, i, j, 4) + Vr * dVzdr;
            S5(o, rhs, i, j, 5) = S5(o, rhs, i, j, 5) + (Vr * dTdr + (gam - 1.0) * T * dVrdr);
            eigen_matrices(1, rho, Vr, T, gam, &e);
          } else {
            continue;
          }
          rec_op(o, pn, i, j);
          /* ComputeNSCBCRHS :471-545: the non-reflecting face always uses z-derivatives */
          double dv[5] = {drhodz, dVrdz, dVtdz, dVzdz, dTdz};
          matvec(e.Ti, dv, w);
          for (int q = 0; q < 5; ++q) {
            if (pt->bc_dir > 0) { if (e.lam[q][q] > 0.0) w[q] = 0.0; }
            else if (pt->bc_dir < 0) { if (e.lam[q][q] < 0.0) w[q] = 0.0; }
          }
          tlam_w(e.Tm, e.lam, w, out);
          for (int q = 0; q < 5; ++q) S5(o, rhs, i, j, q + 1) = S5(o, rhs, i, j, q + 1) - out[q];
        } else if (pt->bc == AXJ_BC_NSCBC_NOSLIP_WALL) {
          double drhodr = o->drhodr[x], dVrdr = o->dVrdr[x];
          double drhodz = o->drhodz[x], dVzdz = o->dVzdz[x];
          double dv[5];
          if (adir == 1) {
            eigen_matrices(0, rho, Vz, T, gam, &e);
            o->Tb[BLK(o, i, j)] = T;
            dv[0] = o->drhodz[x]; dv[1] = o->dVrdz[x]; dv[2] = o->dVtdz[x]; dv[3] = o->dVzdz[x]; dv[4] = o->dTdz[x];
          } else if (adir == 2) {
            eigen_matrices(1, rho, Vr, T, gam, &e);
            o->Tb[BLK(o, i, j)] = T;
            dv[0] = o->drhodr[x]; dv[1] = o->dVrdr[x]; dv[2] = o->dVtdr[x]; dv[3] = o->dVzdr[x]; dv[4] = o->dTdr[x];
          } else {
            continue;
          }
          rec_op(o, pn, i, j);
          matvec(e.Ti, dv, w);
          if (pt->bc_dir < 0) w[3] = -1.0 * w[4];
          else if (pt->bc_dir > 0) w[4] = -1.0 * w[3];
          tlam_w(e.Tm, e.lam, w, out);
          if (adir == 1) S5(o, rhs, i, j, 1) = S5(o, rhs, i, j, 1) + (Vz * drhodz + rho * dVzdz);
          else S5(o, rhs, i, j, 1) = S5(o, rhs, i, j, 1) + (Vr * drhodr + rho * dVrdr);
          for (int q = 0; q < 5; ++q) S5(o, rhs, i, j, q + 1) = S5(o, rhs, i, j, q + 1) - out[q];
          for (int q = 2; q <= 5; ++q) S5(o, rhs, i, j, q) = 0.0;
        }
      }
  }
}

static void sponge_bcs(axo* o) {
  const double n_sponge = 2.0;
  const double st = o->p.sponge_start_top, At = o->p.sponge_A_top;
  const double el = o->p.sponge_end_left, Al = o->p.sponge_A_left;
  I8 Nz = o->Nz, Nr = o->Nr;
#pragma omp parallel for schedule(static)
  for (I8 j = 1; j <= Nr; ++j)
    for (I8 i = 1; i <= Nz; ++i) {
      if (H(o, rvec, i, j) >= st) {
        for (int e = 1; e <= 5; ++e) {
          double zeta = (H(o, rvec, i, j) - st) / (H(o, rvec, i, o->rhi[o->br[j]]) - st);
          S5(o, rhs, i, j, e) =
              S5(o, rhs, i, j, e) - At * pow(zeta, n_sponge) * (S5(o, pv, i, j, e) - S5(o, pv_target, i, j, e));
        }
      }
    }
#pragma omp parallel for schedule(static)
  for (I8 j = 2; j <= Nr; ++j)
    for (I8 i = 1; i <= Nz; ++i) {
      if (H(o, zvec, i, j) <= el) {
        for (int e = 1; e <= 5; ++e) {
          double zeta = (el - H(o, zvec, i, j)) / (el);
          S5(o, rhs, i, j, e) =
              S5(o, rhs, i, j, e) - Al * pow(zeta, n_sponge) * (S5(o, pv, i, j, e) - S5(o, pv_target, i, j, e));
        }
      }
    }
}

/* ControlForcingTerms (ModControlForcing.f90:45-61) with the matrix/window from params. */
static void control_forcing(axo* o) {
  const axj_params* p = &o->p;
#pragma omp parallel for schedule(static)
  for (I8 j = 1; j <= o->Nr; ++j)
    for (I8 i = 1; i <= o->Nz; ++i) {
      double zl = H(o, zvec, i, j), rl = H(o, rvec, i, j);
      double dz = zl - p->forcing_z0, dr = rl - p->forcing_r0;
      double G = exp(-((dz * dz) / (p->forcing_lz * p->forcing_lz)) - (dr * dr) / (p->forcing_lr * p->forcing_lr));
      for (int e = 1; e <= 5; ++e)
        for (int k = 1; k <= 5; ++k)
          S5(o, rhs, i, j, e) = S5(o, rhs, i, j, e) + p->forcing_alpha * p->forcing_mat[(e - 1) * 5 + (k - 1)] * G *
                                                          (S5(o, pv, i, j, k) - S5(o, pv_target, i, j, k));
    }
}

/* Harmonic inflow forcing (control_forcing = 2): an extension with no counterpart in the
 * reference, rhs(V_z) += A omega G cos(omega t) in the ControlForcingTerms window. */
static void harmonic_forcing(axo* o, double t) {
  const axj_params* p = &o->p;
  const double omega = 2.0 * 3.141592653589793 * p->harmonic_st * p->harmonic_uj;
  const double cwt = cos(omega * t);
#pragma omp parallel for schedule(static)
  for (I8 j = 1; j <= o->Nr; ++j)
    for (I8 i = 1; i <= o->Nz; ++i) {
      double zl = H(o, zvec, i, j), rl = H(o, rvec, i, j);
      double dz = zl - p->forcing_z0, dr = rl - p->forcing_r0;
      double G = exp(-((dz * dz) / (p->forcing_lz * p->forcing_lz)) - (dr * dr) / (p->forcing_lr * p->forcing_lr));
      S5(o, rhs, i, j, 4) = S5(o, rhs, i, j, 4) + p->harmonic_amp * omega * G * cwt;
    }
}

/* ComputeRHS (ModRHS.f90:5-258) */
/* T = Tvec(Nz,Nr) at the end of a rank's RHS loops (ModRHS.f90:76,145), which start at
   row 2 on the axis rank (nbrs(2) < 0) and at row 1 elsewhere. */
static void set_T_block_ends(axo* o) {
  for (I8 b = 0; b < o->nbz * o->nbr; ++b) {
    const I8 bzz = b % o->nbz, brr = b / o->nbz;
    const I8 j0 = (o->rlo[brr] == 1) ? 2 : o->rlo[brr];
    if (o->rhi[brr] >= j0) o->Tb[b] = H(o, Tvec, o->zhi[bzz], o->rhi[brr]);
  }
}

static void compute_rhs(axo* o) {
  const I8 Nz = o->Nz, Nr = o->Nr;
  const double gam = o->p.gam, Re = o->p.Re, Pr = o->p.Pr;
  deriv1(o, o->rhovec, 1, o->drhodz);
  deriv1(o, o->Vrvec, 1, o->dVrdz);
  deriv1(o, o->Vtvec, 1, o->dVtdz);
  deriv1(o, o->Vzvec, 1, o->dVzdz);
  deriv1(o, o->Tvec, 1, o->dTdz);
  deriv1(o, o->pvec, 1, o->dpdz);
  deriv1(o, o->rhovec, 2, o->drhodr);
  deriv1(o, o->Vrvec, 2, o->dVrdr);
  deriv1(o, o->Vtvec, 2, o->dVtdr);
  deriv1(o, o->Vzvec, 2, o->dVzdr);
  deriv1(o, o->Tvec, 2, o->dTdr);
  deriv1(o, o->pvec, 2, o->dpdr);
  if (o->p.shock_capturing == 1) shock_capturing(o);
  memset(o->rhs, 0, sizeof(double) * (size_t)Nz * (size_t)Nr * 5);
  const I8 j0 = 2; /* nbrs(2) < 0: the axis row j = 1 is skipped */
#pragma omp parallel for schedule(static)
  for (I8 j = j0; j <= Nr; ++j)
    for (I8 i = 1; i <= Nz; ++i) {
      size_t x = HIX(o, i, j);
      double r = o->rvec[x], rho = o->rhovec[x], Vr = o->Vrvec[x], Vt = o->Vtvec[x], Vz = o->Vzvec[x], T = o->Tvec[x];
      double drhodr = o->drhodr[x], dVrdr = o->dVrdr[x], dVtdr = o->dVtdr[x], dVzdr = o->dVzdr[x];
      double dTdr = o->dTdr[x], dpdr = o->dpdr[x];
      double drhodz = o->drhodz[x], dVrdz = o->dVrdz[x], dVtdz = o->dVtdz[x], dVzdz = o->dVzdz[x];
      double dTdz = o->dTdz[x], dpdz = o->dpdz[x];
      S5(o, rhs, i, j, 1) = Vr * drhodr + Vz * drhodz + rho * (dVrdr + Vr / r + dVzdz);
      S5(o, rhs, i, j, 2) = Vr * dVrdr + Vz * dVrdz + 1.0 / (gam * rho) * dpdr;
      S5(o, rhs, i, j, 3) = Vr * dVtdr + Vr * Vt / r + Vz * dVtdz;
      S5(o, rhs, i, j, 4) = Vr * dVzdr + Vz * dVzdz + 1.0 / (gam * rho) * dpdz;
      S5(o, rhs, i, j, 5) = Vr * dTdr + Vz * dTdz + (gam - 1.0) * T * (dVrdr + Vr / r + dVzdz);
    }
  set_T_block_ends(o);
  {
    const size_t n = (size_t)Nz * (size_t)Nr * 5;
    for (size_t x = 0; x < n; ++x) o->rhs[x] = -1.0 * o->rhs[x];
  }
  if (o->p.do_viscous_terms == 1) {
    deriv2(o, o->Vrvec, 1, o->dVrdz, o->d2Vrdz2);
    deriv2(o, o->Vtvec, 1, o->dVtdz, o->d2Vtdz2);
    deriv2(o, o->Vzvec, 1, o->dVzdz, o->d2Vzdz2);
    deriv2(o, o->Tvec, 1, o->dTdz, o->d2Tdz2);
    deriv1(o, o->muvec, 1, o->dmudz);
    deriv1(o, o->kappavec, 1, o->dkappadz);
    deriv2(o, o->Vrvec, 2, o->dVrdr, o->d2Vrdr2);
    deriv2(o, o->Vtvec, 2, o->dVtdr, o->d2Vtdr2);
    deriv2(o, o->Vzvec, 2, o->dVzdr, o->d2Vzdr2);
    deriv2(o, o->Tvec, 2, o->dTdr, o->d2Tdr2);
    deriv1(o, o->muvec, 2, o->dmudr);
    deriv1(o, o->kappavec, 2, o->dkappadr);
    deriv1(o, o->dVrdz, 2, o->d2Vrdzdr);
    deriv1(o, o->dVzdz, 2, o->d2Vzdzdr);
    const int sc = o->p.shock_capturing == 1;
#pragma omp parallel for schedule(static)
    for (I8 j = j0; j <= Nr; ++j)
      for (I8 i = 1; i <= Nz; ++i) {
        size_t x = HIX(o, i, j);
        double fourby3 = 29.0 / 15.0, oneby3 = 14.0 / 15.0, twoby3 = 1.0 / 15.0;
        double r = o->rvec[x];
        double onebyr = 1.0 / r;
        double rho = o->rhovec[x], Vr = o->Vrvec[x], Vt = o->Vtvec[x], Vz = o->Vzvec[x], T = o->Tvec[x];
        double mu = o->muvec[x], kappa = o->kappavec[x];
        double dVrdr = o->dVrdr[x], dVtdr = o->dVtdr[x], dVzdr = o->dVzdr[x];
        double dTdr = o->dTdr[x], dmudr = o->dmudr[x], dkappadr = o->dkappadr[x];
        double dVrdz = o->dVrdz[x], dVtdz = o->dVtdz[x], dVzdz = o->dVzdz[x];
        double dTdz = o->dTdz[x], dmudz = o->dmudz[x], dkappadz = o->dkappadz[x];
        double d2Vrdz2 = o->d2Vrdz2[x], d2Vtdz2 = o->d2Vtdz2[x], d2Vzdz2 = o->d2Vzdz2[x], d2Tdz2 = o->d2Tdz2[x];
        double d2Vrdr2 = o->d2Vrdr2[x], d2Vtdr2 = o->d2Vtdr2[x], d2Vzdr2 = o->d2Vzdr2[x], d2Tdr2 = o->d2Tdr2[x];
        double d2Vrdzdr = o->d2Vrdzdr[x], d2Vzdzdr = o->d2Vzdzdr[x];
        (void)T;
        if (sc) {
          double tmp = o->lambdavec[x] / o->muvec[x];
          fourby3 = 2.0 + tmp;
          oneby3 = 1.0 + tmp;
          twoby3 = -1.0 * tmp;
        }
        S5(o, rhs, i, j, 2) =
            S5(o, rhs, i, j, 2) +
            1.0 / (Re * rho) *
                (mu * (fourby3 * d2Vrdr2 + fourby3 * onebyr * dVrdr + oneby3 * d2Vzdzdr + d2Vrdz2 -
                       fourby3 * Vr * (onebyr * onebyr)) +
                 dmudr * (fourby3 * dVrdr - twoby3 * Vr * onebyr - twoby3 * dVzdz) + dmudz * (dVrdz + dVzdr));
        S5(o, rhs, i, j, 3) =
            S5(o, rhs, i, j, 3) + 1.0 / (Re * rho) *
                                      (mu * (d2Vtdr2 + d2Vtdz2 + onebyr * dVtdr - Vt * (onebyr * onebyr)) +
                                       dmudr * (dVtdr - Vt * onebyr) + dmudz * dVtdz);
        S5(o, rhs, i, j, 4) =
            S5(o, rhs, i, j, 4) +
            1.0 / (Re * rho) *
                (mu * (d2Vzdr2 + fourby3 * d2Vzdz2 + oneby3 * d2Vrdzdr + onebyr * dVzdr + oneby3 * onebyr * dVrdz) +
                 dmudr * (dVzdr + dVrdz) + dmudz * (fourby3 * dVzdz - twoby3 * dVrdr - twoby3 * Vr * onebyr));
        S5(o, rhs, i, j, 5) =
            S5(o, rhs, i, j, 5) +
            gam / (Re * Pr * rho) * (kappa * (d2Tdr2 + onebyr * dTdr + d2Tdz2) + dkappadr * dTdr + dkappadz * dTdz) +
            gam * (gam - 1.0) / Re * mu / rho *
                (dVrdr * (fourby3 * dVrdr - twoby3 * Vr * onebyr - twoby3 * dVzdz) +
                 (dVtdr - Vt * onebyr) * (dVtdr - Vr * onebyr) +
                 Vr * onebyr * (fourby3 * Vr * onebyr - twoby3 * dVrdr - twoby3 * dVzdz) + dVtdz * dVtdz +
                 dVzdz * (fourby3 * dVzdz - twoby3 * dVrdr - twoby3 * Vr * onebyr) +
                 (dVrdz + dVzdr) * (dVzdr + dVrdz));
      }
    set_T_block_ends(o);
  }
  if (o->p.control_forcing == 1) control_forcing(o);
  else if (o->p.control_forcing == 2) harmonic_forcing(o, o->t_stage);
  boundary_conditions(o);
  sponge_bcs(o);
}

/* axis_conditions (ModAxis.f90:5-35) */
static void axis_conditions(axo* o) {
  for (I8 i = 1; i <= o->Nz; ++i) {
    H(o, rhovec, i, 1) = -1.0 * dotr(&o->SBP1[0][1], 5, o, o->rhovec, i, 2) / o->SBP1[0][0];
    H(o, Vzvec, i, 1) = -1.0 * dotr(&o->SBP1[0][1], 5, o, o->Vzvec, i, 2) / o->SBP1[0][0];
    H(o, Tvec, i, 1) = -1.0 * dotr(&o->SBP1[0][1], 5, o, o->Tvec, i, 2) / o->SBP1[0][0];
  }
  for (I8 i = 1; i <= o->Nz; ++i) {
    S5(o, pv, i, 1, 1) = H(o, rhovec, i, 1);
    S5(o, pv, i, 1, 4) = H(o, Vzvec, i, 1);
    S5(o, pv, i, 1, 5) = H(o, Tvec, i, 1);
  }
}

/* ---------------- public oracle interface ---------------- */

void axo_destroy(axo* o) {
  if (!o) return;
  double** hf[] = {&o->zvec, &o->rvec, &o->dxidz, &o->detadr, &o->dzdxi, &o->drdeta, &o->ddxidxidz,
                   &o->ddetadetadr, &o->rhovec, &o->Vrvec, &o->Vtvec, &o->Vzvec, &o->Tvec, &o->pvec,
                   &o->muvec, &o->kappavec, &o->lambdavec, &o->betavec, &o->drhodz, &o->dVrdz, &o->dVtdz,
                   &o->dVzdz, &o->dTdz, &o->dpdz, &o->dmudz, &o->dkappadz, &o->drhodr, &o->dVrdr, &o->dVtdr,
                   &o->dVzdr, &o->dTdr, &o->dpdr, &o->dmudr, &o->dkappadr, &o->d2Vrdz2, &o->d2Vtdz2,
                   &o->d2Vzdz2, &o->d2Tdz2, &o->d2Vrdr2, &o->d2Vtdr2, &o->d2Vzdr2, &o->d2Tdr2, &o->d2Vrdzdr,
                   &o->d2Vzdzdr, &o->MgnStrRate, &o->d2Sdxi2, &o->d2Sdeta2, &o->d4Sdxi4, &o->d4Sdeta4,
                   &o->d2Tdxi2, &o->d2Tdeta2, &o->d4Tdxi4, &o->d4Tdeta4, &o->dilvec, &o->d2dildxi2,
                   &o->d2dildeta2, &o->d4dildxi4, &o->d4dildeta4, &o->mustarQ, &o->mustar, &o->betastarQ,
                   &o->betastar, &o->kappastarQ, &o->kappastar, &o->ibval, &o->deltvec, &o->pv, &o->pv_old,
                   &o->pv_target, &o->pv_targetI, &o->pv_targetV, &o->k1, &o->k2, &o->k3, &o->k4, &o->rhs};
  for (size_t k = 0; k < sizeof(hf) / sizeof(hf[0]); ++k) free(*hf[k]);
  free(o->is_it_i_patch); free(o->which_i_patch); free(o->is_it_j_patch); free(o->which_j_patch);
  free(o->patch);
  free(o->bz); free(o->br); free(o->zlo); free(o->zhi); free(o->rlo); free(o->rhi); free(o->Tb);
  free(o);
}

static int set_blocks(axo* o, I8 dz, I8 dr);

axo* axo_create(const axj_params* p, I8 Nz, I8 Nr, const double* zvec, const double* rvec, const double* ibval,
                const axj_patch* patches, I8 npatch) {
  if (Nz < 12 || Nr < 12) return NULL;
  axo* o = (axo*)calloc(1, sizeof(axo));
  o->Nz = Nz; o->Nr = Nr; o->LZ = Nz + 8; o->LR = Nr + 8;
  o->p = *p;
  double** hf[] = {&o->zvec, &o->rvec, &o->dxidz, &o->detadr, &o->dzdxi, &o->drdeta, &o->ddxidxidz,
                   &o->ddetadetadr, &o->rhovec, &o->Vrvec, &o->Vtvec, &o->Vzvec, &o->Tvec, &o->pvec,
                   &o->muvec, &o->kappavec, &o->lambdavec, &o->betavec, &o->drhodz, &o->dVrdz, &o->dVtdz,
                   &o->dVzdz, &o->dTdz, &o->dpdz, &o->dmudz, &o->dkappadz, &o->drhodr, &o->dVrdr, &o->dVtdr,
                   &o->dVzdr, &o->dTdr, &o->dpdr, &o->dmudr, &o->dkappadr, &o->d2Vrdz2, &o->d2Vtdz2,
                   &o->d2Vzdz2, &o->d2Tdz2, &o->d2Vrdr2, &o->d2Vtdr2, &o->d2Vzdr2, &o->d2Tdr2, &o->d2Vrdzdr,
                   &o->d2Vzdzdr, &o->MgnStrRate, &o->d2Sdxi2, &o->d2Sdeta2, &o->d4Sdxi4, &o->d4Sdeta4,
                   &o->d2Tdxi2, &o->d2Tdeta2, &o->d4Tdxi4, &o->d4Tdeta4, &o->dilvec, &o->d2dildxi2,
                   &o->d2dildeta2, &o->d4dildxi4, &o->d4dildeta4, &o->mustarQ, &o->mustar, &o->betastarQ,
                   &o->betastar, &o->kappastarQ, &o->kappastar};
  for (size_t k = 0; k < sizeof(hf) / sizeof(hf[0]); ++k) *hf[k] = halloc(o);
  o->ibval = ialloc(o, 1); o->deltvec = ialloc(o, 1);
  o->pv = ialloc(o, 5); o->pv_old = ialloc(o, 5); o->pv_target = ialloc(o, 5);
  o->pv_targetI = ialloc(o, 5); o->pv_targetV = ialloc(o, 5);
  o->k1 = ialloc(o, 5); o->k2 = ialloc(o, 5); o->k3 = ialloc(o, 5); o->k4 = ialloc(o, 5); o->rhs = ialloc(o, 5);
  size_t n = (size_t)Nz * (size_t)Nr;
  o->is_it_i_patch = (I8*)calloc(n, sizeof(I8)); o->which_i_patch = (I8*)calloc(n, sizeof(I8));
  o->is_it_j_patch = (I8*)calloc(n, sizeof(I8)); o->which_j_patch = (I8*)calloc(n, sizeof(I8));
  /* AssignGridCoordinates (ModInputOutput.f90:69-89) */
  for (I8 j = 1; j <= Nr; ++j)
    for (I8 i = 1; i <= Nz; ++i) {
      H(o, zvec, i, j) = zvec[IIX(o, i, j)];
      H(o, rvec, i, j) = rvec[IIX(o, i, j)];
      o->ibval[IIX(o, i, j)] = ibval[IIX(o, i, j)];
    }
  /* CreateAllPatches maps (ModPatch.f90:214-242) */
  o->no_bcs = npatch;
  o->patch = (axj_patch*)calloc((size_t)(npatch > 0 ? npatch : 1), sizeof(axj_patch));
  if (npatch > 0) memcpy(o->patch, patches, sizeof(axj_patch) * (size_t)npatch);
  for (I8 pn = 1; pn <= npatch; ++pn) {
    const axj_patch* pt = &o->patch[pn - 1];
    for (I8 i = pt->i_start; i <= pt->i_end; ++i)
      for (I8 j = pt->j_start; j <= pt->j_end; ++j) {
        if (i < 1 || i > Nz || j < 1 || j > Nr) continue;
        if (pt->bc_dir == -1 || pt->bc_dir == 1) { o->is_it_i_patch[IIX(o, i, j)] = 1; o->which_i_patch[IIX(o, i, j)] = pn; }
        if (pt->bc_dir == -2 || pt->bc_dir == 2) { o->is_it_j_patch[IIX(o, i, j)] = 1; o->which_j_patch[IIX(o, i, j)] = pn; }
      }
  }
  sbp_operator(o);
  /* metrics (ModSolver.f90:57-76) */
  compute_metric(o, o->zvec, 1, o->dzdxi);
  compute_metric(o, o->rvec, 2, o->drdeta);
  for (I8 i = 1; i <= Nz; ++i)
    for (I8 j = 1; j <= Nr; ++j) {
      H(o, dxidz, i, j) = 1.0 / H(o, dzdxi, i, j);
      H(o, detadr, i, j) = 1.0 / H(o, drdeta, i, j);
    }
  compute_metric(o, o->dxidz, 1, o->ddxidxidz);
  compute_metric(o, o->detadr, 2, o->ddetadetadr);
  /* one block: the whole grid; T is never assigned before the first ComputeRHS */
  if (set_blocks(o, 1, 1) != 0) { axo_destroy(o); return NULL; }
  return o;
}

/* DistributeGridDims / DistributeGridPoints (ModDecomp.f90:35-105) along one direction:
   N/d points per block (integer division, as ND/dims is), the last block the rest. */
static void partition(I8 N, I8 d, I8* lo, I8* hi, I8* of) {
  const I8 w = N / d;
  for (I8 b = 0; b < d; ++b) {
    lo[b] = b * w + 1;
    hi[b] = (b == d - 1) ? N : (b + 1) * w;
    for (I8 i = lo[b]; i <= hi[b]; ++i) of[i] = b;
  }
}

static int set_blocks(axo* o, I8 dz, I8 dr) {
  free(o->bz); free(o->br); free(o->zlo); free(o->zhi); free(o->rlo); free(o->rhi); free(o->Tb);
  o->nbz = dz; o->nbr = dr;
  o->bz = (I8*)calloc((size_t)o->Nz + 1, sizeof(I8));
  o->br = (I8*)calloc((size_t)o->Nr + 1, sizeof(I8));
  o->zlo = (I8*)calloc((size_t)dz, sizeof(I8)); o->zhi = (I8*)calloc((size_t)dz, sizeof(I8));
  o->rlo = (I8*)calloc((size_t)dr, sizeof(I8)); o->rhi = (I8*)calloc((size_t)dr, sizeof(I8));
  o->Tb = (double*)calloc((size_t)(dz * dr), sizeof(double));
  if (!o->bz || !o->br || !o->zlo || !o->zhi || !o->rlo || !o->rhi || !o->Tb) return AXJ_ERR_NOMEM;
  partition(o->Nz, dz, o->zlo, o->zhi, o->bz);
  partition(o->Nr, dr, o->rlo, o->rhi, o->br);
  return 0;
}

/* The replica of a dims_z x dims_r run (ModDecomp.f90). Every block must hold at least 8
   points each way, and no 4-wide closure strip may be split along its own direction (the
   rank's PatchCreation would then renumber its closure rows). Resets every block's T to
   0, as at the start of a run. */
int axo_set_decomposition(axo* o, I8 dims_z, I8 dims_r) {
  if (dims_z < 1 || dims_r < 1 || o->Nz / dims_z < 8 || o->Nr / dims_r < 8) return AXJ_ERR_ARG;
  int rc = set_blocks(o, dims_z, dims_r);
  if (rc != 0) return rc;
  for (I8 pn = 1; pn <= o->no_bcs; ++pn) {
    const axj_patch* pt = &o->patch[pn - 1];
    const int adir = (int)(pt->bc_dir < 0 ? -pt->bc_dir : pt->bc_dir);
    if (adir == 1 && o->bz[pt->i_start < 1 ? 1 : pt->i_start] != o->bz[pt->i_end > o->Nz ? o->Nz : pt->i_end])
      rc = AXJ_ERR_BADPATCH;
    if (adir == 2 && o->br[pt->j_start < 1 ? 1 : pt->j_start] != o->br[pt->j_end > o->Nr ? o->Nr : pt->j_end])
      rc = AXJ_ERR_BADPATCH;
  }
  if (rc != 0) set_blocks(o, 1, 1);
  return rc;
}

/* The stencil rows the oracle's operators select per point (zrow / rrow: the SBP row,
   4 where no patch applies), the blanking, and the face operations its bc loop applies
   (recorded from one pass of that loop on the current state; rhs, the SAT wall targets
   and the stale T are restored). x = (i-1) + (j-1)*Nz. */
void axo_point_maps(axo* o, uint8_t* zr, uint8_t* rr, uint8_t* blank, uint8_t* nops, uint64_t* ids) {
  for (I8 j = 1; j <= o->Nr; ++j)
    for (I8 i = 1; i <= o->Nz; ++i) {
      int row; I8 w0;
      const size_t x = IIX(o, i, j);
      int c = zrow(o, i, j, &row, &w0, 5);
      zr[x] = (uint8_t)(c == 1 ? row : (c == 0 ? 4 : 9));
      c = rrow(o, i, j, &row, &w0, 5);
      rr[x] = (uint8_t)(c == 1 ? row : (c == 0 ? 4 : 9));
      blank[x] = o->ibval[x] == 0.0;
    }
  const size_t n = (size_t)o->Nz * (size_t)o->Nr;
  const size_t n5 = n * 5, nb = (size_t)(o->nbz * o->nbr);
  double* save = (double*)malloc(3 * n5 * sizeof(double));
  double* Tsave = (double*)malloc(nb * sizeof(double));
  memcpy(save, o->rhs, n5 * sizeof(double));
  memcpy(save + n5, o->pv_targetI, n5 * sizeof(double));
  memcpy(save + 2 * n5, o->pv_targetV, n5 * sizeof(double));
  memcpy(Tsave, o->Tb, nb * sizeof(double));
  memset(nops, 0, n);
  memset(ids, 0, n * sizeof(uint64_t));
  o->rec_n = nops;
  o->rec_ids = ids;
  boundary_conditions(o);
  o->rec_n = NULL;
  o->rec_ids = NULL;
  memcpy(o->rhs, save, n5 * sizeof(double));
  memcpy(o->pv_targetI, save + n5, n5 * sizeof(double));
  memcpy(o->pv_targetV, save + 2 * n5, n5 * sizeof(double));
  memcpy(o->Tb, Tsave, nb * sizeof(double));
  free(save);
  free(Tsave);
}

/* The module scalar T of every block (block bz + dims_z * br). */
void axo_block_T(axo* o, double* out) {
  for (I8 b = 0; b < o->nbz * o->nbr; ++b) out[b] = o->Tb[b];
}

int axo_set_state(axo* o, const double* pv, const double* pv_target, I8 iteration, double time) {
  size_t n = (size_t)o->Nz * (size_t)o->Nr * 5;
  memcpy(o->pv, pv, n * sizeof(double));
  memcpy(o->pv_target, pv_target, n * sizeof(double));
  o->iteration = iteration;
  o->time = time;
  assign_values(o);
  return 0;
}

int axo_get_state(axo* o, double* pv) {
  memcpy(pv, o->pv, sizeof(double) * (size_t)o->Nz * (size_t)o->Nr * 5);
  return 0;
}

void axo_get_time(axo* o, I8* iteration, double* time, double* stale_T) {
  *iteration = o->iteration; *time = o->time; *stale_T = o->Tb[0];
}

/* ComputeTimeStep (ModInputOutput.f90:389-438) */
int axo_compute_dt(axo* o, double* delt) {
  const double Re = o->p.Re, Pr = o->p.Pr, CFL = o->p.CFL;
  const int phys = o->p.dt_mode == AXJ_DT_PHYSICAL;
#pragma omp parallel for schedule(static)
  for (I8 j = 1; j <= o->Nr; ++j)
    for (I8 i = 1; i <= o->Nz; ++i) {
      if (o->ibval[IIX(o, i, j)] == 0.0) { o->deltvec[IIX(o, i, j)] = 100.0; continue; }
      size_t x = HIX(o, i, j);
      double Ts = phys ? o->Tvec[x] : o->Tb[BLK(o, i, j)];
      double dx = o->dxidz[x], dr = o->detadr[x];
      double inv = fabs(o->Vzvec[x] * dx + o->Vrvec[x] * dr) + sqrt(Ts) * sqrt(dx * dx + dr * dr);
      double a = o->muvec[x] / Re, b = o->lambdavec[x] / Re, c = o->kappavec[x] / (Re * Pr);
      double mx = a; if (b > mx) mx = b; if (c > mx) mx = c;
      double s = fabs(dx) + fabs(dr);
      double visc = 2.0 * mx * (s * s);
      o->deltvec[IIX(o, i, j)] = CFL / (inv + visc);
    }
  double m = o->deltvec[0];
  size_t n = (size_t)o->Nz * (size_t)o->Nr;
  for (size_t x = 1; x < n; ++x) if (o->deltvec[x] < m) m = o->deltvec[x];
  o->delt = m;
  *delt = m;
  if (m == 100.0) return AXJ_ERR_DT_BLOWUP;
  return 0;
}

/* RK4 (ModRungeKutta.f90:5-171) */
int axo_rk4_step(axo* o, double delt) {
  const size_t n = (size_t)o->Nz * (size_t)o->Nr * 5;
  o->delt = delt;
  memcpy(o->pv_old, o->pv, n * sizeof(double));
  double* ks[4] = {o->k1, o->k2, o->k3, o->k4};
  const double a[3] = {0.5, 0.5, 1.0};
  const double cs[4] = {0.0, 0.5, 0.5, 1.0};
  for (int s = 0; s < 4; ++s) {
    assign_values(o);
    o->t_stage = (o->time + delt) - delt + cs[s] * delt;
    compute_rhs(o);
    double* k = ks[s];
    for (size_t x = 0; x < n; ++x) k[x] = delt * o->rhs[x];
    if (s < 3) {
      if (s < 2) for (size_t x = 0; x < n; ++x) o->pv[x] = o->pv_old[x] + 0.5 * k[x];
      else for (size_t x = 0; x < n; ++x) o->pv[x] = o->pv_old[x] + k[x];
      (void)a;
      axis_conditions(o);
    }
  }
  const size_t np = (size_t)o->Nz * (size_t)o->Nr;
  for (int e = 0; e < 5; ++e)
    for (size_t q = 0; q < np; ++q) {
      if (o->ibval[q] == 0.0) continue;
      size_t x = q + (size_t)e * np;
      o->pv[x] = o->pv_old[x] + 1.0 / 6.0 * o->k1[x] + 1.0 / 3.0 * (o->k2[x] + o->k3[x]) + 1.0 / 6.0 * o->k4[x];
    }
  axis_conditions(o);
  assign_values(o);
  o->time = o->time + delt;
  o->iteration = o->iteration + 1;
  return 0;
}

/* AssignValues + ComputeRHS on a given pv; the state is restored afterwards. */
int axo_rhs(axo* o, const double* pv, double* rhs) {
  const size_t n = (size_t)o->Nz * (size_t)o->Nr * 5;
  double* save = (double*)malloc(n * sizeof(double));
  memcpy(save, o->pv, n * sizeof(double));
  const size_t nb = (size_t)(o->nbz * o->nbr);
  double* Tsave = (double*)malloc(nb * sizeof(double));
  memcpy(Tsave, o->Tb, nb * sizeof(double));
  memcpy(o->pv, pv, n * sizeof(double));
  assign_values(o);
  o->t_stage = o->time;
  compute_rhs(o);
  memcpy(rhs, o->rhs, n * sizeof(double));
  memcpy(o->pv, save, n * sizeof(double));
  memcpy(o->Tb, Tsave, nb * sizeof(double));
  free(Tsave);
  assign_values(o);
  free(save);
  return 0;
}

/* Interior (Nz,Nr) <-> halo-padded helpers for the unit entry points. */
static double* to_halo(axo* o, const double* f) {
  double* h = halloc(o);
  for (I8 j = 1; j <= o->Nr; ++j)
    for (I8 i = 1; i <= o->Nz; ++i) h[HIX(o, i, j)] = f[IIX(o, i, j)];
  return h;
}
static void from_halo(axo* o, const double* h, double* f) {
  for (I8 j = 1; j <= o->Nr; ++j)
    for (I8 i = 1; i <= o->Nz; ++i) f[IIX(o, i, j)] = h[HIX(o, i, j)];
}

int axo_deriv1(axo* o, const double* var, I8 dirn, double* out) {
  double *hv = to_halo(o, var), *ho = halloc(o);
  deriv1(o, hv, (int)dirn, ho);
  from_halo(o, ho, out);
  free(hv); free(ho);
  return 0;
}
int axo_deriv2(axo* o, const double* var, I8 dirn, const double* first, double* out) {
  double *hv = to_halo(o, var), *hf = to_halo(o, first), *ho = halloc(o);
  deriv2(o, hv, (int)dirn, hf, ho);
  from_halo(o, ho, out);
  free(hv); free(hf); free(ho);
  return 0;
}
int axo_deriv2comp(axo* o, const double* var, I8 dirn, double* out) {
  double *hv = to_halo(o, var), *ho = halloc(o);
  deriv2comp(o, hv, (int)dirn, ho);
  from_halo(o, ho, out);
  free(hv); free(ho);
  return 0;
}
int axo_tgfilter(axo* o, const double* var, I8 dirn, I8 inplace, double* out) {
  double* ho = to_halo(o, out);
  if (inplace) {
    tgfilter(o, ho, (int)dirn, ho);
  } else {
    double* hv = to_halo(o, var);
    tgfilter(o, hv, (int)dirn, ho);
    free(hv);
  }
  from_halo(o, ho, out);
  free(ho);
  return 0;
}
/* ComputeArtTransCoeffs' sensor on pv: mustar, betastar, kappastar. */
int axo_sensor(axo* o, const double* pv, double* mustar, double* betastar, double* kappastar) {
  const size_t n = (size_t)o->Nz * (size_t)o->Nr * 5;
  double* save = (double*)malloc(n * sizeof(double));
  memcpy(save, o->pv, n * sizeof(double));
  memcpy(o->pv, pv, n * sizeof(double));
  assign_values(o);
  deriv1(o, o->Vrvec, 1, o->dVrdz);
  deriv1(o, o->Vzvec, 1, o->dVzdz);
  deriv1(o, o->Vrvec, 2, o->dVrdr);
  deriv1(o, o->Vzvec, 2, o->dVzdr);
  shock_capturing(o);
  from_halo(o, o->mustar, mustar);
  from_halo(o, o->betastar, betastar);
  from_halo(o, o->kappastar, kappastar);
  memcpy(o->pv, save, n * sizeof(double));
  assign_values(o);
  free(save);
  return 0;
}
/* Operator tables and 1-D metrics, for the known-answer tests. */
void axo_tables(axo* o, double* sbp1, double* sbp2, double* tg) {
  memcpy(sbp1, o->SBP1, sizeof(o->SBP1));
  memcpy(sbp2, o->SBP2, sizeof(o->SBP2));
  memcpy(tg, o->TG, sizeof(o->TG));
}
void axo_metrics(axo* o, double* dxidz, double* detadr, double* ddxidxidz, double* ddetadetadr) {
  from_halo(o, o->dxidz, dxidz);
  from_halo(o, o->detadr, detadr);
  from_halo(o, o->ddxidxidz, ddxidxidz);
  from_halo(o, o->ddetadetadr, ddetadetadr);
}

/* CreateAllPatches + PatchCreation (ModPatch.f90:117-309) for one block holding the
 * whole grid (istart = jstart = 1, Nz = Nz_grid, Nr = Nr_grid), restated with the
 * reference's scan: the first and the last block point (i outer, j inner) inside the
 * 4-wide strip become the patch corners. */
int axo_patches_from_records(const axj_bc_record* rec, I8 nrec, I8 Nz, I8 Nr, axj_patch* out, I8* npatch) {
  I8 bcno = 0;
  for (I8 k = 0; k < nrec; ++k) {
    I8 bctype = rec[k].bc, bcdir = rec[k].bc_dir;
    I8 bcistart = rec[k].istart, bciend = rec[k].iend, bcjstart = rec[k].jstart, bcjend = rec[k].jend;
    I8 exitvalue = 0, procbcistart = 0, procbciend = 0, procbcjstart = 0, procbcjend = 0;
    if (bcistart == -1) bcistart = Nz;
    if (bcjstart == -1) bcjstart = Nr;
    if (bciend == -1) bciend = Nz;
    if (bcjend == -1) bcjend = Nr;
    I8 pis = 0, pie = 0, pjs = 0, pje = 0;
    for (I8 i = 1; i <= Nz; ++i)
      for (I8 j = 1; j <= Nr; ++j) {
        I8 i_indx = i, j_indx = j;
        if (bcdir == 1) { pis = bcistart; pie = bcistart + 3; pjs = bcjstart; pje = bcjend; }
        else if (bcdir == -1) { pis = bciend - 3; pie = bciend; pjs = bcjstart; pje = bcjend; }
        else if (bcdir == 2) { pis = bcistart; pie = bciend; pjs = bcjstart; pje = bcjstart + 3; }
        else if (bcdir == -2) { pis = bcistart; pie = bciend; pjs = bcjend - 3; pje = bcjend; }
        I8 value1 = (i_indx - pis) * (i_indx - pie);
        I8 value2 = (j_indx - pjs) * (j_indx - pje);
        if (exitvalue == 0) {
          if (value1 <= 0 && value2 <= 0) { procbcistart = i_indx; procbcjstart = j_indx; exitvalue = 1; }
        } else {
          if (value1 <= 0 && value2 <= 0) { procbciend = i_indx; procbcjend = j_indx; }
        }
      }
    if (exitvalue != 0) {
      axj_patch p;
      p.bc = bctype;
      p.bc_dir = bcdir;
      I8 istartval = procbcistart, iendval = procbciend, jstartval = procbcjstart, jendval = procbcjend;
      p.i_start = p.i_end = p.j_start = p.j_end = 0;
      if (bcdir == 1) { p.i_start = istartval; p.i_end = istartval + 3; p.j_start = jstartval; p.j_end = jendval; }
      if (bcdir == -1) { p.i_start = iendval - 3; p.i_end = iendval; p.j_start = jstartval; p.j_end = jendval; }
      if (bcdir == 2) { p.i_start = istartval; p.i_end = iendval; p.j_start = jstartval; p.j_end = jstartval + 3; }
      if (bcdir == -2) { p.i_start = istartval; p.i_end = iendval; p.j_start = jendval - 3; p.j_end = jendval; }
      out[bcno++] = p;
    }
  }
  *npatch = bcno;
  return 0;
}
