// axj_kernels.cu -- sm_100a kernels of the per-step hot path.
//
//  stage_kernel<H, GEN>  one fused RK4 stage: loads a (z,r) tile of the stage
//                        input plus its SBP halo into shared memory, forms the 26
//                        derivatives of ComputeRHS, the inviscid and viscous terms,
//                        forcing, SAT/NSCBC face terms, sponges, and the RK4 stage
//                        update with the axis closure (ModRHS.f90, ModBC.f90,
//                        ModAxis.f90, ModRungeKutta.f90).
//                        H = 2 / GEN = false: interior tiles, centred rows only.
//                        H = 5 / GEN = true : tiles with closure rows, blanked
//                        points, face points or domain edges.
//  dt_kernel             ComputeTimeStep with a warp-shuffle / block / last-block
//                        FP64 min reduction (ModInputOutput.f90:389-438).
//  sensor kernels        the artificial-diffusivity chain (ModShockCapturing.f90),
//                        with the in-place z filter as a chunked recurrence.
#include <cuda_runtime.h>

#include <algorithm>

#include "axj_kernels.cuh"
#include "axj_point.cuh"

namespace axj {

__constant__ double cSBP1[9][6];
__constant__ double cSBP2[9][6];
__constant__ double cTG[9][11];
__constant__ PatchDev cPatch[MAX_PATCHES];

void upload_tables(const double sbp1[9][6], const double sbp2[9][6], const double tg[9][11],
                   const PatchDev* patches, int npatch, cudaStream_t s) {
  cudaMemcpyToSymbolAsync(cSBP1, sbp1, sizeof(double) * 54, 0, cudaMemcpyHostToDevice, s);
  cudaMemcpyToSymbolAsync(cSBP2, sbp2, sizeof(double) * 54, 0, cudaMemcpyHostToDevice, s);
  cudaMemcpyToSymbolAsync(cTG, tg, sizeof(double) * 99, 0, cudaMemcpyHostToDevice, s);
  if (npatch > 0) cudaMemcpyToSymbolAsync(cPatch, patches, sizeof(PatchDev) * npatch, 0, cudaMemcpyHostToDevice, s);
}

// Round-to-nearest arithmetic that the compiler may not contract into an FMA; used
// where the reference's two-step rounding (k = delt*rhs, then the RK sums) is kept.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }

// Dot product of an SBP row with a window in shared memory (stride in doubles).
// The sequence starts from the first product, as DOT_PRODUCT's 0 + a1*b1 does.
template <int N>
__device__ __forceinline__ double dotc(const double* __restrict__ c, const double* __restrict__ v, int stride) {
  double s = c[0] * v[0];
#pragma unroll
  for (int m = 1; m < N; ++m) s = s + c[m] * v[m * stride];
  return s;
}

// Derivative stencil of SBP row `row` (0..8; 9 = none) at p (pointer to the point's
// own value), stride 1 along z or the smem row length along r.
__device__ __forceinline__ double sbp_row_apply(const double (*tab)[6], int row, const double* p, int stride) {
  if (row == 4) return dotc<5>(tab[4], p - 2 * stride, stride);
  if (row >= 9) return 0.0;
  const int w0 = sbp_w0(row);
  return dotc<6>(tab[row], p + w0 * stride, stride);
}

template <bool GEN>
__device__ __forceinline__ double d1(int row, const double* p, int stride) {
  if (!GEN) return dotc<5>(cSBP1[4], p - 2 * stride, stride);
  return sbp_row_apply(cSBP1, row, p, stride);
}
template <bool GEN>
__device__ __forceinline__ double d2(int row, const double* p, int stride) {
  if (!GEN) return dotc<5>(cSBP2[4], p - 2 * stride, stride);
  return sbp_row_apply(cSBP2, row, p, stride);
}

// p = rho*T taps for dp/dz, dp/dr: the reference differentiates pvec = rhovec*Tvec.
template <bool GEN>
__device__ __forceinline__ double d1_p(int row, const double* rho, const double* T, int stride) {
  double v[6];
  int w0, n;
  if (!GEN || row == 4) { w0 = -2; n = 5; }
  else if (row >= 9) return 0.0;
  else { w0 = sbp_w0(row); n = 6; }
  const int r = GEN ? row : 4;
#pragma unroll
  for (int m = 0; m < 6; ++m)
    if (m < n) v[m] = rho[(w0 + m) * stride] * T[(w0 + m) * stride];
  double s = cSBP1[r][0] * v[0];
#pragma unroll
  for (int m = 1; m < 6; ++m)
    if (m < n) s = s + cSBP1[r][m] * v[m];
  return s;
}

// ---------------------------------------------------------------------------
// Fused RK-stage kernel.
// ---------------------------------------------------------------------------
template <int H>
struct StageSmem {
  static constexpr int HZ = hz_of(H);
  static constexpr int RZ = TZ + 2 * HZ;
  static constexpr int RR = TR + 2 * H;
  static constexpr int NPT = RZ * RR;
  // doubles: 5 state fields, mu_eff, kappa_eff, 2 dz-derivative fields
  static constexpr size_t bytes_main = sizeof(double) * (size_t)(7 * NPT + 2 * RR * TZ);
  static constexpr size_t bytes(bool gen) { return bytes_main + (gen ? sizeof(uint32_t) * NPT : 0); }
};

template <int H, bool GEN>
__global__ void __launch_bounds__(STAGE_THREADS) stage_kernel(const StageArgs a, const int2* __restrict__ tiles) {
  using SM = StageSmem<H>;
  constexpr int HZ = SM::HZ, RZ = SM::RZ, RR = SM::RR, NPT = SM::NPT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* sU = reinterpret_cast<double*>(smem_raw);  // [5][RR][RZ]
  double* sMu = sU + 5 * NPT;                        // [RR][RZ]
  double* sKa = sMu + NPT;                           // [RR][RZ]
  double* sDz = sKa + NPT;                           // [2][RR][TZ]
  uint32_t* sDesc = reinterpret_cast<uint32_t*>(sDz + 2 * RR * TZ);

  const int tid = threadIdx.x;
  const int2 t0 = tiles[blockIdx.x];
  const int i0 = t0.x, j0 = t0.y;
  const int Nz = a.g.Nz, Nr = a.g.Nr;
  const long long P = a.g.P, PL = a.g.plane;
  const bool sc = a.c.shock_capturing != 0;

  // ---- phase 1: state + halo -> smem; mu = T**0.666 (AssignValues) on the cross
  for (int idx = tid; idx < NPT; idx += STAGE_THREADS) {
    const int rr = idx / RZ, rz = idx - rr * RZ;
    const int i = i0 - HZ + rz, j = j0 - H + rr;
    const bool in = (!GEN) || (i >= 0 && i < Nz && j >= 0 && j < Nr);
    double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    uint32_t dsc = make_desc(ROW_NONE, ROW_NONE, false, 0);
    if (in) {
      const long long o = (long long)j * P + i;
#pragma unroll
      for (int f = 0; f < 5; ++f) v[f] = __ldg(a.Uin + f * PL + o);
      if (GEN) dsc = __ldg(a.desc + o);
    }
#pragma unroll
    for (int f = 0; f < 5; ++f) sU[f * NPT + idx] = v[f];
    if (GEN) sDesc[idx] = dsc;
    const bool cross = (rr >= H && rr < H + TR && rz >= HZ - H && rz < HZ + TZ + H) || (rz >= HZ && rz < HZ + TZ);
    double mu = 0.0, ka = 0.0;
    if (in && cross) {
      mu = pow(v[4], 0.666);
      ka = mu;
      if (sc) {
        const long long o = (long long)j * P + i;
        mu = mu + __ldg(a.mustar + o);
        ka = ka + __ldg(a.kappastar + o);
      }
    }
    sMu[idx] = mu;
    sKa[idx] = ka;
  }
  __syncthreads();

  // ---- phase 2: dVr/dz and dVz/dz on the tile columns, all region rows (needed by
  // the mixed derivatives d/dr(dV/dz), ModRHS.f90:132-133)
  for (int idx = tid; idx < RR * TZ; idx += STAGE_THREADS) {
    const int rr = idx / TZ, c = idx - rr * TZ;
    const int i = i0 + c, j = j0 - H + rr;
    double dvr = 0.0, dvz = 0.0;
    const bool in = (!GEN) || (i < Nz && j >= 0 && j < Nr);
    if (in) {
      const int sidx = rr * RZ + HZ + c;
      int row = 4;
      if (GEN) {
        const uint32_t dsc = sDesc[sidx];
        row = desc_blank(dsc) ? (int)ROW_NONE : desc_zrow(dsc);
      }
      const double m = __ldg(a.dxidz + i);
      dvr = d1<GEN>(row, sU + 1 * NPT + sidx, 1) * m;
      dvz = d1<GEN>(row, sU + 3 * NPT + sidx, 1) * m;
    }
    sDz[idx] = dvr;
    sDz[RR * TZ + idx] = dvz;
  }
  __syncthreads();

  // ---- phase 3: one point per thread per pass
  const double dtv = a.stage > 0 ? *a.dt : 0.0;
  for (int pidx = tid; pidx < TZ * TR; pidx += STAGE_THREADS) {
    const int r = pidx / TZ, c = pidx - r * TZ;
    const int i = i0 + c, j = j0 + r;
    if (GEN && (i >= Nz || j >= Nr)) continue;
    const int rr = H + r, rz = HZ + c;
    const int sidx = rr * RZ + rz;
    int zr = 4, rw = 4;
    bool blank = false;
    uint32_t face = 0;
    if (GEN) {
      const uint32_t dsc = sDesc[sidx];
      blank = desc_blank(dsc);
      zr = blank ? (int)ROW_NONE : desc_zrow(dsc);
      rw = blank ? (int)ROW_NONE : desc_rrow(dsc);
      face = desc_face(dsc);
    }
    const double xz = __ldg(a.dxidz + i), xzz = __ldg(a.ddxidxidz + i);
    const double er = __ldg(a.detadr + j), err = __ldg(a.ddetadetadr + j);
    const double* pR = sU + 0 * NPT + sidx;
    const double* pVr = sU + 1 * NPT + sidx;
    const double* pVt = sU + 2 * NPT + sidx;
    const double* pVz = sU + 3 * NPT + sidx;
    const double* pT = sU + 4 * NPT + sidx;
    const double* pMu = sMu + sidx;
    const double* pKa = sKa + sidx;
    const int dzi = rr * TZ + c;

    Deriv d;
    // first derivatives (Compute1stDerivative: stencil, then * metric)
    d.drhodz = d1<GEN>(zr, pR, 1) * xz;
    d.dVrdz = sDz[dzi];
    d.dVtdz = d1<GEN>(zr, pVt, 1) * xz;
    d.dVzdz = sDz[RR * TZ + dzi];
    d.dTdz = d1<GEN>(zr, pT, 1) * xz;
    d.dpdz = d1_p<GEN>(zr, pR, pT, 1) * xz;
    d.drhodr = d1<GEN>(rw, pR, RZ) * er;
    d.dVrdr = d1<GEN>(rw, pVr, RZ) * er;
    d.dVtdr = d1<GEN>(rw, pVt, RZ) * er;
    d.dVzdr = d1<GEN>(rw, pVz, RZ) * er;
    d.dTdr = d1<GEN>(rw, pT, RZ) * er;
    d.dpdr = d1_p<GEN>(rw, pR, pT, RZ) * er;
    // second derivatives (Compute2ndDerivative: out*metric**2 + f'*metric')
    d.d2Vrdz2 = d2<GEN>(zr, pVr, 1) * (xz * xz) + d.dVrdz * xzz;
    d.d2Vtdz2 = d2<GEN>(zr, pVt, 1) * (xz * xz) + d.dVtdz * xzz;
    d.d2Vzdz2 = d2<GEN>(zr, pVz, 1) * (xz * xz) + d.dVzdz * xzz;
    d.d2Tdz2 = d2<GEN>(zr, pT, 1) * (xz * xz) + d.dTdz * xzz;
    d.d2Vrdr2 = d2<GEN>(rw, pVr, RZ) * (er * er) + d.dVrdr * err;
    d.d2Vtdr2 = d2<GEN>(rw, pVt, RZ) * (er * er) + d.dVtdr * err;
    d.d2Vzdr2 = d2<GEN>(rw, pVz, RZ) * (er * er) + d.dVzdr * err;
    d.d2Tdr2 = d2<GEN>(rw, pT, RZ) * (er * er) + d.dTdr * err;
    d.dmudz = d1<GEN>(zr, pMu, 1) * xz;
    d.dkappadz = sc ? d1<GEN>(zr, pKa, 1) * xz : d.dmudz;
    d.dmudr = d1<GEN>(rw, pMu, RZ) * er;
    d.dkappadr = sc ? d1<GEN>(rw, pKa, RZ) * er : d.dmudr;
    d.d2Vrdzdr = d1<GEN>(rw, sDz + dzi, TZ) * er;
    d.d2Vzdzdr = d1<GEN>(rw, sDz + RR * TZ + dzi, TZ) * er;

    Prim q;
    q.rho = *pR; q.Vr = *pVr; q.Vt = *pVt; q.Vz = *pVz; q.T = *pT;
    q.mu = *pMu;
    q.kappa = *pKa;
    const long long go = (long long)j * P + i;
    {
      // lambda = beta - 2/3 mu with beta = 0.6 mu (+ betastar), ModAssign.f90:22-23,
      // ModShockCapturing.f90:248-251
      const double mu0 = sc ? pow(q.T, 0.666) : q.mu;
      double beta = (3.0 / 5.0) * mu0;
      if (sc) beta = beta + __ldg(a.betastar + go);
      q.lambda = beta - (2.0 / 3.0) * q.mu;
    }
    const double rloc = __ldg(a.rc + j), zloc = __ldg(a.zc + i);
    const bool j1 = (j == 0);
    double rhs[5] = {-0.0, -0.0, -0.0, -0.0, -0.0};
    if (!j1) {
      rhs_inviscid(q, d, rloc, a.c.gam, rhs);
      if (a.c.do_viscous) rhs_viscous(q, d, rloc, a.c.gam, a.c.Re, a.c.Pr, sc, rhs);
    }
    double tg[5];
#pragma unroll
    for (int f = 0; f < 5; ++f) tg[f] = __ldg(a.target + f * PL + go);
    const double pv[5] = {q.rho, q.Vr, q.Vt, q.Vz, q.T};
    if (a.c.control_forcing) control_forcing(zloc, rloc, a.c, a.forcing, pv, tg, rhs);
    if (GEN && face) {
      const int n = __ldg(a.faces + face);
      for (int k = 0; k < n; ++k) {
        const int pid = __ldg(a.faces + face + 1 + k);
        face_op(cPatch[pid].bc, cPatch[pid].dir, j1, q, d, tg, xz, er, a.c.gam, rhs);
      }
    }
    sponge(zloc, rloc, j1, a.c, pv, tg, rhs);

    if (a.stage == 0) {
#pragma unroll
      for (int f = 0; f < 5; ++f) a.Uout[f * PL + go] = rhs[f];
      continue;
    }
    // ---- RK4 stage update (ModRungeKutta.f90:32-51, :134-146)
    const double c6 = 1.0 / 6.0, c3 = 1.0 / 3.0;
    double un[5];
#pragma unroll
    for (int f = 0; f < 5; ++f) {
      const double k = mul_rn(dtv, rhs[f]);
      const long long o = f * PL + go;
      if (a.stage == 1) {
        const double u0 = __ldg(a.U0 + o);
        un[f] = add_rn(u0, mul_rn(0.5, k));
        a.A[o] = add_rn(u0, mul_rn(c6, k));
      } else if (a.stage == 2) {
        const double u0 = __ldg(a.U0 + o);
        un[f] = add_rn(u0, mul_rn(0.5, k));
        a.B[o] = k;
      } else if (a.stage == 3) {
        const double u0 = __ldg(a.U0 + o);
        un[f] = add_rn(u0, k);
        a.A[o] = add_rn(a.A[o], mul_rn(c3, add_rn(a.B[o], k)));
      } else {
        un[f] = blank ? pv[f] : add_rn(a.A[o], mul_rn(c6, k));
      }
    }
    if (j1) {
      // axis_conditions (ModAxis.f90:14-29): rho, V_z, T at j = 1 from rows 2..6 of
      // the stage input (the vectors AssignValues filled before this stage).
      const double s00 = cSBP1[0][0];
      un[0] = -1.0 * dotc<5>(&cSBP1[0][1], pR + RZ, RZ) / s00;
      un[3] = -1.0 * dotc<5>(&cSBP1[0][1], pVz + RZ, RZ) / s00;
      un[4] = -1.0 * dotc<5>(&cSBP1[0][1], pT + RZ, RZ) / s00;
    }
#pragma unroll
    for (int f = 0; f < 5; ++f) a.Uout[f * PL + go] = un[f];
    if (a.stage == 4) {
      bool bad = false;
#pragma unroll
      for (int f = 0; f < 5; ++f) bad |= !isfinite(un[f]);
      if (bad) atomicOr(a.flags, 1);
      if (i == a.iT && j == a.jT) *a.staleT = q.T;
    }
  }
}

template <int H, bool GEN>
static cudaError_t launch_stage_t(const StageArgs& a, int ntiles, const int2* tiles, cudaStream_t s) {
  if (ntiles <= 0) return cudaSuccess;
  const size_t sm = StageSmem<H>::bytes(GEN);
  stage_kernel<H, GEN><<<ntiles, STAGE_THREADS, sm, s>>>(a, tiles);
  return cudaGetLastError();
}

cudaError_t launch_stage(const StageArgs& a, int ntiles_int, const int2* tiles_int, int ntiles_gen,
                         const int2* tiles_gen, cudaStream_t s) {
  cudaError_t e = launch_stage_t<H_GEN, true>(a, ntiles_gen, tiles_gen, s);
  if (e != cudaSuccess) return e;
  return launch_stage_t<H_INT, false>(a, ntiles_int, tiles_int, s);
}

// ---------------------------------------------------------------------------
// ComputeTimeStep: per-point dt, FP64 min via warp shuffles, one partial per
// block, and the last block to finish reduces the partials (no memset needed,
// the counter is returned to 0).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__global__ void __launch_bounds__(DT_THREADS) dt_kernel(const DtArgs a) {
  const int Nz = a.g.Nz, Nr = a.g.Nr;
  const long long n = (long long)Nz * Nr;
  const long long P = a.g.P, PL = a.g.plane;
  const double Tst = *a.staleT;
  const bool phys = a.c.dt_mode == DT_PHYSICAL;
  double m = 1.0e300;
  int bad = 0;
  for (long long p = (long long)blockIdx.x * DT_THREADS + threadIdx.x; p < n; p += (long long)gridDim.x * DT_THREADS) {
    const int j = (int)(p / Nz), i = (int)(p - (long long)j * Nz);
    const long long o = (long long)j * P + i;
    double v;
    if (desc_blank(__ldg(a.desc + o))) {
      v = 100.0;
    } else {
      const double Vr = __ldg(a.U + 1 * PL + o), Vz = __ldg(a.U + 3 * PL + o), T = __ldg(a.U + 4 * PL + o);
      const double mu = pow(T, 0.666);
      const double beta = (3.0 / 5.0) * mu;
      const double lambda = beta - (2.0 / 3.0) * mu;
      v = dt_point(Vz, Vr, phys ? T : Tst, mu, lambda, mu, __ldg(a.dxidz + i), __ldg(a.detadr + j), a.c);
    }
    if (!(v == v)) bad = 1;
    m = fmin(m, v);
  }
  __shared__ double sred[DT_THREADS / 32];
  __shared__ bool last;
  m = warp_min(m);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sred[w] = m;
  if (bad) atomicOr(a.flags, 1);
  __syncthreads();
  if (w == 0) {
    m = lane < DT_THREADS / 32 ? sred[lane] : 1.0e300;
    m = warp_min(m);
    if (lane == 0) {
      a.partial[blockIdx.x] = m;
      __threadfence();
      const unsigned int done = atomicAdd(a.counter, 1u);
      last = (done == gridDim.x - 1);
    }
  }
  __syncthreads();
  if (last) {
    __threadfence();
    double mm = 1.0e300;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += DT_THREADS) mm = fmin(mm, ((volatile double*)a.partial)[b]);
    mm = warp_min(mm);
    if (lane == 0) sred[w] = mm;
    __syncthreads();
    if (threadIdx.x == 0) {
      double r = sred[0];
      for (int k = 1; k < DT_THREADS / 32; ++k) r = fmin(r, sred[k]);
      *a.dt = r;
      if (a.advance) *a.time = *a.time + r;
      if (r == 100.0) atomicOr(a.flags, 2);
      *a.counter = 0u;
    }
  }
}

cudaError_t launch_dt(const DtArgs& a, int nblocks, cudaStream_t s) {
  dt_kernel<<<nblocks, DT_THREADS, 0, s>>>(a);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Global-memory stencils with patch-selected rows, for the sensor chain and the
// unit entry points. Reads outside the block return 0 (never-written halo cells).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double gval(const double* f, const Grid& g, int i, int j) {
  if (i < 0 || i >= g.Nz || j < 0 || j >= g.Nr) return 0.0;
  return __ldg(f + (long long)j * g.P + i);
}

// SBP (6-wide table) stencil along dirn (1 = z, 2 = r) with the point's row code.
__device__ __forceinline__ double gstencil6(const double (*tab)[6], int row, const double* f, const Grid& g, int i,
                                            int j, int dirn) {
  if (row >= 9) return 0.0;
  const int w0 = sbp_w0(row), n = sbp_len(row);
  const int di = dirn == 1 ? 1 : 0, dj = dirn == 1 ? 0 : 1;
  double s = tab[row][0] * gval(f, g, i + w0 * di, j + w0 * dj);
  for (int m = 1; m < n; ++m) s = s + tab[row][m] * gval(f, g, i + (w0 + m) * di, j + (w0 + m) * dj);
  return s;
}

__device__ __forceinline__ int row_of(uint32_t dsc, int dirn) {
  if (desc_blank(dsc)) return (int)ROW_NONE;
  return dirn == 1 ? desc_zrow(dsc) : desc_rrow(dsc);
}

// ---------------------------------------------------------------------------
// Fused sensor tile kernel (ModShockCapturing.f90:18-53, :108-222): strain-rate
// magnitude S, dilatation and f_sw from the first derivatives of V_r, V_z; the
// computational-space SBP2 of S, T and the dilatation twice over (fourth
// derivatives); the three quantities to be filtered. HS is the halo of S/T/dil
// (two SBP2 reaches), HF the reach of one stencil (2 interior, 5 with closures).
// ---------------------------------------------------------------------------
template <int HS, int HF>
struct SensSmem {
  static constexpr int HV = HS + HF;          // halo of V_r, V_z
  static constexpr int HVZ = hz_of(HV);
  static constexpr int VZ = TZ + 2 * HVZ, VR = TR + 2 * HV, NV = VZ * VR;
  static constexpr int SZ = TZ + 2 * HS, SR = TR + 2 * HS, NS = SZ * SR;
  static constexpr int DZ = TZ + 2 * HF;      // z-arm of the second derivatives: [TR][DZ]
  static constexpr int DR = TR + 2 * HF;      // r-arm: [DR][TZ]
  static constexpr size_t bytes(bool gen) {
    return sizeof(double) * (size_t)(2 * NV + 3 * NS + TR * DZ + DR * TZ + TR * TZ) +
           (gen ? sizeof(uint32_t) * NV : 0);
  }
};

template <int HS, int HF, bool GEN>
__global__ void __launch_bounds__(STAGE_THREADS) sensor_tile_kernel(const SensorArgs a, const int2* __restrict__ tiles) {
  using SM = SensSmem<HS, HF>;
  constexpr int HV = SM::HV, HVZ = SM::HVZ, VZ = SM::VZ, NV = SM::NV;
  constexpr int SZ = SM::SZ, NS = SM::NS, DZ = SM::DZ, DR = SM::DR;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* sVr = reinterpret_cast<double*>(smem_raw);  // [VR][VZ]
  double* sVz = sVr + NV;
  double* sS = sVz + NV;                               // [SR][SZ] x 3: S, T, dil
  double* sT = sS + NS;
  double* sD = sT + NS;
  double* sd2z = sD + NS;                              // [TR][DZ]
  double* sd2r = sd2z + TR * DZ;                       // [DR][TZ]
  double* sFsw = sd2r + DR * TZ;                       // [TR][TZ]
  uint32_t* sDesc = reinterpret_cast<uint32_t*>(sFsw + TR * TZ);

  const int tid = threadIdx.x;
  const int2 t0 = tiles[blockIdx.x];
  const int i0 = t0.x, j0 = t0.y;
  const Grid g = a.g;
  const int Nz = g.Nz, Nr = g.Nr;
  auto inside = [&](int i, int j) { return i >= 0 && i < Nz && j >= 0 && j < Nr; };
  auto vdesc = [&](int vidx) -> uint32_t { return GEN ? sDesc[vidx] : make_desc(4, 4, false, 0); };

  // ---- phase 1: V_r, V_z (+ descriptors) on the V region, T on the S region
  for (int idx = tid; idx < NV; idx += STAGE_THREADS) {
    const int vr = idx / VZ, vz = idx - vr * VZ;
    const int i = i0 - HVZ + vz, j = j0 - HV + vr;
    double a1 = 0.0, a3 = 0.0;
    uint32_t dsc = make_desc(ROW_NONE, ROW_NONE, false, 0);
    if (!GEN || inside(i, j)) {
      const long long o = (long long)j * g.P + i;
      a1 = __ldg(a.U + 1 * g.plane + o);
      a3 = __ldg(a.U + 3 * g.plane + o);
      if (GEN) dsc = __ldg(a.desc + o);
    }
    sVr[idx] = a1;
    sVz[idx] = a3;
    if (GEN) sDesc[idx] = dsc;
  }
  for (int idx = tid; idx < NS; idx += STAGE_THREADS) {
    const int sr = idx / SZ, sz = idx - sr * SZ;
    const int i = i0 - HS + sz, j = j0 - HS + sr;
    sT[idx] = (!GEN || inside(i, j)) ? __ldg(a.U + 4 * g.plane + (long long)j * g.P + i) : 0.0;
  }
  __syncthreads();

  // ---- phase 2: S and dilatation on the cross of the S region; f_sw on the tile
  for (int idx = tid; idx < NS; idx += STAGE_THREADS) {
    const int sr = idx / SZ, sz = idx - sr * SZ;
    const bool zarm = sr >= HS && sr < HS + TR;
    const bool rarm = sz >= HS && sz < HS + TZ;
    double S = 0.0, dil = 0.0;
    const int i = i0 - HS + sz, j = j0 - HS + sr;
    if ((zarm || rarm) && (!GEN || inside(i, j))) {
      const int vidx = (sr + HV - HS) * VZ + (sz + HVZ - HS);
      const uint32_t dsc = vdesc(vidx);
      const int zr = desc_blank(dsc) ? (int)ROW_NONE : desc_zrow(dsc);
      const int rw = desc_blank(dsc) ? (int)ROW_NONE : desc_rrow(dsc);
      const double xz = __ldg(a.dxidz + i), er = __ldg(a.detadr + j);
      const double dVrdz = d1<GEN>(zr, sVr + vidx, 1) * xz;
      const double dVzdz = d1<GEN>(zr, sVz + vidx, 1) * xz;
      const double dVrdr = d1<GEN>(rw, sVr + vidx, VZ) * er;
      const double dVzdr = d1<GEN>(rw, sVz + vidx, VZ) * er;
      const double vr = sVr[vidx];
      const double r = __ldg(a.rc + j);
      if (j == 0) dil = 2.0 * dVrdr + dVzdz;
      else dil = dVrdr + vr / r + dVzdz;
      const double S11 = dVrdr - (1.0 / 3.0) * dil;
      const double S13 = 0.5 * (dVrdz + dVzdr);
      const double S33 = dVzdz - (1.0 / 3.0) * dil;
      const double S22 = (j == 0) ? dVrdr - (1.0 / 3.0) * dil : vr / r - (1.0 / 3.0) * dil;
      S = sqrt(S11 * S11 + S13 * S13 + S22 * S22 + S13 * S13 + S33 * S33);
      if (zarm && rarm) {
        const double vort = fabs(dVrdz - dVzdr);
        const double Hm = (-1.0 * dil < 0.0) ? 0.0 : 1.0;
        const double eps = (double)1e-15f;  // single-precision literal of the reference (:202)
        sFsw[(sr - HS) * TZ + (sz - HS)] = Hm * (dil * dil) / (dil * dil + vort * vort + eps);
      }
    }
    sS[idx] = S;
    sD[idx] = dil;
  }
  __syncthreads();

  // ---- phases 3-4 per field: second derivatives on the arms, fourth derivatives at
  // the tile points (kept in registers: 2 points per thread)
  constexpr int PPT = (TZ * TR) / STAGE_THREADS;
  double d4z[3][PPT], d4r[3][PPT];
  const double* srcs[3] = {sS, sT, sD};
#pragma unroll
  for (int f = 0; f < 3; ++f) {
    const double* src = srcs[f];
    for (int idx = tid; idx < TR * DZ + DR * TZ; idx += STAGE_THREADS) {
      if (idx < TR * DZ) {
        const int r = idx / DZ, c = idx - r * DZ;  // point (i0 - HF + c, j0 + r)
        const int i = i0 - HF + c, j = j0 + r;
        double v = 0.0;
        if (!GEN || inside(i, j)) {
          const int sidx = (HS + r) * SZ + (HS - HF + c);
          const uint32_t dsc = vdesc((HV + r) * VZ + (HVZ - HF + c));
          const int zr = desc_blank(dsc) ? (int)ROW_NONE : desc_zrow(dsc);
          v = d2<GEN>(zr, src + sidx, 1);
        }
        sd2z[idx] = v;
      } else {
        const int k = idx - TR * DZ;
        const int r = k / TZ, c = k - r * TZ;      // point (i0 + c, j0 - HF + r)
        const int i = i0 + c, j = j0 - HF + r;
        double v = 0.0;
        if (!GEN || inside(i, j)) {
          const int sidx = (HS - HF + r) * SZ + (HS + c);
          const uint32_t dsc = vdesc((HV - HF + r) * VZ + (HVZ + c));
          const int rw = desc_blank(dsc) ? (int)ROW_NONE : desc_rrow(dsc);
          v = d2<GEN>(rw, src + sidx, SZ);
        }
        sd2r[k] = v;
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < PPT; ++q) {
      const int pidx = tid + q * STAGE_THREADS;
      const int r = pidx / TZ, c = pidx - r * TZ;
      const uint32_t dsc = vdesc((HV + r) * VZ + (HVZ + c));
      const int zr = desc_blank(dsc) ? (int)ROW_NONE : desc_zrow(dsc);
      const int rw = desc_blank(dsc) ? (int)ROW_NONE : desc_rrow(dsc);
      d4z[f][q] = d2<GEN>(zr, sd2z + r * DZ + HF + c, 1);
      d4r[f][q] = d2<GEN>(rw, sd2r + (HF + r) * TZ + c, TZ);
    }
    __syncthreads();
  }

  // ---- quantities to be filtered (ComputeTobeFilteredQuantities :204-215)
#pragma unroll
  for (int q = 0; q < PPT; ++q) {
    const int pidx = tid + q * STAGE_THREADS;
    const int r = pidx / TZ, c = pidx - r * TZ;
    const int i = i0 + c, j = j0 + r;
    if (GEN && !inside(i, j)) continue;
    const long long o = (long long)j * g.P + i;
    const double dz = __ldg(a.dz + i), dr = __ldg(a.dr + j);
    const double rho = __ldg(a.U + o);
    const double T = sT[(HS + r) * SZ + HS + c];
    const double fsw = sFsw[r * TZ + c];
    a.Q[o] = rho * fabs((d4z[0][q] * (dz * dz) + d4r[0][q] * (dr * dr)));
    a.Q[g.plane + o] = rho * fsw * fabs((d4z[2][q] * (dz * dz) + d4r[2][q] * (dr * dr)));
    a.Q[2 * g.plane + o] = rho / (a.c.gam * sqrt(T)) * fabs((d4z[1][q] * dz + d4r[1][q] * dr));
  }
}

// In-place z filter PerformTGfilter(q, 1, q) (ModShockCapturing.f90:63,69,75) as a
// recurrence along i: points left of i are already filtered when i is computed.
// Each thread owns a chunk of one row and starts WARM points early, taking the
// unfiltered values as the filtered ones left of its start; the recurrence is
// contractive (the dominant root of the interior filter's feedback part is about
// 0.47), so after WARM points that start-up difference is below 1e-20 relative.
constexpr int ZF_CHUNK = 128;
constexpr int ZF_WARM = 64;

__global__ void tgfilter_z_inplace_kernel(const Grid g, const uint32_t* __restrict__ desc,
                                          const double* __restrict__ q, double* __restrict__ out, int nfield) {
  const int nchunk = (g.Nz + ZF_CHUNK - 1) / ZF_CHUNK;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = (long long)nfield * g.Nr * nchunk;
  if (t >= total) return;
  const int c = (int)(t % nchunk);
  const int j = (int)((t / nchunk) % g.Nr);
  const int f = (int)(t / ((long long)nchunk * g.Nr));
  const double* x = q + (long long)f * g.plane + (long long)j * g.P;
  double* y = out + (long long)f * g.plane + (long long)j * g.P;
  const uint32_t* dr = desc + (long long)j * g.P;
  const int ib = c * ZF_CHUNK, ie = min(g.Nz, ib + ZF_CHUNK);
  const int is = max(0, ib - ZF_WARM);
  double ring[16];
  for (int i = is; i < ie; ++i) {
    const uint32_t dsc = __ldg(dr + i);
    const int row = row_of(dsc, 1);
    double v;
    if (row >= 9) {
      v = __ldg(x + i);
    } else {
      const int w0 = tg_w0(row), n = tg_len(row);
      double s = 0.0;
      for (int m = 0; m < n; ++m) {
        const int ii = i + w0 + m;
        double val;
        if (ii < 0 || ii >= g.Nz) val = 0.0;
        else if (ii < i && ii >= is) val = ring[ii & 15];
        else val = __ldg(x + ii);
        s = (m == 0) ? cTG[row][0] * val : s + cTG[row][m] * val;
      }
      v = s;
    }
    ring[i & 15] = v;
    if (i >= ib) y[i] = v;
  }
}

// r filter PerformTGfilter(q, 2, star) (:65, :71, :77), scaled by C*Re(*Pr) and the
// z ramp (:66, :72, :79, :85-88). Blanked points keep 0 (the output arrays start
// at 0 and are never written there).
__global__ void sensor_rfilter_kernel(const SensorArgs a) {
  const Grid g = a.g;
  const long long n = (long long)g.Nz * g.Nr;
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int j = (int)(p / g.Nz), i = (int)(p - (long long)j * g.Nz);
  const long long o = (long long)j * g.P + i;
  const uint32_t dsc = __ldg(a.desc + o);
  const int row = row_of(dsc, 2);
  const double scale[3] = {a.c.C_mu_Re, a.c.C_beta_Re, a.c.C_kappa_Re_Pr};
  const double ramp = __ldg(a.ramp + i);
#pragma unroll
  for (int f = 0; f < 3; ++f) {
    double v = 0.0;
    if (row < 9) {
      const double* src = a.Qz + (long long)f * g.plane;
      const int w0 = tg_w0(row), nn = tg_len(row);
      double s = cTG[row][0] * gval(src, g, i, j + w0);
      for (int m = 1; m < nn; ++m) s = s + cTG[row][m] * gval(src, g, i, j + w0 + m);
      v = s;
    }
    a.star[(long long)f * g.plane + o] = scale[f] * v * ramp;
  }
}

cudaError_t launch_sensor(const SensorArgs& a, cudaStream_t s) {
  const long long n = (long long)a.g.Nz * a.g.Nr;
  const int bs = 256;
  const int nb = (int)((n + bs - 1) / bs);
  if (a.ntiles_gen > 0)
    sensor_tile_kernel<SENS_HS_GEN, H_GEN, true>
        <<<a.ntiles_gen, STAGE_THREADS, SensSmem<SENS_HS_GEN, H_GEN>::bytes(true), s>>>(a, a.tiles_gen);
  if (a.ntiles_int > 0)
    sensor_tile_kernel<SENS_HS_INT, H_INT, false>
        <<<a.ntiles_int, STAGE_THREADS, SensSmem<SENS_HS_INT, H_INT>::bytes(false), s>>>(a, a.tiles_int);
  cudaError_t e = launch_tgfilter_z_inplace(a.g, a.desc, a.Q, a.Qz, 3, s);
  if (e != cudaSuccess) return e;
  sensor_rfilter_kernel<<<nb, bs, 0, s>>>(a);
  return cudaGetLastError();
}

// Row-staged version of the same recurrence: one CTA per (row, field); the row of
// unfiltered values and the z row codes sit in shared memory, each thread owns a
// chunk of ZR_L points (odd, so lanes read shared memory without bank conflicts) and
// keeps the last 10 filtered values in registers. Rows up to ZR_MAXNZ points.
constexpr int ZR_L = 33;
constexpr int ZR_W = 48;
constexpr int ZR_MAXNZ = 12288;

// One output of the recurrence for TG row ROW at point i. p[k] = filtered value at
// i-k (or the unfiltered value / 0 left of the chunk's start), xs = unfiltered row.
template <int ROW>
__device__ __forceinline__ double zr_apply(const double (&p)[11], const double* __restrict__ xs, int i, int Nz) {
  constexpr int W0 = ROW < 4 ? -ROW : (ROW == 4 ? -4 : -2 - ROW);
  constexpr int N = ROW == 4 ? 9 : 11;
  double s = 0.0;
#pragma unroll
  for (int m = 0; m < N; ++m) {
    const int o = W0 + m;
    double v;
    if (o < 0) v = p[o < 0 ? -o : 0];
    else v = (i + o < Nz) ? xs[i + o] : 0.0;
    s = (m == 0) ? cTG[ROW][0] * v : s + cTG[ROW][m] * v;
  }
  return s;
}

__global__ void tgfilter_z_rows_kernel(const Grid g, const uint32_t* __restrict__ desc,
                                       const double* __restrict__ q, double* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char zr_smem[];
  const int Nz = g.Nz;
  double* xs = reinterpret_cast<double*>(zr_smem);
  double* ys = xs + Nz;
  unsigned char* rs = reinterpret_cast<unsigned char*>(ys + Nz);
  const int j = blockIdx.x, f = blockIdx.y;
  const double* x = q + (long long)f * g.plane + (long long)j * g.P;
  double* y = out + (long long)f * g.plane + (long long)j * g.P;
  const uint32_t* dr = desc + (long long)j * g.P;
  for (int i = threadIdx.x; i < Nz; i += blockDim.x) {
    xs[i] = __ldg(x + i);
    rs[i] = (unsigned char)row_of(__ldg(dr + i), 1);
  }
  __syncthreads();
  const int nchunk = (Nz + ZR_L - 1) / ZR_L;
  for (int c = threadIdx.x; c < nchunk; c += blockDim.x) {
    const int ib = c * ZR_L, ie = min(Nz, ib + ZR_L), is = max(0, ib - ZR_W);
    double p[11];
    p[0] = 0.0;
#pragma unroll
    for (int k = 1; k <= 10; ++k) p[k] = (is - k >= 0) ? xs[is - k] : 0.0;
    for (int i = is; i < ie; ++i) {
      double v;
      switch (rs[i]) {
        case 4: v = zr_apply<4>(p, xs, i, Nz); break;
        case 0: v = zr_apply<0>(p, xs, i, Nz); break;
        case 1: v = zr_apply<1>(p, xs, i, Nz); break;
        case 2: v = zr_apply<2>(p, xs, i, Nz); break;
        case 3: v = zr_apply<3>(p, xs, i, Nz); break;
        case 5: v = zr_apply<5>(p, xs, i, Nz); break;
        case 6: v = zr_apply<6>(p, xs, i, Nz); break;
        case 7: v = zr_apply<7>(p, xs, i, Nz); break;
        case 8: v = zr_apply<8>(p, xs, i, Nz); break;
        default: v = xs[i]; break;  // blanked / no row: left unchanged in place
      }
#pragma unroll
      for (int k = 10; k >= 2; --k) p[k] = p[k - 1];
      p[1] = v;
      if (i >= ib) ys[i] = v;
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < Nz; i += blockDim.x) y[i] = ys[i];
}

cudaError_t launch_tgfilter_z_inplace(const Grid& g, const uint32_t* desc, const double* q, double* out, int nfield,
                                      cudaStream_t s) {
  if (g.Nz <= ZR_MAXNZ) {
    const size_t sm = (size_t)g.Nz * (2 * sizeof(double) + 1);
    const int nchunk = (g.Nz + ZR_L - 1) / ZR_L;
    const int bs = std::min(1024, (nchunk + 31) / 32 * 32);
    tgfilter_z_rows_kernel<<<dim3(g.Nr, nfield), bs, sm, s>>>(g, desc, q, out);
    return cudaGetLastError();
  }
  const int nchunk = (g.Nz + ZF_CHUNK - 1) / ZF_CHUNK;
  const long long total = (long long)nfield * g.Nr * nchunk;
  const int bs = 128;
  tgfilter_z_inplace_kernel<<<(int)((total + bs - 1) / bs), bs, 0, s>>>(g, desc, q, out, nfield);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Unit entry points.
// ---------------------------------------------------------------------------
// order 1: Compute1stDerivative; order 2: Compute2ndDerivative (first != null);
// order 3: Compute2ndDerivativeComputational.
__global__ void deriv_kernel(const Grid g, const uint32_t* __restrict__ desc, const double* __restrict__ var,
                             const double* __restrict__ first, const double* __restrict__ met,
                             const double* __restrict__ met2, int dirn, int order, double* __restrict__ out) {
  const long long n = (long long)g.Nz * g.Nr;
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int j = (int)(p / g.Nz), i = (int)(p - (long long)j * g.Nz);
  const long long o = (long long)j * g.P + i;
  const int row = row_of(__ldg(desc + o), dirn);
  const int k = dirn == 1 ? i : j;
  double v;
  if (order == 1) {
    v = gstencil6(cSBP1, row, var, g, i, j, dirn) * __ldg(met + k);
  } else if (order == 2) {
    const double m = __ldg(met + k);
    v = gstencil6(cSBP2, row, var, g, i, j, dirn) * (m * m) + __ldg(first + o) * __ldg(met2 + k);
  } else {
    v = gstencil6(cSBP2, row, var, g, i, j, dirn);
  }
  out[o] = v;
}

cudaError_t launch_deriv(const Grid& g, const uint32_t* desc, const double* var, const double* first,
                         const double* met, const double* met2, int dirn, int order, double* out, cudaStream_t s) {
  const long long n = (long long)g.Nz * g.Nr;
  deriv_kernel<<<(int)((n + 255) / 256), 256, 0, s>>>(g, desc, var, first, met, met2, dirn, order, out);
  return cudaGetLastError();
}

// Out-of-place PerformTGfilter; out keeps its value where no row applies.
__global__ void tgfilter_kernel(const Grid g, const uint32_t* __restrict__ desc, const double* __restrict__ var,
                                int dirn, double* __restrict__ out) {
  const long long n = (long long)g.Nz * g.Nr;
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int j = (int)(p / g.Nz), i = (int)(p - (long long)j * g.Nz);
  const long long o = (long long)j * g.P + i;
  const int row = row_of(__ldg(desc + o), dirn);
  if (row >= 9) return;
  const int w0 = tg_w0(row), nn = tg_len(row);
  const int di = dirn == 1 ? 1 : 0, dj = dirn == 1 ? 0 : 1;
  double s = cTG[row][0] * gval(var, g, i + w0 * di, j + w0 * dj);
  for (int m = 1; m < nn; ++m) s = s + cTG[row][m] * gval(var, g, i + (w0 + m) * di, j + (w0 + m) * dj);
  out[o] = s;
}

cudaError_t launch_tgfilter(const Grid& g, const uint32_t* desc, const double* var, int dirn, double* out,
                            cudaStream_t s) {
  const long long n = (long long)g.Nz * g.Nr;
  tgfilter_kernel<<<(int)((n + 255) / 256), 256, 0, s>>>(g, desc, var, dirn, out);
  return cudaGetLastError();
}

}  // namespace axj

namespace axj {

// Opt-in shared-memory sizes; called once per handle at creation (outside any
// stream capture).
cudaError_t init_kernel_attributes() {
  cudaError_t e = cudaFuncSetAttribute(stage_kernel<H_GEN, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)StageSmem<H_GEN>::bytes(true));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(stage_kernel<H_INT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)StageSmem<H_INT>::bytes(false));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(sensor_tile_kernel<SENS_HS_GEN, H_GEN, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)SensSmem<SENS_HS_GEN, H_GEN>::bytes(true));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(sensor_tile_kernel<SENS_HS_INT, H_INT, false>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SensSmem<SENS_HS_INT, H_INT>::bytes(false));
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(tgfilter_z_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)((size_t)ZR_MAXNZ * (2 * sizeof(double) + 1)));
}

}  // namespace axj
