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
#include <type_traits>

#include "axj_kernels.cuh"
#include "axj_point.cuh"
#include "axj_pow.cuh"

namespace axj {

__constant__ double cSBP1[9][6];
__constant__ double cSBP2[9][6];
__constant__ double cTG[9][11];
__constant__ float cSBP1f[9][6];
__constant__ float cSBP2f[9][6];
__constant__ PatchDev cPatch[MAX_PATCHES];
// SBP2 centred row composed with itself: the 9-point fourth-difference row (offsets -4..4)
__constant__ double cC9[9];
__constant__ float cC9f[9];
// tables of the FP64 power mu = T**0.666 (axj_pow.cuh); read through the L1 cache, since
// the points of a warp index them by their own T
__device__ double gPowTab[POW_TAB];

// mu = T**0.666 of the stage input: the table-driven FP64 power, or (FP32 stencils)
// exp2f / log2f
template <typename R>
__device__ __forceinline__ R mu_k(R T) {
  if constexpr (std::is_same<R, double>::value) return pow0666(T, gPowTab);
  else return mu_of_T<float>(T);
}

void upload_tables(const double sbp1[9][6], const double sbp2[9][6], const double tg[9][11],
                   const PatchDev* patches, int npatch, cudaStream_t s) {
  cudaMemcpyToSymbolAsync(cSBP1, sbp1, sizeof(double) * 54, 0, cudaMemcpyHostToDevice, s);
  cudaMemcpyToSymbolAsync(cSBP2, sbp2, sizeof(double) * 54, 0, cudaMemcpyHostToDevice, s);
  cudaMemcpyToSymbolAsync(cTG, tg, sizeof(double) * 99, 0, cudaMemcpyHostToDevice, s);
  // FP32 copies of the SBP tables for the mixed-precision stencils (static: the
  // asynchronous copies read them after this function returns)
  static float f1[9][6], f2[9][6];
  for (int r = 0; r < 9; ++r)
    for (int m = 0; m < 6; ++m) {
      f1[r][m] = (float)sbp1[r][m];
      f2[r][m] = (float)sbp2[r][m];
    }
  cudaMemcpyToSymbolAsync(cSBP1f, f1, sizeof(float) * 54, 0, cudaMemcpyHostToDevice, s);
  cudaMemcpyToSymbolAsync(cSBP2f, f2, sizeof(float) * 54, 0, cudaMemcpyHostToDevice, s);
  if (npatch > 0) cudaMemcpyToSymbolAsync(cPatch, patches, sizeof(PatchDev) * npatch, 0, cudaMemcpyHostToDevice, s);
  static double c9[9];
  static float c9f[9];
  for (int k = 0; k < 9; ++k) c9[k] = 0.0;
  for (int a = 0; a < 5; ++a)
    for (int b = 0; b < 5; ++b) c9[a + b] += sbp2[4][a] * sbp2[4][b];
  for (int k = 0; k < 9; ++k) c9f[k] = (float)c9[k];
  cudaMemcpyToSymbolAsync(cC9, c9, sizeof(double) * 9, 0, cudaMemcpyHostToDevice, s);
  cudaMemcpyToSymbolAsync(cC9f, c9f, sizeof(float) * 9, 0, cudaMemcpyHostToDevice, s);
  static double pw[POW_TAB];
  static bool pw_done = false;
  if (!pw_done) {
    pow0666_fill(pw);
    pw_done = true;
  }
  cudaMemcpyToSymbolAsync(gPowTab, pw, sizeof pw, 0, cudaMemcpyHostToDevice, s);
}

// Round-to-nearest arithmetic that the compiler may not contract into an FMA; used
// where the reference's two-step rounding (k = delt*rhs, then the RK sums) is kept.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }

// SBP / TG tables in the arithmetic type of a stencil.
template <typename R, int TAB>
__device__ __forceinline__ R tabv(int row, int m);
template <> __device__ __forceinline__ double tabv<double, 1>(int row, int m) { return cSBP1[row][m]; }
template <> __device__ __forceinline__ double tabv<double, 2>(int row, int m) { return cSBP2[row][m]; }
template <> __device__ __forceinline__ float tabv<float, 1>(int row, int m) { return cSBP1f[row][m]; }
template <> __device__ __forceinline__ float tabv<float, 2>(int row, int m) { return cSBP2f[row][m]; }

// Dot product of SBP row `row` of table TAB with N values at v (stride in elements),
// evaluated in type R. The sequence starts from the first product, as DOT_PRODUCT's
// 0 + a1*b1 does.
template <typename R, int TAB, int N, typename S>
__device__ __forceinline__ R dotc(int row, const S* __restrict__ v, int stride) {
  R s = tabv<R, TAB>(row, 0) * R(v[0]);
#pragma unroll
  for (int m = 1; m < N; ++m) s = s + tabv<R, TAB>(row, m) * R(v[m * stride]);
  return s;
}

// DOT_PRODUCT of the centred SBP1 row (1/12, -2/3, 0, 2/3, -1/12; ModOperator.f90) with the
// window around p, left to right. Its middle weight is exactly zero, so that term adds
// nothing to the running sum and is left out (the same result, one product fewer).
template <typename R, typename S>
__device__ __forceinline__ R dot_c1(const S* p, int stride) {
  R s = tabv<R, 1>(4, 0) * R(p[-2 * stride]);
  s = s + tabv<R, 1>(4, 1) * R(p[-stride]);
  s = s + tabv<R, 1>(4, 3) * R(p[stride]);
  s = s + tabv<R, 1>(4, 4) * R(p[2 * stride]);
  return s;
}

// Derivative stencil of table TAB with row code `row` (0..8; 9 = none) at p (pointer
// to the point's own value), stride 1 along z or the row length along r. Interior
// tiles (GEN = false) always use the centred row.
template <typename R, int TAB, bool GEN, typename S>
__device__ __forceinline__ R dst(int row, const S* p, int stride) {
  if (!GEN || row == 4) {
    if (TAB == 1) return dot_c1<R>(p, stride);
    return dotc<R, TAB, 5>(4, p - 2 * stride, stride);
  }
  if (row >= 9) return R(0);
  return dotc<R, TAB, 6>(row, p + sbp_w0(row) * stride, stride);
}

// dp/dz, dp/dr: the reference differentiates pvec = rhovec*Tvec, so every tap is a product.
template <typename R, bool GEN, typename S>
__device__ __forceinline__ R dst_p(int row, const S* rho, const S* T, int stride) {
  int w0, n, rw;
  if (!GEN || row == 4) { w0 = -2; n = 5; rw = 4; }
  else if (row >= 9) return R(0);
  else { w0 = sbp_w0(row); n = 6; rw = row; }
  R s = tabv<R, 1>(rw, 0) * (R(rho[w0 * stride]) * R(T[w0 * stride]));
#pragma unroll
  for (int m = 1; m < 6; ++m) {
    if (m >= n) continue;
    if (rw == 4 && m == 2) continue;  // the centred row's exactly zero middle weight
    s = s + tabv<R, 1>(rw, m) * (R(rho[(w0 + m) * stride]) * R(T[(w0 + m) * stride]));
  }
  return s;
}

// 9-point fourth difference cC9 centred at p (stride in elements), left to right.
template <typename R, typename S>
__device__ __forceinline__ R c9dot(const S* p, int stride) {
  const R* c = std::is_same<R, float>::value ? reinterpret_cast<const R*>(cC9f) : reinterpret_cast<const R*>(cC9);
  R s = c[0] * R(p[-4 * stride]);
#pragma unroll
  for (int m = 1; m < 9; ++m) s = s + c[m] * R(p[(m - 4) * stride]);
  return s;
}

// axis_conditions (ModAxis.f90:14-16): f(1) = -DOT_PRODUCT(SBP1(0,1:5), f(2:6)) / SBP1(0,0),
// with p pointing at row 2 of a column (stride = row length).
template <typename S>
__device__ __forceinline__ double axis_extrap(const S* p, int stride) {
  double s = cSBP1[0][1] * double(p[0]);
#pragma unroll
  for (int m = 1; m < 5; ++m) s = s + cSBP1[0][m + 1] * double(p[m * stride]);
  return -1.0 * s / cSBP1[0][0];
}

// ---------------------------------------------------------------------------
// Fused RK-stage kernel.
// ---------------------------------------------------------------------------
// ---- TMA / mbarrier helpers (inline PTX, sm_90+ forms valid on sm_100a) ----------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Tries of a bounded wait before it gives up (about a quarter of a second at the default;
// axj_set_wait_limit lowers it to exercise the timeout path).
constexpr int kWaitTriesDefault = 1 << 20;
__constant__ int c_wait_tries = kWaitTriesDefault;
// Bounded wait: gives up after c_wait_tries polls instead of spinning forever.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  const int tries = c_wait_tries;
  for (int it = 0; it < tries; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if (it > 32) __nanosleep(256);
  }
  return false;
}
// The error path after a bounded wait gave up: wait again, bounded by the default limit,
// for the transfers of that barrier phase still in flight, so that none of them lands in
// the shared memory of a CTA that has exited.
__device__ __forceinline__ void mbar_drain(uint64_t* bar, uint32_t parity) {
  for (int it = 0; it < kWaitTriesDefault; ++it) {
    if (mbar_try_wait(bar, parity)) return;
    if (it > 32) __nanosleep(256);
  }
}
// 3-D tiled TMA load (x = z index, y = r index, z = field plane) into shared memory;
// out-of-range elements are filled with zeros.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// Bulk (non-tensor) global -> shared copy completing on an mbarrier; both addresses
// 16-byte aligned, size a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// Prefetch of a tensor box into L2 (no shared memory, no completion to wait for).
__device__ __forceinline__ void tma_prefetch_3d(const CUtensorMap* map, int x, int y, int z) {
  asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(x), "r"(y), "r"(z)
               : "memory");
}

__host__ __device__ constexpr size_t align128(size_t b) { return (b + 127) / 128 * 128; }

// z halo of a box in elements, rounded up so the box's x coordinate starts on a
// 16-byte boundary (TMA requirement): even for doubles, a multiple of 4 for floats.
__host__ __device__ constexpr int hz_t(int h, int esize) { return (h + 16 / esize - 1) / (16 / esize) * (16 / esize); }

// HZ follows the arithmetic type: the mixed path rounds to 4 elements in every stage
// (valid for its double stage-1 input too), so one coefficient-box map serves all stages.
// CM, the content of the coefficient box (CM_FILT, CM_LRN, CM_PRE: axj_kernels.cuh).
// Half tiles with FP32 stencils (the mixed path) read pv_old and the running sum from
// global memory (L2-prefetched at the tile start) instead of staging them: that leaves them
// about 25 KB of shared memory, and at 80 registers six CTAs share an SM. The FP64 half
// tiles stage them and run four CTAs per SM (at 80 registers their per-point code spills).
template <typename R, int TRT>
__host__ __device__ constexpr bool rk_global() { return TRT < TR && sizeof(R) == 4; }

// TRT: rows of the tile (TR; interior tiles can also run as two halves of TR / 2 rows,
// which need about half the shared memory and so let four to six CTAs share an SM).
template <int H, typename SIN, typename R, int CM = CM_FILT, int TRT = TR>
struct StageSmem {
  static constexpr int HZ = hz_t(H, (int)sizeof(R));
  static constexpr int RZ = TZ + 2 * HZ;
  static constexpr int RR = TRT + 2 * H;
  static constexpr int NPT = RZ * RR;
  static constexpr int NTP = TZ * TRT;
  // r reach of the truncated-Gaussian filter rows: 4 for the centred row, 10 for the
  // 11-point boundary rows (ModTGfilter.f90:31-44)
  static constexpr int HT = CM != CM_FILT ? 0 : ((H == H_INT) ? 4 : 10);
  static constexpr int RQ = RR + 2 * HT;  // rows of the z-filtered coefficient box
  // byte offsets: state box [5][RR][RZ] of the stage-input type; coefficient box
  // [3][RQ][RZ] (doubles) holding the z-filtered quantities on arrival and mu_eff,
  // beta*, kappa_eff (rows HT..HT+RR) after the r filter (without shock capturing plane
  // 0 rows HT.. hold mu); plain mu on the tile [TR][TZ]; interior tiles only: pv_old
  // tile [5][TR][TZ] and running-sum tile [5][TR][TZ] (general tiles read them from
  // global memory, which keeps two of their CTAs on an SM); dV/dz [2][RR][TZ] (stencil
  // type); general tiles only: descriptors [RR][RZ]
  static constexpr size_t oU = 0;
  static constexpr size_t oQ = align128(oU + sizeof(SIN) * 5 * NPT);
  static constexpr size_t oMu0 = align128(oQ + sizeof(double) * 3 * RQ * RZ);
  // (CM_PRE reads beta from the coefficient box and needs no plain mu)
  static constexpr size_t oP0 = align128(oMu0 + (CM == CM_PRE ? 0 : sizeof(double) * NTP));
  static constexpr size_t oPA = align128(oP0 + sizeof(double) * 5 * NTP);
  __host__ __device__ static constexpr size_t oDz(bool gen) {
    return (gen || rk_global<R, TRT>()) ? oP0 : align128(oPA + sizeof(double) * 5 * NTP);
  }
  __host__ __device__ static constexpr size_t oDesc(bool gen) {
    return align128(oDz(gen) + sizeof(double) * 2 * RR * TZ);
  }
  // 1-D metrics and coordinates of the tile: dxidz, ddxidxidz, z on its columns,
  // detadr, ddetadetadr, r, 1/r on its rows
  __host__ __device__ static constexpr size_t oMet(bool gen) {
    return align128(oDesc(gen) + (gen ? sizeof(uint32_t) * NPT : 0));
  }
  static constexpr int NMET = 3 * TZ + 4 * TRT;
  __host__ __device__ static constexpr size_t bytes(bool gen) { return align128(oMet(gen) + sizeof(double) * NMET); }
  static constexpr uint32_t state_bytes = sizeof(SIN) * 5 * NPT;
  static constexpr uint32_t q_bytes = sizeof(double) * 3 * RQ * RZ;
  static constexpr uint32_t tile_bytes = sizeof(double) * 5 * NTP;
  static constexpr int NPER = (NPT + STAGE_THREADS - 1) / STAGE_THREADS;
};


// Fused RK stage. SIN: storage type of the stage input (double, or float for the
// mixed path's intermediate stages); R: arithmetic type of the stencils and, in
// interior tiles, of the pointwise terms. General tiles (closure rows, faces, the axis
// row) evaluate the pointwise terms, face penalties and sponges in double.
// Shared-memory buffers of one stage tile (layout StageSmem: state box, coefficient box,
// plain mu, pv_old and running-sum tiles, dV/dz, descriptors, metrics).
template <typename SIN, typename R>
struct StagePtrs {
  SIN* sU;
  double* sQ;
  double* sMu0;
  double* sP0;
  double* sPA;
  R* sDz;
  const uint32_t* sDesc;
  const double* sMet;
};

// Phases 2-3 of one stage tile (i0, j0; nrow rows of it are owned) whose boxes have
// arrived in shared memory, with NT threads: mu and the coefficients on the cross, dV/dz on
// the tile columns, then the points. The RK operand tiles of interior tiles complete on
// barRK (parity rk_parity). Returns false if that bounded wait gave up (the flag is set and
// the transfers in flight have landed).
template <int H, bool GEN, typename SIN, typename R, int CM, int NT, int TRT>
__device__ __forceinline__ bool stage_compute(const StageArgs& a, int i0, int j0, int nrow,
                                              const StagePtrs<SIN, R>& sp, uint64_t* barRK, uint32_t rk_parity) {
  using SM = StageSmem<H, SIN, R, CM, TRT>;
  using RP = typename std::conditional<GEN, double, R>::type;
  constexpr int HZ = SM::HZ, RZ = SM::RZ, RR = SM::RR, NPT = SM::NPT, NTP = SM::NTP, HT = SM::HT, RQ = SM::RQ;
  constexpr int NPER = (NPT + NT - 1) / NT;
  const SIN* sU = sp.sU;
  double* sQ = sp.sQ;
  double* sMu = sQ + HT * RZ;                                      // [RR][RZ], row stride RZ
  double* sBe = sQ + RQ * RZ + HT * RZ;
  double* sKa = a.c.shock_capturing ? sQ + 2 * RQ * RZ + HT * RZ : sMu;
  double* sMu0 = sp.sMu0;
  const double* sP0 = sp.sP0;
  const double* sPA = sp.sPA;
  R* sDz = sp.sDz;
  const uint32_t* sDesc = sp.sDesc;
  const double* sMet = sp.sMet;
  const int tid = threadIdx.x;
  const int Nz = a.g.Nz, Nr = a.g.Nr;
  const long long P = a.g.P, PL = a.g.plane;
  const bool sc = a.c.shock_capturing != 0;
  // RK operands from global memory (general tiles, FP32 half tiles) or staged by TMA
  constexpr bool RKG = GEN || rk_global<R, TRT>();
  const bool needU0 = !RKG && (a.stage == 2 || a.stage == 3);
  const bool needA = !RKG && (a.stage == 3 || a.stage == 4);
  // mu = T**0.666 (AssignValues) on the cross of the region (CM_PRE: the coefficient box
  // already holds mu_eff, beta and kappa_eff). With shock capturing the
  // coefficient box holds the z-filtered quantities; the r filter PerformTGfilter(q, 2,
  // star) (ModShockCapturing.f90:65,71,77), the C*Re(*Pr) scaling and the z ramp
  // (:66-92) give mu*, beta*, kappa*, and mu_eff = mu + mu*, kappa_eff = mu + kappa*
  // (UpdateTransportCoeffs :248-251). The results overwrite the box only after every
  // thread has read its filter windows. Zero-filled points outside the block give
  // mu = 0, as the never-written halo does; blanked points keep mu* = 0.
  if (CM != CM_PRE) {
    double vmu[NPER], vbe[NPER], vka[NPER];
#pragma unroll
    for (int k = 0; k < NPER; ++k) {
      const int idx = tid + k * NT;
      vmu[k] = vbe[k] = vka[k] = 0.0;
      if (idx >= NPT) continue;
      const int rr = idx / RZ, rz = idx - rr * RZ;
      const bool cross = (rr >= H && rr < H + TRT && rz >= HZ - H && rz < HZ + TZ + H) || (rz >= HZ && rz < HZ + TZ);
      if (!cross) continue;
      const double mu = double(mu_k<R>(R(sU[4 * NPT + idx])));
      vmu[k] = mu;
      if (rr >= H && rr < H + TRT && rz >= HZ && rz < HZ + TZ) sMu0[(rr - H) * TZ + (rz - HZ)] = mu;
      if (sc) {
        int rw = 4;
        if (GEN) {
          const uint32_t dsc = sDesc[idx];
          rw = desc_blank(dsc) ? (int)ROW_NONE : desc_rrow(dsc);
          const int i = i0 - HZ + rz, j = j0 - H + rr;
          if (!(i >= 0 && i < Nz && j >= 0 && j < Nr)) rw = (int)ROW_NONE;
        }
        double f[3] = {0.0, 0.0, 0.0};
        if (CM == CM_LRN) {
          // final coefficients (ramp applied), zero at blanked points as the filter gives
          if (rw < 9) {
#pragma unroll
            for (int q = 0; q < 3; ++q) f[q] = sQ[q * RQ * RZ + idx];
          }
          vmu[k] = mu + f[0];
          vbe[k] = f[1];
          vka[k] = mu + f[2];
          continue;
        }
        if (rw < 9) {
          const int w0 = GEN ? tg_w0(rw) : -4;
          const int n = GEN ? tg_len(rw) : 9;
          const int rowc = GEN ? rw : 4;
#pragma unroll
          for (int q = 0; q < 3; ++q) {
            const double* col = sQ + q * RQ * RZ + (rr + HT + w0) * RZ + rz;
            double s = cTG[rowc][0] * col[0];
            for (int m = 1; m < n; ++m) s = s + cTG[rowc][m] * col[m * RZ];
            f[q] = s;
          }
        }
        const int i = i0 - HZ + rz;
        const double ramp = (i >= 0 && i < Nz) ? __ldg(a.ramp + i) : 0.0;
        vmu[k] = mu + a.c.C_mu_Re * f[0] * ramp;
        vbe[k] = a.c.C_beta_Re * f[1] * ramp;
        vka[k] = mu + a.c.C_kappa_Re_Pr * f[2] * ramp;
      }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NPER; ++k) {
      const int idx = tid + k * NT;
      if (idx >= NPT) continue;
      const int rr = idx / RZ, rz = idx - rr * RZ;
      const bool cross = (rr >= H && rr < H + TRT && rz >= HZ - H && rz < HZ + TZ + H) || (rz >= HZ && rz < HZ + TZ);
      if (!cross) continue;
      sMu[idx] = vmu[k];
      if (sc) {
        sBe[idx] = vbe[k];
        sKa[idx] = vka[k];
      }
    }
  }
  __syncthreads();

  // ---- phase 2: dVr/dz and dVz/dz on the tile columns, all region rows (needed by
  // the mixed derivatives d/dr(dV/dz), ModRHS.f90:132-133)
  for (int idx = tid; idx < RR * TZ; idx += NT) {
    const int rr = idx / TZ, c = idx - rr * TZ;
    const int i = i0 + c, j = j0 - H + rr;
    R dvr = R(0), dvz = R(0);
    const bool in = (!GEN) || (i < Nz && j >= 0 && j < Nr);
    if (in) {
      const int sidx = rr * RZ + HZ + c;
      int row = 4;
      if (GEN) {
        const uint32_t dsc = sDesc[sidx];
        row = desc_blank(dsc) ? (int)ROW_NONE : desc_zrow(dsc);
      }
      const R m = R(sMet[c]);
      dvr = dst<R, 1, GEN>(row, sU + 1 * NPT + sidx, 1) * m;
      dvz = dst<R, 1, GEN>(row, sU + 3 * NPT + sidx, 1) * m;
    }
    sDz[idx] = dvr;
    sDz[RR * TZ + idx] = dvz;
  }
  __syncthreads();

  // ---- phase 3: one point per thread per pass
  if (needU0 || needA) {
    if (!__syncthreads_and(mbar_wait_bounded(barRK, rk_parity))) {
      if (tid == 0) atomicOr(a.flags, 4);
      mbar_drain(barRK, rk_parity);
      return false;
    }
  }
  const double dtv = a.stage > 0 ? *a.dt : 0.0;
  // cos(omega t_s) at this stage's time (harmonic forcing)
  const double cwt = a.c.control_forcing == 2 ? a.harm[a.stage] : 0.0;
  for (int pidx = tid; pidx < TZ * TRT; pidx += NT) {
    const int r = pidx / TZ, c = pidx - r * TZ;
    const int i = i0 + c, j = j0 + r;
    if (GEN && (i >= Nz || j >= Nr || r >= nrow)) continue;
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
    const double xzd = sMet[c], erd = sMet[3 * TZ + r];
    const R xz = R(xzd), xzz = R(sMet[TZ + c]);
    const R er = R(erd), err = R(sMet[3 * TZ + TRT + r]);
    const SIN* pR = sU + 0 * NPT + sidx;
    const SIN* pVr = sU + 1 * NPT + sidx;
    const SIN* pVt = sU + 2 * NPT + sidx;
    const SIN* pVz = sU + 3 * NPT + sidx;
    const SIN* pT = sU + 4 * NPT + sidx;
    const double* pMu = sMu + sidx;
    const double* pKa = sKa + sidx;
    const int dzi = rr * TZ + c;

    DerivT<R> dr;
    // first derivatives (Compute1stDerivative: stencil, then * metric)
    dr.drhodz = dst<R, 1, GEN>(zr, pR, 1) * xz;
    dr.dVrdz = sDz[dzi];
    dr.dVtdz = dst<R, 1, GEN>(zr, pVt, 1) * xz;
    dr.dVzdz = sDz[RR * TZ + dzi];
    dr.dTdz = dst<R, 1, GEN>(zr, pT, 1) * xz;
    dr.dpdz = dst_p<R, GEN>(zr, pR, pT, 1) * xz;
    dr.drhodr = dst<R, 1, GEN>(rw, pR, RZ) * er;
    dr.dVrdr = dst<R, 1, GEN>(rw, pVr, RZ) * er;
    dr.dVtdr = dst<R, 1, GEN>(rw, pVt, RZ) * er;
    dr.dVzdr = dst<R, 1, GEN>(rw, pVz, RZ) * er;
    dr.dTdr = dst<R, 1, GEN>(rw, pT, RZ) * er;
    dr.dpdr = dst_p<R, GEN>(rw, pR, pT, RZ) * er;
    // second derivatives (Compute2ndDerivative: out*metric**2 + f'*metric')
    dr.d2Vrdz2 = dst<R, 2, GEN>(zr, pVr, 1) * (xz * xz) + dr.dVrdz * xzz;
    dr.d2Vtdz2 = dst<R, 2, GEN>(zr, pVt, 1) * (xz * xz) + dr.dVtdz * xzz;
    dr.d2Vzdz2 = dst<R, 2, GEN>(zr, pVz, 1) * (xz * xz) + dr.dVzdz * xzz;
    dr.d2Tdz2 = dst<R, 2, GEN>(zr, pT, 1) * (xz * xz) + dr.dTdz * xzz;
    dr.d2Vrdr2 = dst<R, 2, GEN>(rw, pVr, RZ) * (er * er) + dr.dVrdr * err;
    dr.d2Vtdr2 = dst<R, 2, GEN>(rw, pVt, RZ) * (er * er) + dr.dVtdr * err;
    dr.d2Vzdr2 = dst<R, 2, GEN>(rw, pVz, RZ) * (er * er) + dr.dVzdr * err;
    dr.d2Tdr2 = dst<R, 2, GEN>(rw, pT, RZ) * (er * er) + dr.dTdr * err;
    dr.dmudz = dst<R, 1, GEN>(zr, pMu, 1) * xz;
    dr.dkappadz = sc ? dst<R, 1, GEN>(zr, pKa, 1) * xz : dr.dmudz;
    dr.dmudr = dst<R, 1, GEN>(rw, pMu, RZ) * er;
    dr.dkappadr = sc ? dst<R, 1, GEN>(rw, pKa, RZ) * er : dr.dmudr;
    dr.d2Vrdzdr = dst<R, 1, GEN>(rw, sDz + dzi, TZ) * er;
    dr.d2Vzdzdr = dst<R, 1, GEN>(rw, sDz + RR * TZ + dzi, TZ) * er;

    const double pv[5] = {double(*pR), double(*pVr), double(*pVt), double(*pVz), double(*pT)};
    PrimT<RP> q;
    q.rho = RP(*pR); q.Vr = RP(*pVr); q.Vt = RP(*pVt); q.Vz = RP(*pVz); q.T = RP(*pT);
    q.mu = RP(*pMu);
    q.kappa = RP(*pKa);
    const long long go = (long long)j * P + i;
    {
      // lambda = beta - 2/3 mu with beta = 0.6 mu (+ betastar), ModAssign.f90:22-23,
      // ModShockCapturing.f90:248-251
      double beta;
      if (CM == CM_PRE) {
        beta = sBe[sidx];
      } else {
        const double mu0 = sMu0[r * TZ + c];
        beta = (3.0 / 5.0) * mu0;
        if (sc) beta = beta + sBe[sidx];
      }
      q.lambda = RP(beta - (2.0 / 3.0) * double(*pMu));
    }
    const DerivT<RP> d = convert<RP>(dr);
    const double rloc = sMet[3 * TZ + 2 * TRT + r], zloc = sMet[2 * TZ + c];
    const bool j1 = (j == 0);
    double rhs[5] = {-0.0, -0.0, -0.0, -0.0, -0.0};
    if (!j1) {
      RP rp[5];
      const RhsConst<RP> kc = rhs_const<RP>(a.c);
      const RP onebyr = RP(sMet[3 * TZ + 3 * TRT + r]);
      const RP inv_rho = RP(1.0) / q.rho;
      rhs_inviscid<RP>(q, d, onebyr, inv_rho, kc, rp);
      if (a.c.do_viscous) rhs_viscous<RP>(q, d, onebyr, inv_rho, kc, sc, rp);
#pragma unroll
      for (int f = 0; f < 5; ++f) rhs[f] = double(rp[f]);
    }
    // pv_target is read only where a term uses it: sponges, face operations, forcing
    const bool need_tg = (rloc >= a.c.sponge_start_top) || (!j1 && zloc <= a.c.sponge_end_left) ||
                         a.c.control_forcing == 1 || (GEN && face);
    double tg[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (need_tg) {
#pragma unroll
      for (int f = 0; f < 5; ++f) tg[f] = __ldg(a.target + f * PL + go);
    }
    if (a.c.control_forcing == 1) control_forcing(zloc, rloc, a.c, a.forcing, pv, tg, rhs);
    else if (a.c.control_forcing == 2) harmonic_forcing(zloc, rloc, cwt, a.c, rhs);
    if (GEN && face) {
      const Prim qd = convert<double>(q);
      const Deriv dd = convert<double>(d);
      const int n = __ldg(a.faces + face);
      for (int k = 0; k < n; ++k) {
        const int pid = __ldg(a.faces + face + 1 + k);
        face_op(cPatch[pid].bc, cPatch[pid].dir, j1, qd, dd, tg, xzd, erd, a.c.gam, rhs);
      }
    }
    sponge(zloc, rloc, j1, a.c, pv, tg, rhs);

    if (a.stage == 0) {
#pragma unroll
      for (int f = 0; f < 5; ++f) a.Uout[f * PL + go] = rhs[f];
      continue;
    }
    // ---- RK4 stage update (ModRungeKutta.f90:32-51, :134-146), always in double
    const double c6 = 1.0 / 6.0, c3 = 1.0 / 3.0;
    const int tp = r * TZ + c;  // index in the tile boxes
    double un[5];
#pragma unroll
    for (int f = 0; f < 5; ++f) {
      const double k = mul_rn(dtv, rhs[f]);
      const long long o = f * PL + go;
      if (a.stage == 1) {
        const double u0 = pv[f];  // pv_old = stage-1 input
        un[f] = add_rn(u0, mul_rn(0.5, k));
        a.A[o] = add_rn(u0, mul_rn(c6, k));
      } else if (a.stage == 2) {
        const double u0 = RKG ? __ldg(a.U0 + o) : sP0[f * NTP + tp];
        un[f] = add_rn(u0, mul_rn(0.5, k));
        a.B[o] = k;
      } else if (a.stage == 3) {
        const double u0 = RKG ? __ldg(a.U0 + o) : sP0[f * NTP + tp];
        un[f] = add_rn(u0, k);
        a.A[o] = add_rn(RKG ? a.A[o] : sPA[f * NTP + tp], mul_rn(c3, add_rn(__ldg(a.B + o), k)));
      } else {
        un[f] = blank ? pv[f] : add_rn(RKG ? a.A[o] : sPA[f * NTP + tp], mul_rn(c6, k));
      }
    }
    if (j1) {
      // axis_conditions (ModAxis.f90:14-29): rho, V_z, T at j = 1 from rows 2..6 of
      // the stage input (the vectors AssignValues filled before this stage).
      un[0] = axis_extrap(pR + RZ, RZ);
      un[3] = axis_extrap(pVz + RZ, RZ);
      un[4] = axis_extrap(pT + RZ, RZ);
    }
    if (a.out_f32 && a.stage < 4) {
#pragma unroll
      for (int f = 0; f < 5; ++f) a.Uout_f[f * PL + go] = float(un[f]);
    } else {
#pragma unroll
      for (int f = 0; f < 5; ++f) a.Uout[f * PL + go] = un[f];
    }
    if (a.stage == 4) {
      bool bad = false;
#pragma unroll
      for (int f = 0; f < 5; ++f) bad |= !isfinite(un[f]);
      if (bad) atomicOr(a.flags, 1);
      if (i == a.iT && j == a.jT) *a.staleT = pv[4];
    }
  }
  return true;
}

// One tile (i0, j0) of the fused stage with NT threads and TRT rows. Returns false if a
// bounded wait gave up (the flag is set; the caller stops).
template <int H, bool GEN, typename SIN, typename R, int CM, int NT = STAGE_THREADS, int TRT = TR>
__device__ __forceinline__ bool stage_body(const StageArgs& a, int i0, int j0, const CUtensorMap* mState,
                                           const CUtensorMap* mQ, const CUtensorMap* mU0, const CUtensorMap* mAcc,
                                           const CUtensorMap* mB, const CUtensorMap* mTg,
                                           unsigned char* smem_raw, uint64_t* bar, uint32_t& phase) {
  using SM = StageSmem<H, SIN, R, CM, TRT>;
  constexpr int HZ = SM::HZ, RZ = SM::RZ, NPT = SM::NPT, HT = SM::HT;
  SIN* sU = reinterpret_cast<SIN*>(smem_raw + SM::oU);            // [5][RR][RZ]
  double* sQ = reinterpret_cast<double*>(smem_raw + SM::oQ);      // [3][RQ][RZ]
  double* sMu0 = reinterpret_cast<double*>(smem_raw + SM::oMu0);  // [TR][TZ]
  double* sP0 = reinterpret_cast<double*>(smem_raw + SM::oP0);    // [5][TR][TZ]
  double* sPA = reinterpret_cast<double*>(smem_raw + SM::oPA);    // [5][TR][TZ]
  R* sDz = reinterpret_cast<R*>(smem_raw + SM::oDz(GEN));         // [2][RR][TZ]
  uint32_t* sDesc = reinterpret_cast<uint32_t*>(smem_raw + SM::oDesc(GEN));
  double* sMet = reinterpret_cast<double*>(smem_raw + SM::oMet(GEN));  // [3][TZ] + [4][TR]

  const int tid = threadIdx.x;
  const int Nz = a.g.Nz, Nr = a.g.Nr;
  const long long P = a.g.P;
  const bool sc = a.c.shock_capturing != 0;
  // general tiles of a thin r band own only its rows: TRT - (bits 24-31 of j0)
  int nrow = TRT;
  if (GEN) {
    nrow = TRT - (j0 >> 24);
    j0 &= 0xFFFFFF;
  }
  // pv_old is needed as a tile in stages 2 and 3 (stage 1 reads it from the state box),
  // the running sum A in stages 3 and 4; interior tiles stage them by TMA
  // RK operands from global memory (general tiles, FP32 half tiles) or staged by TMA
  constexpr bool RKG = GEN || rk_global<R, TRT>();
  const bool needU0 = !RKG && (a.stage == 2 || a.stage == 3);
  const bool needA = !RKG && (a.stage == 3 || a.stage == 4);

  // ---- phase 1: one thread issues the TMA loads; the RK operands complete on the
  // second barrier while phases 1-2 run. The barriers are initialised once per CTA by the
  // caller; phase bit b is the parity of bar[b]'s next completion. Prior generic-proxy
  // accesses of the shared buffers (a previous tile of a persistent CTA) are ordered
  // before the TMA writes by the proxy fence.
  __syncthreads();
  if (tid == 0) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&bar[0], SM::state_bytes + (sc ? SM::q_bytes : 0u));
    tma_load_3d(sU, mState, i0 - HZ, j0 - H, 0, &bar[0]);
    if (sc) tma_load_3d(sQ, mQ, i0 - HZ, j0 - H - HT, 0, &bar[0]);
    if (needU0 || needA) {
      mbar_expect_tx(&bar[1], (needU0 ? SM::tile_bytes : 0u) + (needA ? SM::tile_bytes : 0u));
      if (needU0) tma_load_3d(sP0, mU0, i0, j0, 0, &bar[1]);
      if (needA) tma_load_3d(sPA, mAcc, i0, j0, 0, &bar[1]);
    }
    // operands the RK update reads from global memory: into L2 now (k2 in stage 3; pv_old
    // and the running sum in general tiles, which do not stage them)
    if (mB && a.stage == 3) tma_prefetch_3d(mB, i0, j0, 0);
    // pv_target, which the sponges (and the face operations, the feedback forcing) read per
    // point from global memory: into L2 for the tiles that reach a sponge
    if (mTg) {
      const bool tgt = GEN || a.c.control_forcing == 1 || __ldg(a.zc + i0) <= a.c.sponge_end_left ||
                       __ldg(a.rc + min(j0 + TRT - 1, Nr - 1)) >= a.c.sponge_start_top;
      if (tgt) tma_prefetch_3d(mTg, i0, j0, 0);
    }
    if (RKG && (a.stage == 2 || a.stage == 3)) tma_prefetch_3d(mU0, i0, j0, 0);
    if (RKG && (a.stage == 3 || a.stage == 4)) tma_prefetch_3d(mAcc, i0, j0, 0);
  }
  if (GEN) {
    for (int idx = tid; idx < NPT; idx += NT) {
      const int rr = idx / RZ, rz = idx - rr * RZ;
      const int i = i0 - HZ + rz, j = j0 - H + rr;
      sDesc[idx] = (i >= 0 && i < Nz && j >= 0 && j < Nr) ? __ldg(a.desc + (long long)j * P + i)
                                                            : make_desc(ROW_NONE, ROW_NONE, false, 0);
    }
  }
  // the tile's metrics and coordinates (read per point in phases 2-3)
  if (tid < TZ) {
    const int i = min(i0 + tid, Nz - 1);
    sMet[tid] = __ldg(a.dxidz + i);
    sMet[TZ + tid] = __ldg(a.ddxidxidz + i);
    sMet[2 * TZ + tid] = __ldg(a.zc + i);
  } else if (tid < TZ + TRT) {
    const int r = tid - TZ, j = min(j0 + r, Nr - 1);
    sMet[3 * TZ + r] = __ldg(a.detadr + j);
    sMet[3 * TZ + TRT + r] = __ldg(a.ddetadetadr + j);
    sMet[3 * TZ + 2 * TRT + r] = __ldg(a.rc + j);
    sMet[3 * TZ + 3 * TRT + r] = __ldg(a.invr + j);
  }
  if (!__syncthreads_and(mbar_wait_bounded(&bar[0], phase & 1u))) {
    if (tid == 0) atomicOr(a.flags, 4);
    mbar_drain(&bar[0], phase & 1u);
    if (needU0 || needA) mbar_drain(&bar[1], (phase >> 1) & 1u);
    return false;
  }
  phase ^= 1u;
  const StagePtrs<SIN, R> sp{sU, sQ, sMu0, sP0, sPA, sDz, sDesc, sMet};
  const bool ok = stage_compute<H, GEN, SIN, R, CM, NT, TRT>(a, i0, j0, nrow, sp, &bar[1], (phase >> 1) & 1u);
  if (ok && (needU0 || needA)) phase ^= 2u;
  return ok;
}



// Threads of a stage CTA: 256 for tiles of TR rows (two CTAs per SM), 128 for the half
// tiles of TR / 2 rows (four CTAs per SM, six with FP32 stencils: while one waits for its
// boxes, the others compute).
__host__ __device__ constexpr int stage_threads(int trt) { return trt == TR ? STAGE_THREADS : STAGE_THREADS / 2; }
template <typename R, int TRT>
__host__ __device__ constexpr int stage_ctas() { return TRT == TR ? 2 : (rk_global<R, TRT>() ? 6 : 4); }

// One tile per CTA; with TRT < TR (interior tiles only) CTA k takes rows (k % NH) * TRT ..
// of tile k / NH, NH = TR / TRT.
template <int H, bool GEN, typename SIN, typename R, int CM, int TRT = TR>
__global__ void __launch_bounds__(stage_threads(TRT), (stage_ctas<R, TRT>()))
    stage_kernel(const StageArgs a, const int2* __restrict__ tiles, const __grid_constant__ CUtensorMap mState,
                 const __grid_constant__ CUtensorMap mQ, const __grid_constant__ CUtensorMap mU0,
                 const __grid_constant__ CUtensorMap mAcc, const __grid_constant__ CUtensorMap mB,
                 const __grid_constant__ CUtensorMap mTg) {
  static_assert(TRT == TR || !GEN, "general tiles run whole");
  constexpr int NH = TR / TRT;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bar[2];
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  uint32_t phase = 0;
  const int2 t0 = tiles[blockIdx.x / NH];
  const int j0 = NH > 1 ? t0.y + (int)(blockIdx.x % NH) * TRT : t0.y;
  stage_body<H, GEN, SIN, R, CM, stage_threads(TRT), TRT>(a, t0.x, j0, &mState, &mQ, &mU0, &mAcc, &mB, &mTg,
                                                          smem_raw, bar, phase);
}

// Batched form: a persistent grid-stride loop over the tiles (i0, j0, instance) of many
// solver instances; each instance's arguments and tensor maps come from device tables
// (the arguments are staged in shared memory per tile). With TRT < TR the table holds the
// half tiles of the interior class (their own origins) and the maps their boxes.
template <int H, bool GEN, typename SIN, typename R, int CM, int TRT = TR>
__global__ void __launch_bounds__(stage_threads(TRT), TRT == TR ? 1 : (stage_ctas<R, TRT>()))
    stage_kernel_batch(const StageArgs* __restrict__ argv, const int4* __restrict__ tiles, int ntiles,
                       const CUtensorMap* __restrict__ mapv, int nmaps, int4 kmaps) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ __align__(16) StageArgs sa;
  // the barriers live across the CTA's tiles: initialised once, phases tracked
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  uint32_t phase = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int4 tt = tiles[t];
    __syncthreads();  // the previous tile is finished with the arguments and the buffers
    for (int k = threadIdx.x; k < (int)(sizeof(StageArgs) / 8); k += blockDim.x)
      reinterpret_cast<unsigned long long*>(&sa)[k] = reinterpret_cast<const unsigned long long*>(argv + tt.z)[k];
    __syncthreads();
    const CUtensorMap* m = mapv + (size_t)tt.z * nmaps;
    if (!stage_body<H, GEN, SIN, R, CM, stage_threads(TRT), TRT>(sa, tt.x, tt.y, m + kmaps.x, m + kmaps.y,
                                                                 m + kmaps.z, m + kmaps.w, nullptr, nullptr, smem_raw,
                                                                 bar, phase))
      return;
  }
}

template <int H, bool GEN, typename SIN, typename R, int TRT = TR>
static cudaError_t launch_stage_t(const StageArgs& a, int ntiles, const int2* tiles, const StageMaps& m,
                                  cudaStream_t s) {
  if (ntiles <= 0) return cudaSuccess;
  const int grid = ntiles * (TR / TRT), nt = stage_threads(TRT);
  if (a.learned == CM_LRN) {
    const size_t sm = StageSmem<H, SIN, R, CM_LRN, TRT>::bytes(GEN);
    stage_kernel<H, GEN, SIN, R, CM_LRN, TRT>
        <<<grid, nt, sm, s>>>(a, tiles, *m.state, *m.star, *m.u0, *m.acc, *m.bt, *m.tg);
  } else if (a.learned == CM_PRE) {
    const size_t sm = StageSmem<H, SIN, R, CM_PRE, TRT>::bytes(GEN);
    stage_kernel<H, GEN, SIN, R, CM_PRE, TRT>
        <<<grid, nt, sm, s>>>(a, tiles, *m.state, *m.star, *m.u0, *m.acc, *m.bt, *m.tg);
  } else {
    const size_t sm = StageSmem<H, SIN, R, CM_FILT, TRT>::bytes(GEN);
    stage_kernel<H, GEN, SIN, R, CM_FILT, TRT>
        <<<grid, nt, sm, s>>>(a, tiles, *m.state, *m.star, *m.u0, *m.acc, *m.bt, *m.tg);
  }
  return cudaGetLastError();
}

// The general tiles (few, heavy, one CTA per SM) run on a side stream next to the
// interior tiles so that they fill SMs the interior launch leaves idle.
static cudaError_t fork(const SideStream& side, cudaStream_t s) {
  if (!side.stream) return cudaSuccess;
  cudaError_t e = cudaEventRecord(side.fork, s);
  if (e != cudaSuccess) return e;
  return cudaStreamWaitEvent(side.stream, side.fork, 0);
}
static cudaError_t join(const SideStream& side, cudaStream_t s) {
  if (!side.stream) return cudaSuccess;
  cudaError_t e = cudaEventRecord(side.join, side.stream);
  if (e != cudaSuccess) return e;
  return cudaStreamWaitEvent(s, side.join, 0);
}

template <typename SIN, typename R>
static cudaError_t launch_stage_pair(const StageArgs& a, int ntiles_int, const int2* tiles_int, const StageMaps& mint,
                                     int ntiles_gen, const int2* tiles_gen, const StageMaps& mgen,
                                     const SideStream& side, cudaStream_t s, int int_rows) {
  cudaError_t e = fork(side, s);
  if (e != cudaSuccess) return e;
  e = launch_stage_t<H_GEN, true, SIN, R>(a, ntiles_gen, tiles_gen, mgen, side.stream ? side.stream : s);
  if (e != cudaSuccess) return e;
  e = int_rows == TR / 2 ? launch_stage_t<H_INT, false, SIN, R, TR / 2>(a, ntiles_int, tiles_int, mint, s)
                        : launch_stage_t<H_INT, false, SIN, R>(a, ntiles_int, tiles_int, mint, s);
  if (e != cudaSuccess) return e;
  return join(side, s);
}

// FP64 path: double state, double stencils. Mixed path: the stage-1 input is pv_old
// (double), later inputs are FP32 stage states; stencils in FP32.
cudaError_t launch_stage(const StageArgs& a, int ntiles_int, const int2* tiles_int, const StageMaps& mint,
                         int ntiles_gen, const int2* tiles_gen, const StageMaps& mgen, const SideStream& side,
                         cudaStream_t s, int int_rows) {
  if (!a.mixed)
    return launch_stage_pair<double, double>(a, ntiles_int, tiles_int, mint, ntiles_gen, tiles_gen, mgen, side, s,
                                             int_rows);
  if (!a.in_f32)
    return launch_stage_pair<double, float>(a, ntiles_int, tiles_int, mint, ntiles_gen, tiles_gen, mgen, side, s,
                                            int_rows);
  return launch_stage_pair<float, float>(a, ntiles_int, tiles_int, mint, ntiles_gen, tiles_gen, mgen, side, s,
                                         int_rows);
}

void stage_boxes(bool gen, bool mixed, int* halo_w, int* halo_h, int* q_h, int* tile_w, int* tile_h, int* qlrn_h,
                 int rows) {
  if (!gen && rows == TR / 2) {
    using S = StageSmem<H_INT, double, double, CM_FILT, TR / 2>;
    *halo_w = mixed ? StageSmem<H_INT, float, float, CM_FILT, TR / 2>::RZ : S::RZ;
    *halo_h = S::RR;
    *q_h = S::RQ;
    if (qlrn_h) *qlrn_h = StageSmem<H_INT, double, double, CM_LRN, TR / 2>::RQ;
    *tile_w = TZ;
    *tile_h = TR / 2;
    return;
  }
  if (mixed) {
    *halo_w = gen ? StageSmem<H_GEN, float, float>::RZ : StageSmem<H_INT, float, float>::RZ;
  } else {
    *halo_w = gen ? StageSmem<H_GEN, double, double>::RZ : StageSmem<H_INT, double, double>::RZ;
  }
  *halo_h = gen ? StageSmem<H_GEN, double, double>::RR : StageSmem<H_INT, double, double>::RR;
  *q_h = gen ? StageSmem<H_GEN, double, double>::RQ : StageSmem<H_INT, double, double>::RQ;
  if (qlrn_h)
    *qlrn_h = gen ? StageSmem<H_GEN, double, double, CM_LRN>::RQ : StageSmem<H_INT, double, double, CM_LRN>::RQ;
  *tile_w = TZ;
  *tile_h = TR;
}

// ---------------------------------------------------------------------------
// ComputeTimeStep: per-point dt, FP64 min via warp shuffles, one partial per
// block, and the last block to finish reduces the partials (no memset needed,
// the counter is returned to 0).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// ComputeTimeStep over one instance with blocks blk = 0..nblk-1 (per-block minima in
// a.partial, the last block to finish reduces them).
// The minimum of dt = CFL / x over the points is CFL / (maximum of x): division by a
// positive x is monotonic and correctly rounded, so the two agree exactly; the kernel
// reduces x and divides once. Likewise max(mu/Re, lambda/Re) = max(mu, lambda)/Re. The
// divisions by Re and Re Pr are products with the reciprocals (within an ulp of the
// quotients). The stale T's square root is formed once. Blanked points contribute dt = 100
// (ModInputOutput.f90:398-400). A thread's (i, j) advances by the grid stride without a
// division per point.
__device__ __forceinline__ void dt_body(const DtArgs& a, int blk, int nblk) {
  const int Nz = a.g.Nz, Nr = a.g.Nr;
  const long long n = (long long)Nz * Nr;
  const long long PL = a.g.plane;
  const bool phys = a.c.dt_mode == DT_PHYSICAL;
  const double sqrtTst = sqrt(*a.staleT);
  const double inv_Re = 1.0 / a.c.Re, inv_RePr = 1.0 / (a.c.Re * a.c.Pr);
  double xm = 0.0;  // maximum of the denominators (0: no unblanked point yet)
  int bad = 0, blank = 0;
  const long long stride = (long long)nblk * DT_THREADS;
  const int sj = (int)(stride / Nz), si = (int)(stride - (long long)sj * Nz);
  long long p = (long long)blk * DT_THREADS + threadIdx.x;
  int j = (int)(p / Nz), i = (int)(p - (long long)j * Nz);
  for (; p < n; p += stride, i += si, j += sj) {
    if (i >= Nz) {  // i + si < 2 Nz: one carry at most
      i -= Nz;
      ++j;
    }
    const long long o = (long long)j * a.g.P + i;
    if (desc_blank(__ldg(a.desc + o))) {
      blank = 1;
      continue;
    }
    const double Vr = __ldg(a.U + 1 * PL + o), Vz = __ldg(a.U + 3 * PL + o), T = __ldg(a.U + 4 * PL + o);
    const double dxidz = __ldg(a.dxidz + i), detadr = __ldg(a.detadr + j);
    const double mu = mu_k<double>(T);
    const double beta = (3.0 / 5.0) * mu;
    const double lambda = beta - (2.0 / 3.0) * mu;
    // dt_point's denominator, term for term
    const double inv = fabs(Vz * dxidz + Vr * detadr) + (phys ? sqrt(T) : sqrtTst) * sqrt(dxidz * dxidz + detadr * detadr);
    double mx = (lambda > mu ? lambda : mu) * inv_Re;
    const double k = mu * inv_RePr;
    if (k > mx) mx = k;
    const double sabs = fabs(dxidz) + fabs(detadr);
    const double x = inv + 2.0 * mx * (sabs * sabs);
    if (!isfinite(x)) bad = 1;  // NaN, or an infinite input (which would give dt = 0)
    xm = fmax(xm, x);
  }
  __shared__ double sred[DT_THREADS / 32];
  __shared__ bool last;
  const bool anyblank = __syncthreads_or(blank);
  xm = warp_max(xm);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sred[w] = xm;
  if (bad) atomicOr(a.flags, 1);
  __syncthreads();
  if (w == 0) {
    xm = lane < DT_THREADS / 32 ? sred[lane] : 0.0;
    xm = warp_max(xm);
    if (lane == 0) {
      // per-block dt (CFL / its largest denominator; 100 if it only met blanked points)
      double v = a.c.CFL / xm;
      if (anyblank) v = fmin(v, 100.0);
      a.partial[blk] = v;
      __threadfence();
      const unsigned int done = atomicAdd(a.counter, 1u);
      last = (done == (unsigned int)nblk - 1);
    }
  }
  __syncthreads();
  if (last) {
    __threadfence();
    double mm = 1.0e300;
    for (int b = threadIdx.x; b < nblk; b += DT_THREADS) mm = fmin(mm, ((volatile double*)a.partial)[b]);
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

__global__ void __launch_bounds__(DT_THREADS) dt_kernel(const DtArgs a) { dt_body(a, blockIdx.x, gridDim.x); }

// Batched: blockIdx.y = instance.
__global__ void __launch_bounds__(DT_THREADS) dt_kernel_batch(const DtArgs* __restrict__ argv) {
  __shared__ __align__(16) DtArgs sa;
  for (int k = threadIdx.x; k < (int)(sizeof(DtArgs) / 8); k += blockDim.x)
    reinterpret_cast<unsigned long long*>(&sa)[k] = reinterpret_cast<const unsigned long long*>(argv + blockIdx.y)[k];
  __syncthreads();
  dt_body(sa, blockIdx.x, gridDim.x);
}

__global__ void harmonic_phase_kernel(const double* time, const double* dt, double omega, int rhs_mode, double* out) {
  const int s = threadIdx.x;
  if (rhs_mode) {
    if (s == 0) out[0] = cos(omega * *time);
    return;
  }
  if (s < 1 || s > 4) return;
  const double tend = *time, d = *dt;
  const double cs = s == 1 ? 0.0 : (s == 4 ? 1.0 : 0.5);
  out[s] = cos(omega * ((tend - d) + cs * d));
}

cudaError_t launch_harmonic_phase(const double* time, const double* dt, double omega, int rhs_mode, double* out,
                                  cudaStream_t s) {
  harmonic_phase_kernel<<<1, 32, 0, s>>>(time, dt, omega, rhs_mode, out);
  return cudaGetLastError();
}

// Blocks of the dt kernel for the current device: as many as are resident at once (one
// wave, every SM full), so that every thread's loads are in flight together.
int dt_grid_blocks() {
  int dev = 0, nsm = 148, per_sm = 4;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dt_kernel, DT_THREADS, 0) != cudaSuccess || per_sm < 1)
    per_sm = 4;
  return nsm * per_sm;
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
template <int HS, int HF, typename SIN, typename R>
struct SensSmem {
  static constexpr int HV = HS + HF;          // halo of V_r, V_z
  static constexpr int HVZ = hz_t(HV, (int)sizeof(R));
  static constexpr int HSZ = hz_t(HS, (int)sizeof(R));  // z halo of the temperature box
  static constexpr int VZ = TZ + 2 * HVZ, VR = TR + 2 * HV, NV = VZ * VR;
  static constexpr int SZ = TZ + 2 * HSZ, SR = TR + 2 * HS, NS = SZ * SR;
  static constexpr int DZ = TZ + 2 * HF;      // z-arm of the second derivatives: [TR][DZ]
  static constexpr int DR = TR + 2 * HF;      // r-arm: [DR][TZ]
  // byte offsets (every TMA destination 128-byte aligned): V_r, V_z [VR][VZ] each;
  // T [SR][SZ] (TMA); S and dil [SR][SZ]; general tiles: descriptors [VR][VZ]. V and T
  // are in the stage-input type, the rest in the stencil type. Once phase 2 has formed the
  // strain rates the V boxes are spent: f_sw [TR][TZ] then lives in the V_r box (interior
  // tiles) or the V_z box (general tiles), and the general tiles' second derivatives on the
  // arms ([TR][DZ] + [DR][TZ]) in the V_r box. rho is read from the stage input.
  static constexpr size_t oVr = 0;
  static constexpr size_t oVz = align128(sizeof(SIN) * NV);
  static constexpr size_t oT = align128(oVz + sizeof(SIN) * NV);
  static constexpr size_t oS = align128(oT + sizeof(SIN) * NS);
  static constexpr size_t oD = align128(oS + sizeof(R) * NS);
  static_assert(sizeof(R) * (TR * DZ + DR * TZ) <= sizeof(SIN) * NV && sizeof(R) * TR * TZ <= sizeof(SIN) * NV,
                "the arms and f_sw fit in a spent V box");
  static constexpr size_t oDesc = align128(oD + sizeof(R) * NS);
  // metrics of the S region: dxidz on its columns [SZ], detadr and 1/r on its rows
  // [2][SR]; deltaz, deltar on the tile [TZ] + [TR]
  __host__ __device__ static constexpr size_t oMet(bool gen) {
    return align128(oDesc + (gen ? sizeof(uint32_t) * NV : 0));
  }
  static constexpr int NMET = SZ + 2 * SR + TZ + TR;
  __host__ __device__ static constexpr size_t bytes(bool gen) { return align128(oMet(gen) + sizeof(double) * NMET); }
  static constexpr uint32_t tx_bytes = sizeof(SIN) * (2 * NV + NS);
};

// Threads of a sensor tile CTA: general tiles 512, one point per thread in the stencil
// phases (two CTAs per SM at 105 KB of shared memory and 64 registers); interior tiles
// 128, a 2 x 2 block of points per thread (five CTAs per SM at 44 KB).
__host__ __device__ constexpr int sens_threads(bool gen) { return gen ? 512 : 128; }

template <typename R>
__device__ __forceinline__ R sqrt_t(R x) { return sqrt(x); }

// Two neighbouring values of a shared-memory row in one 16-byte (double) or 8-byte
// (float) load; p must be aligned to the pair.
template <typename T>
struct Pair2;
template <>
struct Pair2<double> { using t = double2; };
template <>
struct Pair2<float> { using t = float2; };
template <typename T>
__device__ __forceinline__ void ld_pair(const T* p, T& a, T& b) {
  const typename Pair2<T>::t v = *reinterpret_cast<const typename Pair2<T>::t*>(p);
  a = v.x;
  b = v.y;
}
template <typename T>
__device__ __forceinline__ void st_pair(T* p, T a, T b) {
  typename Pair2<T>::t v;
  v.x = a;
  v.y = b;
  *reinterpret_cast<typename Pair2<T>::t*>(p) = v;
}
// The centred SBP1 row on values at offsets -2, -1, 1, 2 (the zero middle weight left
// out), in dot_c1's order.
template <typename R>
__device__ __forceinline__ R c1_of(R xm2, R xm1, R xp1, R xp2) {
  R s = tabv<R, 1>(4, 0) * xm2;
  s = s + tabv<R, 1>(4, 1) * xm1;
  s = s + tabv<R, 1>(4, 3) * xp1;
  s = s + tabv<R, 1>(4, 4) * xp2;
  return s;
}
// The 9-point fourth difference cC9 on x[0..8], left to right (c9dot's order).
template <typename R>
__device__ __forceinline__ R c9_of(const R* x) {
  const R* c = std::is_same<R, float>::value ? reinterpret_cast<const R*>(cC9f) : reinterpret_cast<const R*>(cC9);
  R s = c[0] * x[0];
#pragma unroll
  for (int m = 1; m < 9; ++m) s = s + c[m] * x[m];
  return s;
}
template <>
__device__ __forceinline__ float sqrt_t<float>(float x) { return sqrtf(x); }

// One sensor tile (i0, j0); false if a bounded wait gave up.
template <int HS, int HF, bool GEN, typename SIN, typename R>
__device__ __forceinline__ bool sensor_body(const SensorArgs& a, int i0, int j0, const CUtensorMap* mV,
                                            const CUtensorMap* mT, unsigned char* smem_raw,
                                            uint64_t& bar, uint32_t& phase) {
  using SM = SensSmem<HS, HF, SIN, R>;
  constexpr int NT = sens_threads(GEN);
  constexpr int HV = SM::HV, HVZ = SM::HVZ, HSZ = SM::HSZ, VZ = SM::VZ, NV = SM::NV;
  constexpr int SZ = SM::SZ, NS = SM::NS, DZ = SM::DZ, DR = SM::DR;
  SIN* sVr = reinterpret_cast<SIN*>(smem_raw + SM::oVr);   // [VR][VZ]
  SIN* sVz = reinterpret_cast<SIN*>(smem_raw + SM::oVz);   // [VR][VZ]
  SIN* sT = reinterpret_cast<SIN*>(smem_raw + SM::oT);     // [SR][SZ]
  R* sS = reinterpret_cast<R*>(smem_raw + SM::oS);         // [SR][SZ]
  R* sD = reinterpret_cast<R*>(smem_raw + SM::oD);         // [SR][SZ]
  R* sd2z = reinterpret_cast<R*>(smem_raw + SM::oVr);      // [TR][DZ] (general tiles, phase 3)
  R* sd2r = sd2z + TR * DZ;                                 // [DR][TZ] (general tiles, phase 3)
  // f_sw [TR][TZ] in a spent V box (after phase 2): V_z (general tiles) or V_r (interior)
  R* sFsw = reinterpret_cast<R*>(smem_raw + (GEN ? SM::oVz : SM::oVr));
  const SIN* rho0 = std::is_same<SIN, float>::value ? reinterpret_cast<const SIN*>(a.Uf)
                                                     : reinterpret_cast<const SIN*>(a.U);  // rho plane
  uint32_t* sDesc = reinterpret_cast<uint32_t*>(smem_raw + SM::oDesc);
  double* sMz = reinterpret_cast<double*>(smem_raw + SM::oMet(GEN));  // dxidz, column i0 - HSZ + k
  double* sMr = sMz + SZ;                                               // detadr, row j0 - HS + k
  double* sIr = sMr + SM::SR;                                           // 1/r (0 on the axis row)
  double* sDzv = sIr + SM::SR;                                          // deltaz on the tile columns
  double* sDrv = sDzv + TZ;                                             // deltar on the tile rows

  const int tid = threadIdx.x;
  const Grid g = a.g;
  const int Nz = g.Nz, Nr = g.Nr;
  // general tiles of a thin r band own only its rows: TR - (bits 24-31 of j0)
  int nrow = TR;
  if (GEN) {
    nrow = TR - (j0 >> 24);
    j0 &= 0xFFFFFF;
  }
  auto inside = [&](int i, int j) { return i >= 0 && i < Nz && j >= 0 && j < Nr; };
  auto vdesc = [&](int vidx) -> uint32_t { return GEN ? sDesc[vidx] : make_desc(4, 4, false, 0); };

  // ---- phase 1: V_r, V_z on the V region, T on the S region and rho on the tile by
  // TMA (zero outside the block), descriptors by plain loads meanwhile. The barrier is
  // initialised once per CTA by the caller (phase = parity of its next completion); the
  // proxy fence orders a previous tile's generic accesses before the TMA writes.
  __syncthreads();
  if (tid == 0) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&bar, SM::tx_bytes);
    tma_load_3d(sVr, mV, i0 - HVZ, j0 - HV, 1, &bar);
    tma_load_3d(sVz, mV, i0 - HVZ, j0 - HV, 3, &bar);
    tma_load_3d(sT, mT, i0 - HSZ, j0 - HS, 4, &bar);
  }
  // interior tiles: rho of the thread's 2 x 2 block of phase 3 (rows r, r + 1, columns
  // c, c + 1) into registers now, from the stage input (the tile lies inside the grid)
  SIN rho_pf[2][2];
  if constexpr (!GEN) {
    const int r = 2 * (tid / (TZ / 2)), c = 2 * (tid - (tid / (TZ / 2)) * (TZ / 2));
#pragma unroll
    for (int w = 0; w < 2; ++w) {
      const typename Pair2<SIN>::t v =
          __ldg(reinterpret_cast<const typename Pair2<SIN>::t*>(rho0 + (long long)(j0 + r + w) * g.P + (i0 + c)));
      rho_pf[w][0] = v.x;
      rho_pf[w][1] = v.y;
    }
  }
  if (GEN) {
    for (int idx = tid; idx < NV; idx += NT) {
      const int vr = idx / VZ, vz = idx - vr * VZ;
      const int i = i0 - HVZ + vz, j = j0 - HV + vr;
      sDesc[idx] = inside(i, j) ? __ldg(a.desc + (long long)j * g.P + i) : make_desc(ROW_NONE, ROW_NONE, false, 0);
    }
  }
  // metrics and coordinates of the region (clamped indices: values outside the grid are
  // never used)
  for (int k = tid; k < SM::NMET; k += NT) {
    double v;
    if (k < SZ) {
      v = __ldg(a.dxidz + min(max(i0 - HSZ + k, 0), Nz - 1));
    } else if (k < SZ + 2 * SM::SR) {
      const int q = (k - SZ) % SM::SR, j = min(max(j0 - HS + q, 0), Nr - 1);
      v = (k - SZ) < SM::SR ? __ldg(a.detadr + j) : __ldg(a.invr + j);
    } else if (k < SZ + 2 * SM::SR + TZ) {
      v = __ldg(a.dz + min(i0 + (k - SZ - 2 * SM::SR), Nz - 1));
    } else {
      v = __ldg(a.dr + min(j0 + (k - SZ - 2 * SM::SR - TZ), Nr - 1));
    }
    sMz[k] = v;
  }
  if (!__syncthreads_and(mbar_wait_bounded(&bar, phase & 1u))) {
    if (tid == 0) atomicOr(a.flags, 4);
    mbar_drain(&bar, phase & 1u);
    return false;
  }
  phase ^= 1u;

  R fkeep[2][2][2];     // interior tiles: f_sw of the thread's (up to two) blocks
  int fidx[2] = {-1, -1};  // their first point in the [TR][TZ] f_sw layout (-1: none)
  constexpr int NSIT = (NS + NT - 1) / NT;  // general tiles: S points per thread
  R fkg[GEN ? NSIT : 1];                    // general tiles: f_sw of the thread's tile points
  int fig[GEN ? NSIT : 1];                  // their index in the f_sw layout (-1: none)
#pragma unroll
  for (int u = 0; u < (GEN ? NSIT : 1); ++u) fig[u] = -1;
  // ---- phase 2: S and dilatation on the cross of the S region (reach HS either way);
  // f_sw on the tile. Interior tiles: 2 x 2 blocks of S points (rows sr, sr + 1, columns
  // sz, sz + 1; sr, sz even) over the z arm (the tile rows, TZ + 2 HS columns) and the r
  // arm (HS rows either side, the tile columns). Each block row's z windows come in three
  // pair loads per field, which also hold the block's own values; its r windows need the
  // rows sr - 2, sr - 1, sr + 2, sr + 3 besides. The arithmetic per point is the general
  // loop's (dot_c1's order, the zero middle weight left out). Points off the cross are
  // never read.
  if constexpr (!GEN) {
    static_assert(SZ % 2 == 0 && VZ % 2 == 0 && HSZ % 2 == 0 && HVZ % 2 == 0 && HS % 2 == 0 && TZ % 2 == 0 &&
                      TR % 2 == 0,
                  "pair loads need even offsets");
    constexpr int ZBW = (TZ + 2 * HS) / 2;        // blocks per z-arm row pair
    constexpr int NZB = (TR / 2) * ZBW;           // z-arm blocks
    constexpr int NRB = HS * (TZ / 2);            // r-arm blocks (2 HS rows, in pairs)
    const R k0 = tabv<R, 1>(4, 0), k1 = tabv<R, 1>(4, 1), k3 = tabv<R, 1>(4, 3), k4 = tabv<R, 1>(4, 4);
    static_assert(NZB + NRB <= 2 * NT, "two blocks per thread at most");
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int bq = tid + u * NT;
      if (bq >= NZB + NRB) break;
      int sr, sz;
      if (bq < NZB) {
        const int br = bq / ZBW;
        sr = HS + 2 * br;
        sz = HSZ - HS + 2 * (bq - br * ZBW);
      } else {
        const int k = bq - NZB, br = k / (TZ / 2);
        sr = 2 * br < HS ? 2 * br : 2 * br + TR;
        sz = HSZ + 2 * (k - br * (TZ / 2));
      }
      const bool zarm = bq < NZB;
      const bool rarm = sz >= HSZ && sz < HSZ + TZ;
      const int vidx = (sr + HV - HS) * VZ + (sz + HVZ - HSZ);
      // z: the centred SBP1 row at both points of a block row, accumulated pair load by pair
      // load (offsets -2, -1, +1, +2 of each point's own column); c0, c1 the points' values
      auto zpair = [&](const SIN* row, R& p0, R& p1, R& c0, R& c1v) {
        SIN u, v;
        ld_pair(row - 2, u, v);  // columns -2, -1
        p0 = k0 * R(u);
        p0 = p0 + k1 * R(v);
        p1 = k0 * R(v);
        ld_pair(row, u, v);      // columns 0, +1 (the points themselves)
        c0 = R(u);
        c1v = R(v);
        p0 = p0 + k3 * R(v);
        p1 = p1 + k1 * R(u);
        ld_pair(row + 2, u, v);  // columns +2, +3
        p0 = p0 + k4 * R(u);
        p1 = p1 + k3 * R(u);
        p1 = p1 + k4 * R(v);
      };
      // r: both block rows from rows sr - 2, sr - 1, sr + 2, sr + 3 and the block's own
      // values (ce[w][h] at row sr + w)
      auto rblock = [&](const SIN* col, const R ce[2][2], R g[2][2]) {
        SIN u, v;
        R m2[2], m1[2], p2[2], p3[2];
        ld_pair(col - 2 * VZ, u, v);
        m2[0] = R(u);
        m2[1] = R(v);
        ld_pair(col - VZ, u, v);
        m1[0] = R(u);
        m1[1] = R(v);
        ld_pair(col + 2 * VZ, u, v);
        p2[0] = R(u);
        p2[1] = R(v);
        ld_pair(col + 3 * VZ, u, v);
        p3[0] = R(u);
        p3[1] = R(v);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          R a0 = k0 * m2[h];
          a0 = a0 + k1 * m1[h];
          a0 = a0 + k3 * ce[1][h];
          a0 = a0 + k4 * p2[h];
          g[0][h] = a0;
          R a1 = k0 * m1[h];
          a1 = a1 + k1 * ce[0][h];
          a1 = a1 + k3 * p2[h];
          a1 = a1 + k4 * p3[h];
          g[1][h] = a1;
        }
      };
      R gzr[2][2], gzz[2][2], grr[2][2], grz[2][2], vr[2][2], vz[2][2];
#pragma unroll
      for (int w = 0; w < 2; ++w) {
        zpair(sVr + vidx + w * VZ, gzr[w][0], gzr[w][1], vr[w][0], vr[w][1]);
        zpair(sVz + vidx + w * VZ, gzz[w][0], gzz[w][1], vz[w][0], vz[w][1]);
      }
      rblock(sVr + vidx, vr, grr);
      rblock(sVz + vidx, vz, grz);
#pragma unroll
      for (int w = 0; w < 2; ++w) {
        const int j = j0 - HS + sr + w;
        const R er = R(sMr[sr + w]), ir = R(sIr[sr + w]);
        R S[2], dil[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const R xz = R(sMz[sz + h]);
          const R dVrdz = gzr[w][h] * xz;
          const R dVzdz = gzz[w][h] * xz;
          const R dVrdr = grr[w][h] * er;
          const R dVzdr = grz[w][h] * er;
          // V_r / r as V_r * (1/r) (the reference divides; the two differ by rounding)
          const R vr_r = vr[w][h] * ir;
          R d;
          if (j == 0) d = R(2.0) * dVrdr + dVzdz;
          else d = dVrdr + vr_r + dVzdz;
          const R S11 = dVrdr - R(1.0 / 3.0) * d;
          const R S13 = R(0.5) * (dVrdz + dVzdr);
          const R S33 = dVzdz - R(1.0 / 3.0) * d;
          const R S22 = (j == 0) ? dVrdr - R(1.0 / 3.0) * d : vr_r - R(1.0 / 3.0) * d;
          S[h] = sqrt_t<R>(S11 * S11 + S13 * S13 + S22 * S22 + S13 * S13 + S33 * S33);
          dil[h] = d;
          if (zarm && rarm) {
            const R vort = fabs(dVrdz - dVzdr);
            const R Hm = (R(-1.0) * d < R(0)) ? R(0) : R(1);
            const R eps = R((double)1e-15f);  // single-precision literal of the reference (:202)
            // kept in registers: the V_r box that holds f_sw is still being read
            fkeep[u][w][h] = Hm * (d * d) / (d * d + vort * vort + eps);
            fidx[u] = (sr - HS) * TZ + (sz - HSZ);
          }
        }
        st_pair(sS + (sr + w) * SZ + sz, S[0], S[1]);
        st_pair(sD + (sr + w) * SZ + sz, dil[0], dil[1]);
      }
    }
  } else {
#pragma unroll
  for (int u = 0; u < NSIT; ++u) {
    const int idx = tid + u * NT;
    if (idx >= NS) break;
    const int sr = idx / SZ, sz = idx - sr * SZ;
    const bool zarm = sr >= HS && sr < HS + TR && sz >= HSZ - HS && sz < HSZ + TZ + HS;
    const bool rarm = sz >= HSZ && sz < HSZ + TZ;
    R S = R(0), dil = R(0);
    const int i = i0 - HSZ + sz, j = j0 - HS + sr;
    if ((zarm || rarm) && (!GEN || inside(i, j))) {
      const int vidx = (sr + HV - HS) * VZ + (sz + HVZ - HSZ);
      const uint32_t dsc = vdesc(vidx);
      const int zr = desc_blank(dsc) ? (int)ROW_NONE : desc_zrow(dsc);
      const int rw = desc_blank(dsc) ? (int)ROW_NONE : desc_rrow(dsc);
      const R xz = R(sMz[sz]), er = R(sMr[sr]);
      const R dVrdz = dst<R, 1, GEN>(zr, sVr + vidx, 1) * xz;
      const R dVzdz = dst<R, 1, GEN>(zr, sVz + vidx, 1) * xz;
      const R dVrdr = dst<R, 1, GEN>(rw, sVr + vidx, VZ) * er;
      const R dVzdr = dst<R, 1, GEN>(rw, sVz + vidx, VZ) * er;
      const R vr = R(sVr[vidx]);
      // V_r / r as V_r * (1/r) (the reference divides; the two differ by rounding)
      const R vr_r = vr * R(sIr[sr]);
      if (j == 0) dil = R(2.0) * dVrdr + dVzdz;
      else dil = dVrdr + vr_r + dVzdz;
      const R S11 = dVrdr - R(1.0 / 3.0) * dil;
      const R S13 = R(0.5) * (dVrdz + dVzdr);
      const R S33 = dVzdz - R(1.0 / 3.0) * dil;
      const R S22 = (j == 0) ? dVrdr - R(1.0 / 3.0) * dil : vr_r - R(1.0 / 3.0) * dil;
      S = sqrt_t<R>(S11 * S11 + S13 * S13 + S22 * S22 + S13 * S13 + S33 * S33);
      if (zarm && rarm) {
        const R vort = fabs(dVrdz - dVzdr);
        const R Hm = (R(-1.0) * dil < R(0)) ? R(0) : R(1);
        const R eps = R((double)1e-15f);  // single-precision literal of the reference (:202)
        // kept in registers: the V_z box that holds f_sw is still being read
        fkg[u] = Hm * (dil * dil) / (dil * dil + vort * vort + eps);
        fig[u] = (sr - HS) * TZ + (sz - HSZ);
      }
    }
    sS[idx] = S;
    sD[idx] = dil;
  }
  }
  __syncthreads();
  if constexpr (GEN) {
    // every thread is done with the V boxes: f_sw into the V_z box
#pragma unroll
    for (int u = 0; u < NSIT; ++u)
      if (fig[u] >= 0) sFsw[fig[u]] = fkg[u];
    __syncthreads();
  }
  if constexpr (!GEN) {
    // every thread is done with the V boxes: f_sw into the V_r box
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      if (fidx[u] < 0) continue;
#pragma unroll
      for (int w = 0; w < 2; ++w) st_pair(sFsw + fidx[u] + w * TZ, fkeep[u][w][0], fkeep[u][w][1]);
    }
    __syncthreads();
  }

  // ---- phases 3-4 per field: fourth derivatives at the tile points (kept in registers:
  // PPT points per thread, 4 in interior tiles, 1 in general tiles, the general tiles'
  // arms in the spent V_r box). Interior tiles: SBP2 of SBP2 with the centred row both times is
  // the 9-point row cC9 = c * c (c the centred SBP2 row), applied to S, T, the dilatation
  // directly (one rounding per product instead of two stencil passes: the difference is
  // rounding only). General tiles: second derivatives on the arms with each arm point's
  // row, then the tile point's row.
  constexpr int PPT = (TZ * TR) / NT;
  // point q of a thread: a warp owns PPT consecutive rows of the tile, so a thread's
  // points are vertically adjacent and share most taps of their r stencils (loaded once)
  auto ppoint = [](int t, int q) { return (t >> 5) * (TZ * PPT) + q * TZ + (t & 31); };
  R d4z[3][PPT], d4r[3][PPT];
  if constexpr (!GEN) {
    // 2 x 2 blocks of points (rows r, r + 1 and columns c, c + 1; r, c even), every window
    // in pair loads: along z each block row's five pairs (columns c - 4 .. c + 5) serve its
    // two points, along r each of the ten rows r - 4 .. r + 5 serves the block rows it
    // reaches. Every point's sum keeps c9dot's order (taps left to right). The quantities
    // of a field leave as soon as its sums are complete.
    static_assert(NT * 4 == TZ * TR, "one 2 x 2 block of points per thread");
    const int r = 2 * (tid / (TZ / 2)), c = 2 * (tid - (tid / (TZ / 2)) * (TZ / 2));
    const int sidx = (HS + r) * SZ + (HSZ + c);
    const R* c9 = std::is_same<R, float>::value ? reinterpret_cast<const R*>(cC9f) : reinterpret_cast<const R*>(cC9);
    R zs[2][2], rs[2][2], Tc[2][2];
    auto four = [&](const auto* base, int f) {
      using E = std::remove_cv_t<std::remove_reference_t<decltype(base[0])>>;
#pragma unroll
      for (int w = 0; w < 2; ++w) {
        R z0 = R(0), z1 = R(0);
#pragma unroll
        for (int q = 0; q < 5; ++q) {
          R u, v;
          {
            E uu, vv;
            ld_pair(base + sidx + w * SZ - 4 + 2 * q, uu, vv);
            u = R(uu);
            v = R(vv);
          }
          const int m = 2 * q;  // u is column m - 4, v column m - 3
          if (q == 0) {
            z0 = c9[0] * u;
            z0 = z0 + c9[1] * v;
            z1 = c9[0] * v;
          } else if (q < 4) {
            z0 = z0 + c9[m] * u;
            z0 = z0 + c9[m + 1] * v;
            z1 = z1 + c9[m - 1] * u;
            z1 = z1 + c9[m] * v;
          } else {
            z0 = z0 + c9[8] * u;
            z1 = z1 + c9[7] * u;
            z1 = z1 + c9[8] * v;
          }
          if (f == 1 && q == 2) {
            Tc[w][0] = u;
            Tc[w][1] = v;
          }
        }
        zs[w][0] = z0;
        zs[w][1] = z1;
      }
#pragma unroll
      for (int m = 0; m < 10; ++m) {
        E uu, vv;
        ld_pair(base + sidx + (m - 4) * SZ, uu, vv);
        const R u = R(uu), v = R(vv);
        if (m == 0) {
          rs[0][0] = c9[0] * u;
          rs[0][1] = c9[0] * v;
        } else if (m < 9) {
          rs[0][0] = rs[0][0] + c9[m] * u;
          rs[0][1] = rs[0][1] + c9[m] * v;
        }
        if (m == 1) {
          rs[1][0] = c9[0] * u;
          rs[1][1] = c9[0] * v;
        } else if (m > 1) {
          rs[1][0] = rs[1][0] + c9[m - 1] * u;
          rs[1][1] = rs[1][1] + c9[m - 1] * v;
        }
      }
    };
    // ---- quantities to be filtered (ComputeTobeFilteredQuantities :204-215)
    const long long o = (long long)(j0 + r) * g.P + (i0 + c);
    R dzp[2], rho[2][2], fsw[2][2];
    {
      double a0, a1;
      ld_pair(sDzv + c, a0, a1);
      dzp[0] = R(a0);
      dzp[1] = R(a1);
#pragma unroll
      for (int w = 0; w < 2; ++w) {
        rho[w][0] = R(rho_pf[w][0]);
        rho[w][1] = R(rho_pf[w][1]);
        ld_pair(sFsw + (r + w) * TZ + c, fsw[w][0], fsw[w][1]);
      }
    }
    const R drw[2] = {R(sDrv[r]), R(sDrv[r + 1])};
    double out[2][2];
    four(sS, 0);
#pragma unroll
    for (int w = 0; w < 2; ++w)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const R dz = dzp[h], dr = drw[w];
        out[w][h] = double(rho[w][h] * fabs((zs[w][h] * (dz * dz) + rs[w][h] * (dr * dr))));
      }
#pragma unroll
    for (int w = 0; w < 2; ++w) st_pair(a.Q + o + w * g.P, out[w][0], out[w][1]);
    four(sD, 2);
#pragma unroll
    for (int w = 0; w < 2; ++w)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const R dz = dzp[h], dr = drw[w];
        out[w][h] = double(rho[w][h] * fsw[w][h] * fabs((zs[w][h] * (dz * dz) + rs[w][h] * (dr * dr))));
      }
#pragma unroll
    for (int w = 0; w < 2; ++w) st_pair(a.Q + g.plane + o + w * g.P, out[w][0], out[w][1]);
    four(sT, 1);
#pragma unroll
    for (int w = 0; w < 2; ++w)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const R dz = dzp[h], dr = drw[w];
        out[w][h] = double(rho[w][h] / (R(a.c.gam) * sqrt_t<R>(Tc[w][h])) * fabs((zs[w][h] * dz + rs[w][h] * dr)));
      }
#pragma unroll
    for (int w = 0; w < 2; ++w) st_pair(a.Q + 2 * g.plane + o + w * g.P, out[w][0], out[w][1]);
    return true;
  } else {
#pragma unroll
  for (int f = 0; f < 3; ++f) {
    for (int idx = tid; idx < TR * DZ + DR * TZ; idx += NT) {
      if (idx < TR * DZ) {
        const int r = idx / DZ, c = idx - r * DZ;  // point (i0 - HF + c, j0 + r)
        const int i = i0 - HF + c, j = j0 + r;
        R v = R(0);
        if (!GEN || inside(i, j)) {
          const int sidx = (HS + r) * SZ + (HSZ - HF + c);
          const uint32_t dsc = vdesc((HV + r) * VZ + (HVZ - HF + c));
          const int zr = desc_blank(dsc) ? (int)ROW_NONE : desc_zrow(dsc);
          v = f == 1 ? dst<R, 2, GEN>(zr, sT + sidx, 1) : dst<R, 2, GEN>(zr, (f == 0 ? sS : sD) + sidx, 1);
        }
        sd2z[idx] = v;
      } else {
        const int k = idx - TR * DZ;
        const int r = k / TZ, c = k - r * TZ;      // point (i0 + c, j0 - HF + r)
        const int i = i0 + c, j = j0 - HF + r;
        R v = R(0);
        if (!GEN || inside(i, j)) {
          const int sidx = (HS - HF + r) * SZ + (HSZ + c);
          const uint32_t dsc = vdesc((HV - HF + r) * VZ + (HVZ + c));
          const int rw = desc_blank(dsc) ? (int)ROW_NONE : desc_rrow(dsc);
          v = f == 1 ? dst<R, 2, GEN>(rw, sT + sidx, SZ) : dst<R, 2, GEN>(rw, (f == 0 ? sS : sD) + sidx, SZ);
        }
        sd2r[k] = v;
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < PPT; ++q) {
      const int pidx = ppoint(tid, q);
      const int r = pidx / TZ, c = pidx - r * TZ;
      const uint32_t dsc = vdesc((HV + r) * VZ + (HVZ + c));
      const int zr = desc_blank(dsc) ? (int)ROW_NONE : desc_zrow(dsc);
      const int rw = desc_blank(dsc) ? (int)ROW_NONE : desc_rrow(dsc);
      d4z[f][q] = dst<R, 2, GEN>(zr, sd2z + r * DZ + HF + c, 1);
      d4r[f][q] = dst<R, 2, GEN>(rw, sd2r + (HF + r) * TZ + c, TZ);
    }
    __syncthreads();
  }
  }

  // ---- quantities to be filtered (ComputeTobeFilteredQuantities :204-215); the interior
  // tiles returned above
  if constexpr (GEN) {
#pragma unroll
  for (int q = 0; q < PPT; ++q) {
    const int pidx = ppoint(tid, q);
    const int r = pidx / TZ, c = pidx - r * TZ;
    const int i = i0 + c, j = j0 + r;
    if (!inside(i, j) || r >= nrow) continue;
    const long long o = (long long)j * g.P + i;
    const R dz = R(sDzv[c]), dr = R(sDrv[r]);
    const R rho = R(rho0[o]);
    const R T = R(sT[(HS + r) * SZ + HSZ + c]);
    const R fsw = sFsw[r * TZ + c];
    a.Q[o] = double(rho * fabs((d4z[0][q] * (dz * dz) + d4r[0][q] * (dr * dr))));
    a.Q[g.plane + o] = double(rho * fsw * fabs((d4z[2][q] * (dz * dz) + d4r[2][q] * (dr * dr))));
    a.Q[2 * g.plane + o] = double(rho / (R(a.c.gam) * sqrt_t<R>(T)) * fabs((d4z[1][q] * dz + d4r[1][q] * dr)));
  }
  }
  return true;
}

template <int HS, int HF, bool GEN, typename SIN, typename R>
__global__ void __launch_bounds__(sens_threads(GEN), GEN ? 2 : 5)
    sensor_tile_kernel(const SensorArgs a, const int2* __restrict__ tiles, const __grid_constant__ CUtensorMap mV,
                       const __grid_constant__ CUtensorMap mT) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  uint32_t phase = 0;
  const int2 t0 = tiles[blockIdx.x];
  sensor_body<HS, HF, GEN, SIN, R>(a, t0.x, t0.y, &mV, &mT, smem_raw, bar, phase);
}

// Batched form: persistent loop over (i0, j0, instance) tiles; kmaps = indices of the
// V and T maps in each instance's block of nmaps maps.
template <int HS, int HF, bool GEN, typename SIN, typename R>
__global__ void __launch_bounds__(sens_threads(GEN), GEN ? 2 : 5)
    sensor_tile_kernel_batch(const SensorArgs* __restrict__ argv, const int4* __restrict__ tiles, int ntiles,
                             const CUtensorMap* __restrict__ mapv, int nmaps, int4 kmaps) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ __align__(16) SensorArgs sa;
  // the barrier lives across the CTA's tiles: initialised once, its phase tracked
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  uint32_t phase = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int4 tt = tiles[t];
    __syncthreads();
    for (int k = threadIdx.x; k < (int)(sizeof(SensorArgs) / 8); k += blockDim.x)
      reinterpret_cast<unsigned long long*>(&sa)[k] = reinterpret_cast<const unsigned long long*>(argv + tt.z)[k];
    __syncthreads();
    const CUtensorMap* m = mapv + (size_t)tt.z * nmaps;
    if (!sensor_body<HS, HF, GEN, SIN, R>(sa, tt.x, tt.y, m + kmaps.x, m + kmaps.y, smem_raw, bar, phase))
      return;
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
__device__ __forceinline__ void rfilter_body(const SensorArgs& a, long long p) {
  const Grid g = a.g;
  const long long n = (long long)g.Nz * g.Nr;
  if (p >= n) return;
  const int j = (int)(p / g.Nz), i = (int)(p - (long long)j * g.Nz);
  const long long o = (long long)j * g.P + i;
  const uint32_t dsc = __ldg(a.desc + o);
  const int row = row_of(dsc, 2);
  const double scale[3] = {a.c.C_mu_Re, a.c.C_beta_Re, a.c.C_kappa_Re_Pr};
  const double ramp = a.ramp_off ? 1.0 : __ldg(a.ramp + i);
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

template <typename SIN, typename R>
static void launch_sensor_tiles(const SensorArgs& a, const SideStream& side, cudaStream_t s) {
  using SG = SensSmem<SENS_HS_GEN, H_GEN, SIN, R>;
  using SI = SensSmem<SENS_HS_INT, H_INT, SIN, R>;
  if (a.ntiles_gen > 0)
    sensor_tile_kernel<SENS_HS_GEN, H_GEN, true, SIN, R><<<a.ntiles_gen, sens_threads(true), SG::bytes(true),
                                                           side.stream ? side.stream : s>>>(a, a.tiles_gen, *a.mv_gen,
                                                                                            *a.mt_gen);
  if (a.ntiles_int > 0)
    sensor_tile_kernel<SENS_HS_INT, H_INT, false, SIN, R>
        <<<a.ntiles_int, sens_threads(false), SI::bytes(false), s>>>(a, a.tiles_int, *a.mv_int, *a.mt_int);
}

__global__ void sensor_rfilter_kernel(const SensorArgs a) {
  rfilter_body(a, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

// Batched: blockIdx.y = instance.
__global__ void sensor_rfilter_kernel_batch(const SensorArgs* __restrict__ argv) {
  rfilter_body(argv[blockIdx.y], (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

cudaError_t launch_sensor(const SensorArgs& a, bool rfilter, const SideStream& side, cudaStream_t s) {
  const long long n = (long long)a.g.Nz * a.g.Nr;
  const int bs = 256;
  const int nb = (int)((n + bs - 1) / bs);
  cudaError_t e = fork(side, s);
  if (e != cudaSuccess) return e;
  if (!a.mixed) launch_sensor_tiles<double, double>(a, side, s);
  else if (!a.in_f32) launch_sensor_tiles<double, float>(a, side, s);
  else launch_sensor_tiles<float, float>(a, side, s);
  e = join(side, s);
  if (e != cudaSuccess) return e;
  e = launch_tgfilter_z_inplace(a.g, a.desc, a.zcode, a.Q, a.Qz, 3, a.flags, s);
  if (e != cudaSuccess) return e;
  if (rfilter) sensor_rfilter_kernel<<<nb, bs, 0, s>>>(a);  // the stage kernel applies it on the fly
  return cudaGetLastError();
}

// Row-staged version of the same recurrence: one CTA per (row, field). The row of
// unfiltered values and its z row codes are bulk-copied into shared memory with ZR_PADL
// zeros (row code 4) on the left and ZR_PADR on the right, the never-written halo of
// the reference. Each chunk of ZR_L points runs ZR_STEPS = ZR_W + ZR_L steps of the
// recurrence; left of its window it starts from unfiltered values (the recurrence
// forgets them: see ZR_W). Two kinds of chunk:
//  * centred chunks (every row code in the window is 4, window inside the row): a
//    fully unrolled loop with the last 10 filtered values in a statically renamed
//    register ring and the ZR_L outputs in registers, which go back through shared
//    memory and leave as coalesced row stores;
//  * general chunks (closure rows, blanked points, or a window that starts left of the
//    row, which then starts exactly at i = 0 from the zero halo): a rolled loop with a
//    shifted register ring; centred points use the same arithmetic as above, the others
//    the padded 21-tap form of their row (left to right, as DOT_PRODUCT sums). They
//    store their outputs directly.
// Chunks are reordered so the general ones share warps (thread t runs chunk order[t]).
constexpr int ZR_L = 31;
constexpr int ZR_W = 49;
constexpr int ZR_STEPS = ZR_L + ZR_W;  // 80 = 8 x 10
constexpr int ZR_PADL = 64;            // >= ZR_W + 10, a multiple of 16 doubles
constexpr int ZR_PADR = 48;            // >= ZR_L + 10 - 1: windows read up to i+10 past the row
constexpr int ZR_MAXNZ = 10240;  // the staged row and its codes fit in shared memory
constexpr int ZR_MAXCHUNK = (ZR_MAXNZ + ZR_L - 1) / ZR_L;


__host__ __device__ constexpr int zr_pad(int nz) { return (nz + 15) & ~15; }
__host__ __device__ constexpr int zr_xlen(int nz) { return ZR_PADL + zr_pad(nz) + ZR_PADR; }

// Shared-memory layout of one row: unfiltered row (doubles, padded) | the 21-tap padded
// TG rows [10][21] (doubles; row 9 = identity) | row codes (bytes, padded) | chunk order
// (int16) | chunk flags (bytes).
__host__ __device__ constexpr size_t zr_off_w(int nz) { return sizeof(double) * (size_t)zr_xlen(nz); }
__host__ __device__ constexpr size_t zr_off_codes(int nz) { return zr_off_w(nz) + sizeof(double) * 10 * 21; }
__host__ __device__ constexpr size_t zr_off_order(int nz, long long P) {
  return (zr_off_codes(nz) + (size_t)(ZR_PADL + P + ZR_PADR) + 1) & ~(size_t)1;
}
__host__ __device__ constexpr size_t zr_off_flags(int nz, long long P) {
  return zr_off_order(nz, P) + sizeof(short) * (size_t)ZR_MAXCHUNK;
}

// Requires blockDim.x >= the number of chunks, (Nz + ZR_L - 1) / ZR_L, and a multiple of 32.
__device__ __forceinline__ void zrows_body(const Grid& g, const unsigned char* __restrict__ zcode,
                                           const double* __restrict__ q, double* __restrict__ out, int* flags, int j,
                                           int f, unsigned char* zr_smem, uint64_t& bar) {
  const int Nz = g.Nz, P = (int)g.P;
  const int nchunk = (Nz + ZR_L - 1) / ZR_L;
  double* xs = reinterpret_cast<double*>(zr_smem);                           // [zr_xlen(Nz)]
  double* wt = reinterpret_cast<double*>(zr_smem + zr_off_w(Nz));           // [10][21]
  unsigned char* rs = zr_smem + zr_off_codes(Nz);                            // [ZR_PADL + P + ZR_PADR]
  short* order = reinterpret_cast<short*>(zr_smem + zr_off_order(Nz, P));   // [nchunk]
  unsigned char* genf = zr_smem + zr_off_flags(Nz, P);                       // [nchunk]
  __shared__ int warp_gen[32];
  const double* x = q + (long long)f * g.plane + (long long)j * g.P;
  double* y = out + (long long)f * g.plane + (long long)j * g.P;
  // the row of Q and its z stencil codes arrive by two bulk copies
  const uint32_t xbytes = (uint32_t)(Nz / 2) * 16u;
  const uint32_t rbytes = (uint32_t)P;  // P is a multiple of 32
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    mbar_expect_tx(&bar, xbytes + rbytes);
    bulk_g2s(xs + ZR_PADL, x, xbytes, &bar);
    bulk_g2s(rs + ZR_PADL, zcode + (long long)j * g.P, rbytes, &bar);
  }
  // pads (disjoint from the bulk destinations) and the padded TG rows: row r's taps
  // sit at offsets tg_w0(r) .. tg_w0(r) + tg_len(r) - 1 of [-10, 10]; row 9 copies x(i)
  for (int k = threadIdx.x; k < ZR_PADL; k += blockDim.x) {
    xs[k] = 0.0;
    rs[k] = 4;
  }
  for (int k = ZR_PADL + 2 * (Nz / 2) + threadIdx.x; k < zr_xlen(Nz); k += blockDim.x) xs[k] = 0.0;
  for (int k = threadIdx.x; k < ZR_PADR; k += blockDim.x) rs[ZR_PADL + P + k] = 4;
  for (int k = threadIdx.x; k < 10 * 21; k += blockDim.x) {
    const int r = k / 21, o = k - r * 21 - 10;
    double w = 0.0;
    if (r < 9) {
      const int m = o - tg_w0(r);
      if (m >= 0 && m < tg_len(r)) w = cTG[r][m];
    } else {
      w = (o == 0) ? 1.0 : 0.0;
    }
    wt[k] = w;
  }
  if (!__syncthreads_and(mbar_wait_bounded(&bar, 0))) {
    if (threadIdx.x == 0) atomicOr(flags, 4);
    mbar_drain(&bar, 0);
    return;
  }
  if ((Nz & 1) && threadIdx.x == 0) xs[ZR_PADL + Nz - 1] = __ldg(x + Nz - 1);
  // positions past Nz are not part of the row: treat them as centred (their outputs
  // are never stored and only feed later, also unstored, positions)
  for (int k = Nz + threadIdx.x; k < P; k += blockDim.x) rs[ZR_PADL + k] = 4;
  __syncthreads();
  const double* X = xs + ZR_PADL;  // X[i], i in [-ZR_PADL, Nz + pad)
  const unsigned char* R = rs + ZR_PADL;
  // classify the chunks, then order them: general chunks first (an exclusive scan over
  // the block of the general flags)
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  bool g_me = false;
  if (t < nchunk) {
    const int is = t * ZR_L - ZR_W;
    g_me = is < 0;
    for (int k = max(is, 0); k < min(is + ZR_STEPS, Nz) && !g_me; ++k) g_me = R[k] != 4;
    genf[t] = g_me ? 1 : 0;
  }
  const unsigned bal = __ballot_sync(0xffffffffu, g_me);
  if (lane == 0) warp_gen[wid] = __popc(bal);
  __syncthreads();
  int gbefore = 0, ngen = 0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
    gbefore += (w < wid) ? warp_gen[w] : 0;
    ngen += warp_gen[w];
  }
  if (t < nchunk) {
    const int grank = gbefore + __popc(bal & ((1u << lane) - 1u));
    order[g_me ? grank : ngen + (t - grank)] = (short)t;
  }
  __syncthreads();

  const double t0 = cTG[4][0], t1 = cTG[4][1], t2 = cTG[4][2], t3 = cTG[4][3], t4 = cTG[4][4];
  const double t5 = cTG[4][5], t6 = cTG[4][6], t7 = cTG[4][7], t8 = cTG[4][8];
  const int c = (t < nchunk) ? order[t] : 0;
  const int ib = c * ZR_L, is = ib - ZR_W;
  double outv[ZR_L];
  if (t < ngen) {
    // general chunk: h1..h10 = filtered values at i-1..i-10
    const int i0c = max(is, 0);
    const int ie = min(Nz, ib + ZR_L);
    double h1 = X[i0c - 1], h2 = X[i0c - 2], h3 = X[i0c - 3], h4 = X[i0c - 4], h5 = X[i0c - 5];
    double h6 = X[i0c - 6], h7 = X[i0c - 7], h8 = X[i0c - 8], h9 = X[i0c - 9], h10 = X[i0c - 10];
    for (int i = i0c; i < ie; ++i) {
      const double* xp = X + i;
      const int row = R[i];
      double v;
      if (row == 4) {
        const double ff = t4 * xp[0] + t5 * xp[1] + t6 * xp[2] + t7 * xp[3] + t8 * xp[4];
        const double fb = t0 * h4 + t1 * h3 + t2 * h2;
        v = (ff + fb) + t3 * h1;
      } else {
        const double* w = wt + (row < 9 ? row : 9) * 21;  // w[o + 10], o = -10..10
        double sacc = w[0] * h10;
        sacc = sacc + w[1] * h9;
        sacc = sacc + w[2] * h8;
        sacc = sacc + w[3] * h7;
        sacc = sacc + w[4] * h6;
        sacc = sacc + w[5] * h5;
        sacc = sacc + w[6] * h4;
        sacc = sacc + w[7] * h3;
        sacc = sacc + w[8] * h2;
        sacc = sacc + w[9] * h1;
#pragma unroll
        for (int o = 0; o <= 10; ++o) sacc = sacc + w[10 + o] * xp[o];
        v = sacc;
      }
      h10 = h9; h9 = h8; h8 = h7; h7 = h6; h6 = h5; h5 = h4; h4 = h3; h3 = h2; h2 = h1; h1 = v;
      if (i >= ib) y[i] = v;
    }
  } else if (t < nchunk) {
    double ring[10];
#pragma unroll
    for (int m = 1; m <= 10; ++m) ring[10 - m] = X[is - m];
#pragma unroll
    for (int s = 0; s < ZR_STEPS; ++s) {
      const double* xp = X + is + s;
      // the feed-forward terms and the older feedback terms first, the newest
      // filtered value last: one FMA of latency per step on the recurrence (the
      // reference sums left to right; the two orders differ by rounding only)
      const double ff = t4 * xp[0] + t5 * xp[1] + t6 * xp[2] + t7 * xp[3] + t8 * xp[4];
      const double fb = t0 * ring[(s + 6) % 10] + t1 * ring[(s + 7) % 10] + t2 * ring[(s + 8) % 10];
      const double v = (ff + fb) + t3 * ring[(s + 9) % 10];
      ring[s % 10] = v;
      if (s >= ZR_W) outv[s - ZR_W] = v;
    }
  }
  // every thread has finished reading the unfiltered row: the centred chunks' outputs
  // replace it, and leave with the rest of the row (general chunks stored theirs)
  __syncthreads();
  if (t >= ngen && t < nchunk) {
#pragma unroll
    for (int k = 0; k < ZR_L; ++k) xs[ZR_PADL + ib + k] = outv[k];  // ib + k < zr_xlen(Nz) - ZR_PADL
  }
  __syncthreads();
  for (int k = t; k < Nz; k += blockDim.x)
    if (!genf[k / ZR_L]) y[k] = X[k];
}

__global__ void tgfilter_z_rows_kernel(const Grid g, const unsigned char* __restrict__ zcode,
                                       const double* __restrict__ q, double* __restrict__ out, int* flags) {
  extern __shared__ __align__(128) unsigned char zr_smem[];
  __shared__ __align__(8) uint64_t bar;
  zrows_body(g, zcode, q, out, flags, blockIdx.x, blockIdx.y, zr_smem, bar);
}

// Batched: blockIdx.x indexes rows (instance, j) of all instances, blockIdx.y the field;
// the instance's grid and buffers come from its sensor arguments.
__global__ void tgfilter_z_rows_kernel_batch(const SensorArgs* __restrict__ argv, const int2* __restrict__ rows) {
  extern __shared__ __align__(128) unsigned char zr_smem[];
  __shared__ __align__(8) uint64_t bar;
  const int2 r = rows[blockIdx.x];
  const SensorArgs& a = argv[r.x];
  const Grid g = a.g;
  zrows_body(g, a.zcode, a.Q, a.Qz, a.flags, r.y, blockIdx.y, zr_smem, bar);
}

// ---------------------------------------------------------------------------
// Fused z filter, r filter and transport coefficients (ModShockCapturing.f90:63-92,
// :248-251; ModAssign.f90:20-23): from the unfiltered sensor quantities Q to
// mu_eff = mu + mu*, beta = 0.6 mu + beta* and kappa_eff = mu + kappa* at every point.
//
// A CTA owns a segment of z positions (a multiple of ZRK_BZ) and ZRK_RB rows. It runs the
// in-place z recurrence of PerformTGfilter(q, 1, q) for the three quantities on its rows
// and ZRK_HR rows either side (the reach of the 11-point TG boundary rows of the r
// filter): one thread per (quantity, row), marching along z in blocks of ZRK_BZ
// positions. Segments start ZRK_WARM positions early from a zero history (the
// recurrence forgets its start: the dominant root of its feedback part is about 0.47, so
// 0.47**64 < 1e-20); the first segment starts exactly at i = 0 from the reference's zero
// halo. The z-filtered block goes to shared memory, where the r filter
// PerformTGfilter(q, 2, star) of the CTA's rows is applied with the point's r row, then
// the C*Re(*Pr) scaling, the z ramp and mu = T**0.666 of the stage input.
// Blocks of Q arrive by TMA (128-byte swizzle: a thread reads its row's 16 values as 8
// conflict-free 16-byte loads) into two slots: block k supplies the up to 10 values
// right of block k-1 that the filter rows reach, and once both are in registers the
// slot of block k-1 takes block k+1, which lands while block k-1 is filtered.
// ---------------------------------------------------------------------------
constexpr int ZRK_LANES = 3 * ZRK_NR;  // 156 recurrences per CTA
constexpr int ZRK_WARM = 64;           // warm-up positions (4 blocks)
constexpr int ZRK_QROW = ZRK_BZ * 8;   // bytes of one row of a Q block (128)

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// Byte offset of 16-byte chunk c of row R in a Q block stored with the 128-byte swizzle
// (chunk index XOR row mod 8), as TMA writes it.
__device__ __forceinline__ int zrk_chunk(int R, int c) { return R * ZRK_QROW + ((c ^ (R & 7)) << 4); }
// The z-filtered block is stored transposed, [quantity][position][row] with ZRK_ZP rows
// (odd: the r filter's reads, 16 positions x 2 rows per warp, and the recurrence's writes,
// consecutive rows per warp, are free of bank conflicts), so the r filter's taps are
// consecutive doubles at fixed offsets.
constexpr int ZRK_ZP = ZRK_NR + 1;

template <typename SIN>
struct ZrSmem {
  static constexpr size_t qbytes = (size_t)ZRK_LANES * ZRK_QROW;
  static constexpr size_t qslot = (qbytes + 1023) / 1024 * 1024;
  static constexpr size_t zslot = ((size_t)3 * ZRK_BZ * ZRK_ZP * sizeof(double) + 1023) / 1024 * 1024;
  static constexpr size_t oQ = 0;                                            // [2] Q blocks (swizzled)
  static constexpr size_t oZ = 2 * qslot;                                    // z-filtered block [3][16][ZRK_ZP]
  static constexpr size_t oZc = oZ + zslot;                                  // [2][ZRK_NR][16] z row codes
  static constexpr size_t zcbytes = (size_t)ZRK_NR * ZRK_BZ;
  static constexpr size_t oT = oZc + 2 * 1024;                               // [2][ZRK_RB][16] T
  static constexpr size_t tbytes = (size_t)ZRK_RB * ZRK_BZ * sizeof(SIN);
  static constexpr size_t oRc = oT + 2 * ((tbytes + 127) / 128 * 128);       // [2][ZRK_RB][16] r row codes
  static constexpr size_t rcbytes = (size_t)ZRK_RB * ZRK_BZ;
  static constexpr size_t oW = oRc + 2 * 512;                                // [10][21] padded TG rows
  static constexpr size_t bytes = oW + 10 * 21 * sizeof(double) + 1024;      // + alignment slack
  static constexpr uint32_t tx = (uint32_t)(qbytes + zcbytes + tbytes + rcbytes);
  static_assert(zcbytes <= 1024 && rcbytes <= 512, "code slots");
};

// The fused z/r filter for the CTA (bx, by): z positions bx * a.seg .., rows by * ZRK_RB ..
template <typename SIN, typename R>
__device__ __forceinline__ void zr_body(const ZrArgs& a, const CUtensorMap* pQ, const CUtensorMap* pZc,
                                        const CUtensorMap* pRc, const CUtensorMap* pT, int bx, int by,
                                        unsigned char* zrk_raw, uint64_t* bar) {
  using SM = ZrSmem<SIN>;
  unsigned char* base = zrk_raw + ((1024u - (smem_u32(zrk_raw) & 1023u)) & 1023u);
  double* wt = reinterpret_cast<double*>(base + SM::oW);
  const int tid = threadIdx.x;
  const int Nz = a.g.Nz, Nr = a.g.Nr;
  const long long P = a.g.P, PL = a.g.plane;
  const int zs = bx * a.seg, ze = min(Nz, zs + a.seg);
  const int j0 = by * ZRK_RB;
  const int bs = max(0, zs - ZRK_WARM) / ZRK_BZ;  // first block filtered (zs is a multiple of ZRK_BZ)
  const int be = (ze + ZRK_BZ - 1) / ZRK_BZ;       // blocks bs..be-1 are filtered, block be is loaded too
  // padded TG rows: row r's taps at offsets tg_w0(r) .. tg_w0(r) + tg_len(r) - 1 of
  // [-10, 10]; row 9 (blanked, or no filter row) keeps the value in place
  for (int k = tid; k < 10 * 21; k += ZRK_THREADS) {
    const int r = k / 21, o = k - r * 21 - 10;
    double w = 0.0;
    if (r < 9) {
      const int m = o - tg_w0(r);
      if (m >= 0 && m < tg_len(r)) w = cTG[r][m];
    } else {
      w = (o == 0) ? 1.0 : 0.0;
    }
    wt[k] = w;
  }
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  // slot k & 1 receives Q and the z codes of block k, and T and the r codes of block
  // k - 1 (the block the r filter handles in iteration k)
  auto issue = [&](int k) {
    const int sl = k & 1;
    unsigned char* q = base + SM::oQ + sl * SM::qslot;
    mbar_expect_tx(&bar[sl], SM::tx);
    tma_load_3d(q, pQ, ZRK_BZ * k, j0 - ZRK_HR, 0, &bar[sl]);
    tma_load_2d(base + SM::oZc + sl * 1024, pZc, ZRK_BZ * k, j0 - ZRK_HR, &bar[sl]);
    tma_load_3d(base + SM::oT + sl * ((SM::tbytes + 127) / 128 * 128), pT, ZRK_BZ * (k - 1), j0, 4, &bar[sl]);
    tma_load_2d(base + SM::oRc + sl * 512, pRc, ZRK_BZ * (k - 1), j0, &bar[sl]);
  };
  if (tid == 0) issue(bs);

  const bool lane_on = tid < ZRK_LANES;
  const int fq = lane_on ? tid / ZRK_NR : 0;
  const int rr = lane_on ? tid - fq * ZRK_NR : 0;
  const int Rq = fq * ZRK_NR + rr;  // row of this recurrence in the Q / Z blocks
  const int jr = j0 - ZRK_HR + rr;
  const bool row_on = lane_on && jr >= 0 && jr < Nr;
  const double t0 = cTG[4][0], t1 = cTG[4][1], t2 = cTG[4][2], t3 = cTG[4][3], t4 = cTG[4][4];
  const double t5 = cTG[4][5], t6 = cTG[4][6], t7 = cTG[4][7], t8 = cTG[4][8];
  double ring[16];  // filtered values, ring[p & 15] at position p
#pragma unroll
  for (int k = 0; k < 16; ++k) ring[k] = 0.0;
  uint32_t par = 0;  // bit s: parity of the next wait on slot s
  for (int k = bs; k <= be; ++k) {
    const int sl = k & 1;
    const bool ok = mbar_wait_bounded(&bar[sl], (par >> sl) & 1u);
    par ^= 1u << sl;
    if (!__syncthreads_and(ok)) {
      if (tid == 0) atomicOr(a.flags, 4);
      mbar_drain(&bar[sl], ((par >> sl) & 1u) ^ 1u);
      return;
    }
    const int m = k - 1;  // the block filtered in this iteration
    unsigned char* zb = base + SM::oZ;
    const bool work = k > bs && row_on;
    double xv[26];  // Q at positions 16m .. 16m + 25
    uint32_t cws[4];
    if (work) {
      const unsigned char* qm = base + SM::oQ + (sl ^ 1) * SM::qslot;
      const unsigned char* qk = base + SM::oQ + sl * SM::qslot;
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const double2 v = *reinterpret_cast<const double2*>(qm + zrk_chunk(Rq, c));
        xv[2 * c] = v.x;
        xv[2 * c + 1] = v.y;
      }
#pragma unroll
      for (int c = 0; c < 5; ++c) {
        const double2 v = *reinterpret_cast<const double2*>(qk + zrk_chunk(Rq, c));
        xv[16 + 2 * c] = v.x;
        xv[16 + 2 * c + 1] = v.y;
      }
      const uint4 cw = *reinterpret_cast<const uint4*>(base + SM::oZc + (sl ^ 1) * 1024 + rr * ZRK_BZ);
      cws[0] = cw.x;
      cws[1] = cw.y;
      cws[2] = cw.z;
      cws[3] = cw.w;
    }
    // block k-1's slot is free (its T and r codes were used in iteration k-1): block k+1
    __syncthreads();
    if (tid == 0 && k + 1 <= be) {
      // the slot's previous contents were read through the generic proxy
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(k + 1);
    }
    if (k > bs && lane_on) {
      // a block of centred points inside the row (the common case) needs no per-step checks
      const bool centred = row_on && cws[0] == 0x04040404u && cws[1] == 0x04040404u && cws[2] == 0x04040404u &&
                           cws[3] == 0x04040404u && ZRK_BZ * m + ZRK_BZ <= Nz;
      if (centred) {
#pragma unroll
        for (int s2 = 0; s2 < 16; ++s2) {
          const double ff = t4 * xv[s2] + t5 * xv[s2 + 1] + t6 * xv[s2 + 2] + t7 * xv[s2 + 3] + t8 * xv[s2 + 4];
          const double fb = t0 * ring[(s2 + 12) & 15] + t1 * ring[(s2 + 13) & 15] + t2 * ring[(s2 + 14) & 15];
          ring[s2] = (ff + fb) + t3 * ring[(s2 + 15) & 15];
        }
        double* zt = reinterpret_cast<double*>(zb) + fq * ZRK_BZ * ZRK_ZP + rr;
#pragma unroll
        for (int s2 = 0; s2 < 16; ++s2) zt[s2 * ZRK_ZP] = ring[s2];
      } else if (row_on) {
#pragma unroll
        for (int s2 = 0; s2 < 16; ++s2) {
          const int p = ZRK_BZ * m + s2;  // z position of this step
          const int code = (int)((cws[s2 >> 2] >> (8 * (s2 & 3))) & 255u);
          double v;
          if (p >= Nz) {
            v = 0.0;  // past the row: never stored, feeds only later positions past the row
          } else if (code == 4) {
            // feed-forward and older feedback terms first, the newest filtered value last:
            // one FMA of latency per step (the reference sums left to right; the orders
            // differ by rounding only)
            const double ff = t4 * xv[s2] + t5 * xv[s2 + 1] + t6 * xv[s2 + 2] + t7 * xv[s2 + 3] + t8 * xv[s2 + 4];
            const double fb = t0 * ring[(s2 + 12) & 15] + t1 * ring[(s2 + 13) & 15] + t2 * ring[(s2 + 14) & 15];
            v = (ff + fb) + t3 * ring[(s2 + 15) & 15];
          } else {
            // closure rows and blanked points: the padded 21-tap row, left to right
            const double* w = wt + (code < 9 ? code : 9) * 21;
            double acc = w[0] * ring[(s2 + 6) & 15];
#pragma unroll
            for (int o = -9; o < 0; ++o) acc = acc + w[10 + o] * ring[(s2 + 16 + o) & 15];
#pragma unroll
            for (int o = 0; o <= 10; ++o) acc = acc + w[10 + o] * xv[s2 + o];
            v = acc;
          }
          ring[s2] = v;
        }
        double* zt = reinterpret_cast<double*>(zb) + fq * ZRK_BZ * ZRK_ZP + rr;
#pragma unroll
        for (int s2 = 0; s2 < 16; ++s2) zt[s2 * ZRK_ZP] = ring[s2];
      } else {
        double* zt = reinterpret_cast<double*>(zb) + fq * ZRK_BZ * ZRK_ZP + rr;
#pragma unroll
        for (int s2 = 0; s2 < 16; ++s2) zt[s2 * ZRK_ZP] = 0.0;
      }
    }
    __syncthreads();
    if (k > bs && ZRK_BZ * m + ZRK_BZ > zs) {
      // r filter, scaling and coefficients of block m on the CTA's rows
      const SIN* tb = reinterpret_cast<const SIN*>(base + SM::oT + sl * ((SM::tbytes + 127) / 128 * 128));
      const unsigned char* rcb = base + SM::oRc + sl * 512;
      // the points of a thread are independent: unrolled so their T**0.666 and filter
      // chains interleave
#pragma unroll
      for (int u = 0; u < (ZRK_RB * ZRK_BZ + ZRK_THREADS - 1) / ZRK_THREADS; ++u) {
        const int qd = tid + u * ZRK_THREADS;
        const int row = qd / ZRK_BZ, p = qd - row * ZRK_BZ;
        const int j = j0 + row, i = ZRK_BZ * m + p;
        if (qd >= ZRK_RB * ZRK_BZ || j >= Nr || i < zs || i >= ze) continue;
        const double mu = double(mu_k<R>(R(tb[qd])));
        const int rw = rcb[qd];
        double fv[3] = {0.0, 0.0, 0.0};
        // column of this point in the transposed block: row j0 + row is Z row row + ZRK_HR
        const double* zc = reinterpret_cast<const double*>(zb) + p * ZRK_ZP + row + ZRK_HR;
        if (rw == 4) {
#pragma unroll
          for (int f = 0; f < 3; ++f) {
            const double* col = zc + f * ZRK_BZ * ZRK_ZP - 4;
            double sacc = t0 * col[0];
#pragma unroll
            for (int mm = 1; mm < 9; ++mm) sacc = sacc + cTG[4][mm] * col[mm];
            fv[f] = sacc;
          }
        } else if (rw < 9) {
          const int w0 = tg_w0(rw), n = tg_len(rw);
#pragma unroll
          for (int f = 0; f < 3; ++f) {
            const double* col = zc + f * ZRK_BZ * ZRK_ZP + w0;
            double sacc = cTG[rw][0] * col[0];
            for (int mm = 1; mm < n; ++mm) sacc = sacc + cTG[rw][mm] * col[mm];
            fv[f] = sacc;
          }
        }
        const double ramp = __ldg(a.ramp + i);
        const long long o = (long long)j * P + i;
        a.coef[o] = mu + a.c.C_mu_Re * fv[0] * ramp;
        a.coef[PL + o] = (3.0 / 5.0) * mu + a.c.C_beta_Re * fv[1] * ramp;
        a.coef[2 * PL + o] = mu + a.c.C_kappa_Re_Pr * fv[2] * ramp;
      }
    }
    __syncthreads();
  }
}

template <typename SIN, typename R>
__global__ void __launch_bounds__(ZRK_THREADS, 3)
    zr_kernel(const ZrArgs a, const __grid_constant__ CUtensorMap mQ, const __grid_constant__ CUtensorMap mZc,
              const __grid_constant__ CUtensorMap mRc, const __grid_constant__ CUtensorMap mT) {
  extern __shared__ __align__(128) unsigned char zrk_raw[];
  __shared__ __align__(8) uint64_t bar[2];
  zr_body<SIN, R>(a, &mQ, &mZc, &mRc, &mT, blockIdx.x, blockIdx.y, zrk_raw, bar);
}

// Batched: one CTA per entry (segment, row block, instance) of a table over all instances;
// each instance's arguments (staged in shared memory) and maps come from device tables.
template <typename SIN, typename R>
__global__ void __launch_bounds__(ZRK_THREADS, 3)
    zr_kernel_batch(const ZrArgs* __restrict__ argv, const int4* __restrict__ items, const CUtensorMap* __restrict__ mapv,
                    int nmaps, int4 kmaps) {
  extern __shared__ __align__(128) unsigned char zrk_raw[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ __align__(16) ZrArgs sa;
  const int4 it = items[blockIdx.x];
  for (int k = threadIdx.x; k < (int)(sizeof(ZrArgs) / 8); k += blockDim.x)
    reinterpret_cast<unsigned long long*>(&sa)[k] = reinterpret_cast<const unsigned long long*>(argv + it.z)[k];
  __syncthreads();
  const CUtensorMap* m = mapv + (size_t)it.z * nmaps;
  zr_body<SIN, R>(sa, m + kmaps.x, m + kmaps.y, m + kmaps.z, m + kmaps.w, it.x, it.y, zrk_raw, bar);
}

template <typename SIN, typename R>
static cudaError_t launch_zr_t(const ZrArgs& a, const ZrMaps& m, cudaStream_t s) {
  const dim3 grid((a.g.Nz + a.seg - 1) / a.seg, (a.g.Nr + ZRK_RB - 1) / ZRK_RB);
  zr_kernel<SIN, R><<<grid, ZRK_THREADS, ZrSmem<SIN>::bytes, s>>>(a, *m.q, *m.zc, *m.rc, *m.t);
  return cudaGetLastError();
}

static_assert(sizeof(ZrArgs) % 8 == 0, "ZrArgs is staged in 8-byte words");

template <typename SIN, typename R>
static cudaError_t launch_zr_batch_t(const ZrArgs* argv, const int4* items, int nitems, const CUtensorMap* mapv,
                                     int kin, cudaStream_t s) {
  const int4 k = make_int4(bmap_zrQ, bmap_zrZc, bmap_zrRc, bmap_zrT(kin));
  zr_kernel_batch<SIN, R><<<nitems, ZRK_THREADS, ZrSmem<SIN>::bytes, s>>>(argv, items, mapv, NM_BATCH, k);
  return cudaGetLastError();
}

cudaError_t launch_zr_batch(const ZrArgs* argv, const int4* items, int nitems, const CUtensorMap* mapv, int kin,
                            bool mixed, bool in_f32, cudaStream_t s) {
  if (nitems <= 0) return cudaSuccess;
  if (!mixed) return launch_zr_batch_t<double, double>(argv, items, nitems, mapv, kin, s);
  if (!in_f32) return launch_zr_batch_t<double, float>(argv, items, nitems, mapv, kin, s);
  return launch_zr_batch_t<float, float>(argv, items, nitems, mapv, kin, s);
}

cudaError_t launch_zr(const ZrArgs& a, const ZrMaps& m, bool mixed, bool in_f32, cudaStream_t s) {
  if (!mixed) return launch_zr_t<double, double>(a, m, s);
  if (!in_f32) return launch_zr_t<double, float>(a, m, s);
  return launch_zr_t<float, float>(a, m, s);
}

cudaError_t launch_sensor_tiles_only(const SensorArgs& a, const SideStream& side, cudaStream_t s) {
  cudaError_t e = fork(side, s);
  if (e != cudaSuccess) return e;
  if (!a.mixed) launch_sensor_tiles<double, double>(a, side, s);
  else if (!a.in_f32) launch_sensor_tiles<double, float>(a, side, s);
  else launch_sensor_tiles<float, float>(a, side, s);
  e = join(side, s);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

static int zr_threads(int Nz) {
  const int nchunk = (Nz + ZR_L - 1) / ZR_L;
  return std::min(1024, (nchunk + 31) / 32 * 32);
}
static size_t zr_smem_bytes(int Nz, long long P, int bs) {
  (void)bs;
  return (zr_off_flags(Nz, P) + ZR_MAXCHUNK + 15) & ~(size_t)15;
}
static size_t zr_smem_bytes(int Nz, long long P) { return zr_smem_bytes(Nz, P, zr_threads(Nz)); }

cudaError_t launch_tgfilter_z_inplace(const Grid& g, const uint32_t* desc, const unsigned char* zcode, const double* q,
                                      double* out, int nfield, int* flags, cudaStream_t s) {
  if (g.Nz <= ZR_MAXNZ) {
    const int nchunk = (g.Nz + ZR_L - 1) / ZR_L;
    const int bs = std::min(1024, (nchunk + 31) / 32 * 32);
    tgfilter_z_rows_kernel<<<dim3(g.Nr, nfield), bs, zr_smem_bytes(g.Nz, g.P), s>>>(g, zcode, q, out, flags);
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

void sensor_boxes(bool gen, bool mixed, int* vw, int* vh, int* tw, int* th) {
  using GD = SensSmem<SENS_HS_GEN, H_GEN, double, double>;
  using ID = SensSmem<SENS_HS_INT, H_INT, double, double>;
  using GF = SensSmem<SENS_HS_GEN, H_GEN, float, float>;
  using IF = SensSmem<SENS_HS_INT, H_INT, float, float>;
  if (mixed) {
    *vw = gen ? GF::VZ : IF::VZ;
    *vh = gen ? GF::VR : IF::VR;
    *tw = gen ? GF::SZ : IF::SZ;
    *th = gen ? GF::SR : IF::SR;
  } else {
    *vw = gen ? GD::VZ : ID::VZ;
    *vh = gen ? GD::VR : ID::VR;
    *tw = gen ? GD::SZ : ID::SZ;
    *th = gen ? GD::SR : ID::SR;
  }
}

template <int H, bool GEN, typename SIN, typename R, int TRT = TR>
static cudaError_t stage_attr() {
  cudaError_t e = cudaFuncSetAttribute(stage_kernel<H, GEN, SIN, R, CM_FILT, TRT>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)StageSmem<H, SIN, R, CM_FILT, TRT>::bytes(GEN));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(stage_kernel<H, GEN, SIN, R, CM_PRE, TRT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)StageSmem<H, SIN, R, CM_PRE, TRT>::bytes(GEN));
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(stage_kernel<H, GEN, SIN, R, CM_LRN, TRT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)StageSmem<H, SIN, R, CM_LRN, TRT>::bytes(GEN));
}
template <int HS, int HF, bool GEN, typename SIN, typename R>
static cudaError_t sensor_attr() {
  return cudaFuncSetAttribute(sensor_tile_kernel<HS, HF, GEN, SIN, R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)SensSmem<HS, HF, SIN, R>::bytes(GEN));
}
template <int H, bool GEN, typename SIN, typename R, int TRT = TR>
static cudaError_t stage_batch_attr() {
  cudaError_t e = cudaFuncSetAttribute(stage_kernel_batch<H, GEN, SIN, R, CM_FILT, TRT>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)StageSmem<H, SIN, R, CM_FILT, TRT>::bytes(GEN));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(stage_kernel_batch<H, GEN, SIN, R, CM_PRE, TRT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)StageSmem<H, SIN, R, CM_PRE, TRT>::bytes(GEN));
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(stage_kernel_batch<H, GEN, SIN, R, CM_LRN, TRT>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)StageSmem<H, SIN, R, CM_LRN, TRT>::bytes(GEN));
}
template <int HS, int HF, bool GEN, typename SIN, typename R>
static cudaError_t sensor_batch_attr() {
  return cudaFuncSetAttribute(sensor_tile_kernel_batch<HS, HF, GEN, SIN, R>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SensSmem<HS, HF, SIN, R>::bytes(GEN));
}
template <typename SIN, typename R>
static cudaError_t pair_attrs() {
  cudaError_t e = stage_batch_attr<H_GEN, true, SIN, R>();
  if (e == cudaSuccess) e = stage_batch_attr<H_INT, false, SIN, R>();
  if (e == cudaSuccess) e = stage_batch_attr<H_INT, false, SIN, R, TR / 2>();
  if (e == cudaSuccess) e = sensor_batch_attr<SENS_HS_GEN, H_GEN, true, SIN, R>();
  if (e == cudaSuccess) e = sensor_batch_attr<SENS_HS_INT, H_INT, false, SIN, R>();
  if (e != cudaSuccess) return e;
  e = stage_attr<H_GEN, true, SIN, R>();
  if (e == cudaSuccess) e = stage_attr<H_INT, false, SIN, R>();
  if (e == cudaSuccess) e = stage_attr<H_INT, false, SIN, R, TR / 2>();
  if (e == cudaSuccess) e = sensor_attr<SENS_HS_GEN, H_GEN, true, SIN, R>();
  if (e == cudaSuccess) e = sensor_attr<SENS_HS_INT, H_INT, false, SIN, R>();
  return e;
}

// Poll limit of the bounded waits of this file's kernels on the current device (tries < 0:
// the default; 0: every wait gives up at once). Kernels read it when they run, so captured
// graphs see a change too.
cudaError_t set_wait_tries(int tries) {
  const int v = tries >= 0 ? tries : kWaitTriesDefault;
  return cudaMemcpyToSymbol(c_wait_tries, &v, sizeof(int));
}

// Opt-in shared-memory sizes; called once per handle at creation (outside any
// stream capture).
cudaError_t init_kernel_attributes() {
  cudaError_t e = pair_attrs<double, double>();
  if (e == cudaSuccess) e = pair_attrs<double, float>();
  if (e == cudaSuccess) e = pair_attrs<float, float>();
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(tgfilter_z_rows_kernel_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)zr_smem_bytes(ZR_MAXNZ, ZR_MAXNZ + 32, 1024));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(zr_kernel<double, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)ZrSmem<double>::bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(zr_kernel_batch<double, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)ZrSmem<double>::bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(zr_kernel_batch<double, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)ZrSmem<double>::bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(zr_kernel_batch<float, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)ZrSmem<float>::bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(zr_kernel<double, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)ZrSmem<double>::bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(zr_kernel<float, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)ZrSmem<float>::bytes);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(tgfilter_z_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)zr_smem_bytes(ZR_MAXNZ, ZR_MAXNZ + 32));
}

// ---------------------------------------------------------------------------
// Batched launches
// ---------------------------------------------------------------------------
size_t zrows_smem(int Nz, long long P, int bs) { return zr_smem_bytes(Nz, P, bs); }
int zrows_threads(int Nz) { return zr_threads(Nz); }

template <int H, bool GEN, typename SIN, typename R, int CM, int TRT = TR>
static cudaError_t launch_stage_batch_t(const StageArgs* argv, const BatchTiles& t, const CUtensorMap* mapv, int kin,
                                        cudaStream_t s) {
  if (t.ntiles <= 0) return cudaSuccess;
  const int cls = GEN ? 1 : 0;
  int4 k;
  if (TRT == TR) {
    const int star = CM == CM_PRE ? bmap_coef(cls) : bmap_star(cls, CM == CM_LRN);
    k = make_int4(bmap_state(kin, cls), star, 14, 15);
  } else {
    const int star = CM == CM_PRE ? bmap_coef(2) : bmap_starH(CM == CM_LRN);
    k = make_int4(bmap_stateH(kin), star, bmap_u0H, bmap_accH);
  }
  const size_t sm = StageSmem<H, SIN, R, CM, TRT>::bytes(GEN);
  stage_kernel_batch<H, GEN, SIN, R, CM, TRT>
      <<<t.grid, stage_threads(TRT), sm, s>>>(argv, t.tiles, t.ntiles, mapv, NM_BATCH, k);
  return cudaGetLastError();
}

template <typename SIN, typename R, int CM>
static cudaError_t launch_stage_batch_pair(const StageArgs* argv, const BatchTiles& tint, const BatchTiles& tgen,
                                           const CUtensorMap* mapv, int kin, const SideStream& side, cudaStream_t s,
                                           int int_rows) {
  cudaError_t e = fork(side, s);
  if (e != cudaSuccess) return e;
  e = launch_stage_batch_t<H_GEN, true, SIN, R, CM>(argv, tgen, mapv, kin, side.stream ? side.stream : s);
  if (e != cudaSuccess) return e;
  e = int_rows == TR / 2 ? launch_stage_batch_t<H_INT, false, SIN, R, CM, TR / 2>(argv, tint, mapv, kin, s)
                         : launch_stage_batch_t<H_INT, false, SIN, R, CM>(argv, tint, mapv, kin, s);
  if (e != cudaSuccess) return e;
  return join(side, s);
}

template <typename SIN, typename R>
static cudaError_t launch_stage_batch_cm(const StageArgs* argv, int cm, const BatchTiles& tint, const BatchTiles& tgen,
                                         const CUtensorMap* mapv, int kin, const SideStream& side, cudaStream_t s,
                                         int int_rows) {
  if (cm == CM_LRN) return launch_stage_batch_pair<SIN, R, CM_LRN>(argv, tint, tgen, mapv, kin, side, s, int_rows);
  if (cm == CM_PRE) return launch_stage_batch_pair<SIN, R, CM_PRE>(argv, tint, tgen, mapv, kin, side, s, int_rows);
  return launch_stage_batch_pair<SIN, R, CM_FILT>(argv, tint, tgen, mapv, kin, side, s, int_rows);
}

cudaError_t launch_stage_batch(const StageArgs* argv, const StageArgs& a0, const BatchTiles& tint, const BatchTiles& tgen,
                               const CUtensorMap* mapv, int kin, const SideStream& side, cudaStream_t s, int int_rows) {
  if (!a0.mixed) return launch_stage_batch_cm<double, double>(argv, a0.learned, tint, tgen, mapv, kin, side, s, int_rows);
  if (!a0.in_f32) return launch_stage_batch_cm<double, float>(argv, a0.learned, tint, tgen, mapv, kin, side, s, int_rows);
  return launch_stage_batch_cm<float, float>(argv, a0.learned, tint, tgen, mapv, kin, side, s, int_rows);
}

template <typename SIN, typename R>
static void launch_sensor_tiles_batch(const SensorArgs* argv, const BatchTiles& tint, const BatchTiles& tgen,
                                      const CUtensorMap* mapv, int kin, const SideStream& side, cudaStream_t s) {
  using SG = SensSmem<SENS_HS_GEN, H_GEN, SIN, R>;
  using SI = SensSmem<SENS_HS_INT, H_INT, SIN, R>;
  if (tgen.ntiles > 0)
    sensor_tile_kernel_batch<SENS_HS_GEN, H_GEN, true, SIN, R>
        <<<tgen.grid, sens_threads(true), SG::bytes(true), side.stream ? side.stream : s>>>(
            argv, tgen.tiles, tgen.ntiles, mapv, NM_BATCH, make_int4(bmap_sens(kin, 1), bmap_sensT(kin, 1), 0, 0));
  if (tint.ntiles > 0)
    sensor_tile_kernel_batch<SENS_HS_INT, H_INT, false, SIN, R><<<tint.grid, sens_threads(false), SI::bytes(false), s>>>(
        argv, tint.tiles, tint.ntiles, mapv, NM_BATCH, make_int4(bmap_sens(kin, 0), bmap_sensT(kin, 0), 0, 0));
}

cudaError_t launch_sensor_batch(const SensorArgs* argv, const SensorArgs& a0, const BatchTiles& tint,
                                const BatchTiles& tgen, const CUtensorMap* mapv, int kin, const int2* zrows,
                                int nzrows, int zthreads, size_t zsmem, bool rfilter, int ninst, long long max_pts,
                                const SideStream& side, cudaStream_t s) {
  cudaError_t e = fork(side, s);
  if (e != cudaSuccess) return e;
  if (!a0.mixed) launch_sensor_tiles_batch<double, double>(argv, tint, tgen, mapv, kin, side, s);
  else if (!a0.in_f32) launch_sensor_tiles_batch<double, float>(argv, tint, tgen, mapv, kin, side, s);
  else launch_sensor_tiles_batch<float, float>(argv, tint, tgen, mapv, kin, side, s);
  e = join(side, s);
  if (e != cudaSuccess) return e;
  if (nzrows > 0) tgfilter_z_rows_kernel_batch<<<dim3(nzrows, 3), zthreads, zsmem, s>>>(argv, zrows);
  if (rfilter) {
    const int bs = 256;
    sensor_rfilter_kernel_batch<<<dim3((unsigned)((max_pts + bs - 1) / bs), ninst), bs, 0, s>>>(argv);
  }
  return cudaGetLastError();
}

cudaError_t launch_dt_batch(const DtArgs* argv, int ninst, int nblocks, cudaStream_t s) {
  dt_kernel_batch<<<dim3(nblocks, ninst), DT_THREADS, 0, s>>>(argv);
  return cudaGetLastError();
}

__global__ void harmonic_phase_kernel_batch(const HarmArgs* argv) {
  const HarmArgs a = argv[blockIdx.x];
  const int s = threadIdx.x;
  if (s < 1 || s > 4) return;
  const double tend = *a.time, d = *a.dt;
  const double cs = s == 1 ? 0.0 : (s == 4 ? 1.0 : 0.5);
  a.out[s] = cos(a.omega * ((tend - d) + cs * d));
}

cudaError_t launch_harmonic_phase_batch(const HarmArgs* argv, int ninst, cudaStream_t s) {
  harmonic_phase_kernel_batch<<<ninst, 32, 0, s>>>(argv);
  return cudaGetLastError();
}

}  // namespace axj
