// axj_api.cu -- the extern "C" boundary of libaxj.so (declared in include/axj.h):
// handle lifetime, set-up of the stencil maps, face lists, tile classes and 1-D
// metrics, host<->device copies, and the step sequence (plain calls or a CUDA graph).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/axj.h"
#include "axj_common.cuh"
#include "axj_prep.cuh"
#include "axj_kernels.cuh"
#include "axj_mlp.cuh"
#include "axj_pow.cuh"

using namespace axj;

namespace {

std::string g_create_error;

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

}  // namespace

struct axj_handle {
  int device = 0;
  int Nz = 0, Nr = 0;
  long long P = 0, plane = 0;
  axj_params params{};
  Consts c{};
  cudaStream_t stream = nullptr;
  SideStream side{nullptr, nullptr, nullptr};  // general-tile launches run here, joined back
  std::string err;
  std::vector<void*> allocs;
  // state and RK4 work buffers (5 planes each)
  double *U0 = nullptr, *Ua = nullptr, *Ub = nullptr, *A = nullptr, *B = nullptr, *target = nullptr;
  // mixed precision: the intermediate stage states as FP32 planes (pitch P) in the
  // memory of Ua / Ub, which the unit entry points use as FP64 scratch
  float *Uaf = nullptr, *Ubf = nullptr;
  bool mixed = false;
  // shock-capturing buffers
  double *Q = nullptr, *Qz = nullptr, *star = nullptr;
  double* coef = nullptr;            // mu_eff, beta, kappa_eff of the stage input (fused z/r filter)
  unsigned char* rcode = nullptr;    // r stencil code per point (9 = blanked)
  int2 *stiles_int = nullptr, *stiles_gen = nullptr;  // sensor tile classes
  int nstiles_int = 0, nstiles_gen = 0;
  uint32_t* desc = nullptr;
  unsigned char* zcode = nullptr;  // z stencil code per point for the z filter (9 = blanked)
  int* faces = nullptr;
  double *dxidz = nullptr, *ddxidxidz = nullptr, *detadr = nullptr, *ddetadetadr = nullptr;
  double* invr = nullptr;  // 1/r_j (0 on the axis row)
  double *zc = nullptr, *rc = nullptr, *dzv = nullptr, *drv = nullptr, *ramp = nullptr, *forcing = nullptr;
  double *dt = nullptr, *staleT = nullptr, *partial = nullptr, *time = nullptr;
  double* harm = nullptr;  // cos(omega t_s) of the harmonic forcing per stage
  int* flags = nullptr;
  unsigned int* counter = nullptr;
  int2 *tiles_int = nullptr, *tiles_gen = nullptr;
  int ntiles_int = 0, ntiles_gen = 0;
  int dt_blocks = 0;
  int iT = 0, jT = 0;
  int64_t iteration = 0;
  double time_host = 0.0;
  double time_end = 0.0;  // staging for the device time upload of axj_rk4_step
  bool state_set = false;
  cudaGraphExec_t graph_exec = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_judge_exec = nullptr;  // learned sensor: the judge step
  // RK4 alone (dt from the host: axj_rk4_step), plain and judge step
  cudaGraphExec_t graph_rk4_exec[2] = {nullptr, nullptr};
  cudaGraph_t graph_rk4[2] = {nullptr, nullptr};
  cudaGraph_t graph_judge = nullptr;
  // learned sensor
  double S1[9][6];              // SBP first-derivative rows (feature stencils)
  bool learned = false;         // learned sensor (or its held-coefficient baseline)
  bool held_only = false;       // AXJ_SENSOR_HELD: no network between judge steps
  bool judged = false;          // a judge step has run since the state or the model changed
  int64_t judge_every = 50;
  bool judge_all = true;        // a judge step runs the plain sensor on all four stages
  double judge_thr = 0.1;
  float* mlp = nullptr;         // flat FP32 parameters (MLP_NPARAM)
  MlpNorm norm{};
  bool mlp_set = false;
  float4* feat = nullptr;       // feature channels of the current stage input
  double* pred = nullptr;       // 2 planes: predictions at the judge
  double* held = nullptr;       // 2 planes: plain betastar, kappastar of the last judge
  unsigned char* mask = nullptr;
  unsigned long long* counts = nullptr;  // judged point-outputs, fallbacks
  int64_t njudges = 0;
  // training data set: features and plain targets of nsnap snapshots
  float4* ds_feat = nullptr;
  float2* ds_targ = nullptr;
  int64_t ds_cap = 0, ds_n = 0;
  // output of axj_run (the WriteOutput hook): a device snapshot of the state taken in
  // stream order, copied to pinned host memory on its own stream while the next steps
  // run, handed to the callback one output later (or at the end of the run)
  double* out_snap = nullptr;     // 5 planes (pitch P) + time + flags (device)
  double* out_host = nullptr;     // 5 * Nz * Nr + time + flags (pinned host)
  cudaStream_t out_stream = nullptr;
  cudaEvent_t out_snapped = nullptr, out_copied = nullptr;
  bool out_pending = false;
  int64_t out_iter = 0;
  // TMA descriptors: stage-input halo boxes for the stage buffers x {interior, general}
  // tiles, coefficient halo boxes, and tile boxes of pv_old and the running sum A
  CUtensorMap map_state[5][2];
  CUtensorMap map_star[2];
  CUtensorMap map_starL[2];    // final mu*, beta*, kappa* planes (learned sensor)
  CUtensorMap map_u0_tile, map_acc_tile, map_b_tile;
  CUtensorMap map_sens[5][2];  // sensor V boxes of the stage buffers x {interior, general}
  CUtensorMap map_sensT[5][2]; // sensor temperature boxes
  // fused z/r filter: Q blocks, z and r code blocks, temperature blocks of the stage
  // buffers; the coefficient planes it writes, as boxes of the two tile classes
  CUtensorMap map_zrQ, map_zrZc, map_zrRc, map_zrT[5];
  CUtensorMap map_coef[2];
  // interior tiles as two CTAs of TR / 2 rows (int_rows == TR / 2, or a batch tuned so):
  // their boxes
  int int_rows = TR;
  CUtensorMap map_stateH[5], map_starH, map_starLH, map_coefH, map_u0H, map_accH, map_bH;
  CUtensorMap map_tgt, map_tgtH;  // pv_target tile boxes (L2 prefetch of the sponge tiles)
};

namespace {
// Stage buffers by id: U0, Ua, Ub in FP64; Ua, Ub as FP32 planes (mixed path only).
enum { BU0 = 0, BUA = 1, BUB = 2, BUAF = 3, BUBF = 4, NBUF = 5 };
inline bool buf_f32(int b) { return b >= BUAF; }
inline void* buf_ptr(axj_handle* h, int b) {
  switch (b) {
    case BU0: return h->U0;
    case BUA: return h->Ua;
    case BUB: return h->Ub;
    case BUAF: return h->Uaf;
    default: return h->Ubf;
  }
}
}  // namespace

namespace {

int fail(axj_handle* h, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (h) h->err = buf;
  else g_create_error = buf;
  return code;
}

#define AXJ_CUDA(h, call)                                                                                 \
  do {                                                                                                    \
    cudaError_t e_ = (call);                                                                              \
    if (e_ != cudaSuccess) return fail((h), AXJ_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

// SBP_operator (ModOperator.f90:5-121). The truncated-Gaussian boundary rows are
// default-kind (single-precision) literals in the reference, so they are rounded
// to float before widening, exactly as the Fortran assignment does.
void build_tables(double S1[9][6], double S2[9][6], double G[9][11]) {
  std::memset(S1, 0, sizeof(double) * 54);
  std::memset(S2, 0, sizeof(double) * 54);
  std::memset(G, 0, sizeof(double) * 99);
  const double s1[4][6] = {{-24.0 / 17.0, 59.0 / 34.0, -4.0 / 17.0, -3.0 / 34.0, 0.0, 0.0},
                           {-1.0 / 2.0, 0.0, 1.0 / 2.0, 0.0, 0.0, 0.0},
                           {4.0 / 43.0, -59.0 / 86.0, 0.0, 59.0 / 86.0, -4.0 / 43.0, 0.0},
                           {3.0 / 98.0, 0.0, -59.0 / 98.0, 0.0, 32.0 / 49.0, -4.0 / 49.0}};
  const double s2[4][6] = {{2.0, -5.0, 4.0, -1.0, 0.0, 0.0},
                           {1.0, -2.0, 1.0, 0.0, 0.0, 0.0},
                           {-4.0 / 43.0, 59.0 / 43.0, -110.0 / 43.0, 59.0 / 43.0, -4.0 / 43.0, 0.0},
                           {-1.0 / 49.0, 0.0, 59.0 / 49.0, -118.0 / 49.0, 64.0 / 49.0, -4.0 / 49.0}};
  for (int r = 0; r < 4; ++r)
    for (int m = 0; m < 6; ++m) {
      S1[r][m] = s1[r][m];
      S2[r][m] = s2[r][m];
      S1[8 - r][5 - m] = -1.0 * s1[r][m];  // bottom block = -mirror (:32-38)
      S2[8 - r][5 - m] = 1.0 * s2[r][m];   // bottom block = +mirror (:68-74)
    }
  const double i1[5] = {1.0 / 12.0, -2.0 / 3.0, 0.0, 2.0 / 3.0, -1.0 / 12.0};
  const double i2[5] = {-1.0 / 12.0, 4.0 / 3.0, -5.0 / 2.0, 4.0 / 3.0, -1.0 / 12.0};
  for (int m = 0; m < 5; ++m) { S1[4][m] = i1[m]; S2[4][m] = i2[m]; }
  const float g1[7] = {0.085777408970000f, 0.722371828476000f, 0.356848072173000f, -0.223119093072000f,
                       0.057347064865000f, 0.000747264596000f, 0.000027453993000f};
  const float g2[7] = {-0.032649010764000f, 0.143339502575000f, 0.726678822020000f, 0.294622121167000f,
                       -0.186711738069000f, 0.062038376258000f, -0.007318073189000f};
  const float g3[11] = {0.000054596010000f, -0.042124772446000f, 0.173103107841000f, 0.700384128648000f,
                        0.276543612935000f, -0.131223506571000f, 0.023424966418000f, -0.013937561779000f,
                        0.024565095706000f, -0.013098287852000f, 0.002308621090000f};
  G[0][0] = 1.0;
  for (int m = 0; m < 7; ++m) { G[1][m] = (double)g1[m]; G[2][m] = (double)g2[m]; }
  for (int m = 0; m < 11; ++m) G[3][m] = (double)g3[m];
  for (int r = 0; r < 4; ++r)
    for (int m = 0; m < 11; ++m) G[8 - r][10 - m] = 1.0 * G[r][m];
  const double gi[9] = {107.0 / 103680.0, 149.0 / 12960.0, 1997.0 / 25920.0, 3091.0 / 12960.0, 3565.0 / 10368.0,
                        3091.0 / 12960.0, 1997.0 / 25920.0, 149.0 / 12960.0, 107.0 / 103680.0};
  for (int m = 0; m < 9; ++m) G[4][m] = gi[m];
}

// ComputeMetric (ModDeriv.f90:241-382) on a 1-D coordinate line with closures at
// both ends (single block: every neighbour is MPI_PROC_NULL). Sums start from 0.
void metric_1d(const double S1[9][6], const std::vector<double>& v, std::vector<double>& out) {
  const int n = (int)v.size();
  out.assign(n, 0.0);
  for (int i = 5; i <= n - 4; ++i) {
    double s = 0.0;
    for (int m = 0; m < 5; ++m) s = s + S1[4][m] * v[i - 2 + m - 1];
    out[i - 1] = s;
  }
  for (int i = 1; i <= 4; ++i) {
    double s = 0.0;
    for (int m = 0; m < 6; ++m) s = s + S1[i - 1][m] * v[m];
    out[i - 1] = s;
  }
  for (int i = n - 3; i <= n; ++i) {
    double s = 0.0;
    for (int m = 0; m < 6; ++m) s = s + S1[8 - n + i][m] * v[n - 6 + m];
    out[i - 1] = s;
  }
}

template <class T>
T* dalloc(axj_handle* h, size_t count, int* rc) {
  void* p = nullptr;
  if (*rc != AXJ_OK) return nullptr;
  cudaError_t e = cudaMalloc(&p, count * sizeof(T) + 16);
  if (e != cudaSuccess) {
    *rc = fail(h, AXJ_ERR_NOMEM, "cudaMalloc(%zu) failed: %s", count * sizeof(T), cudaGetErrorString(e));
    return nullptr;
  }
  cudaMemset(p, 0, count * sizeof(T) + 16);
  h->allocs.push_back(p);
  return static_cast<T*>(p);
}

Grid grid_of(const axj_handle* h) {
  Grid g;
  g.Nz = h->Nz;
  g.Nr = h->Nr;
  g.P = h->P;
  g.plane = h->plane;
  return g;
}

// host (Nz x Nr x nf, z fastest) <-> device (pitch P) copies
cudaError_t h2d(axj_handle* h, double* dst, const double* src, int nf) {
  return cudaMemcpy2DAsync(dst, (size_t)h->P * sizeof(double), src, (size_t)h->Nz * sizeof(double),
                           (size_t)h->Nz * sizeof(double), (size_t)h->Nr * nf, cudaMemcpyHostToDevice, h->stream);
}
cudaError_t d2h(axj_handle* h, double* dst, const double* src, int nf) {
  return cudaMemcpy2DAsync(dst, (size_t)h->Nz * sizeof(double), src, (size_t)h->P * sizeof(double),
                           (size_t)h->Nz * sizeof(double), (size_t)h->Nr * nf, cudaMemcpyDeviceToHost, h->stream);
}

SensorArgs sensor_args(axj_handle* h, int b) {
  SensorArgs s;
  s.g = grid_of(h);
  s.U = buf_f32(b) ? nullptr : static_cast<const double*>(buf_ptr(h, b));
  s.Uf = buf_f32(b) ? static_cast<const float*>(buf_ptr(h, b)) : nullptr;
  s.mv_int = &h->map_sens[b][0];
  s.mv_gen = &h->map_sens[b][1];
  s.mt_int = &h->map_sensT[b][0];
  s.mt_gen = &h->map_sensT[b][1];
  s.desc = h->desc;
  s.dxidz = h->dxidz;
  s.detadr = h->detadr;
  s.zc = h->zc;
  s.rc = h->rc;
  s.invr = h->invr;
  s.dz = h->dzv;
  s.dr = h->drv;
  s.ramp = h->ramp;
  s.tiles_int = h->stiles_int;
  s.tiles_gen = h->stiles_gen;
  s.ntiles_int = h->nstiles_int;
  s.ntiles_gen = h->nstiles_gen;
  s.zcode = h->zcode;
  s.flags = h->flags;
  s.Q = h->Q;
  s.Qz = h->Qz;
  s.star = h->star;
  s.mixed = h->mixed;
  s.in_f32 = buf_f32(b);
  s.ramp_off = 0;
  s.c = h->c;
  return s;
}

StageArgs stage_args(axj_handle* h, int bin, int bout, int stage) {
  StageArgs a;
  a.g = grid_of(h);
  a.Uin = buf_f32(bin) ? nullptr : static_cast<const double*>(buf_ptr(h, bin));
  a.U0 = h->U0;
  a.A = h->A;
  a.B = h->B;
  a.Uout = buf_f32(bout) ? nullptr : static_cast<double*>(buf_ptr(h, bout));
  a.Uout_f = buf_f32(bout) ? static_cast<float*>(buf_ptr(h, bout)) : nullptr;
  a.target = h->target;
  a.mustar = h->star;
  a.betastar = h->star + h->plane;
  a.kappastar = h->star + 2 * h->plane;
  a.desc = h->desc;
  a.faces = h->faces;
  a.tiles = nullptr;
  a.dxidz = h->dxidz;
  a.ddxidxidz = h->ddxidxidz;
  a.detadr = h->detadr;
  a.ddetadetadr = h->ddetadetadr;
  a.zc = h->zc;
  a.rc = h->rc;
  a.invr = h->invr;
  a.forcing = h->forcing;
  a.ramp = h->ramp;
  a.dt = h->dt;
  a.staleT = h->staleT;
  a.harm = h->harm;
  a.flags = h->flags;
  a.stage = stage;
  a.iT = h->iT;
  a.jT = h->jT;
  a.mixed = h->mixed;
  a.in_f32 = buf_f32(bin);
  a.out_f32 = buf_f32(bout);
  a.learned = 0;
  a.c = h->c;
  return a;
}

// cuTensorMapEncodeTiled, resolved from the driver at run time (no link-time libcuda).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// 3-D map over nplanes planes of (Nz, Nr) doubles (or floats) with pitch P;
// out-of-range elements of a box read as zero.
int make_map(axj_handle* h, CUtensorMap* m, const void* base, int nplanes, int bw, int bh, int bp, bool f32 = false) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return fail(h, AXJ_ERR_NODEVICE, "cuTensorMapEncodeTiled is not available from the driver");
  const size_t es_bytes = f32 ? sizeof(float) : sizeof(double);
  const cuuint64_t dims[3] = {(cuuint64_t)h->Nz, (cuuint64_t)h->Nr, (cuuint64_t)nplanes};
  const cuuint64_t strides[2] = {(cuuint64_t)h->P * es_bytes, (cuuint64_t)h->plane * es_bytes};
  const cuuint32_t box[3] = {(cuuint32_t)bw, (cuuint32_t)bh, (cuuint32_t)bp};
  const cuuint32_t es[3] = {1, 1, 1};
  CUresult r = fn(m, f32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
                  const_cast<void*>(base), dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(h, AXJ_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return AXJ_OK;
}

// 2-D map over an (Nz, Nr) byte array with pitch P (zero outside).
int make_map_u8(axj_handle* h, CUtensorMap* m, const void* base, int bw, int bh) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return fail(h, AXJ_ERR_NODEVICE, "cuTensorMapEncodeTiled is not available from the driver");
  const cuuint64_t dims[2] = {(cuuint64_t)h->Nz, (cuuint64_t)h->Nr};
  const cuuint64_t strides[1] = {(cuuint64_t)h->P};
  const cuuint32_t box[2] = {(cuuint32_t)bw, (cuuint32_t)bh};
  const cuuint32_t es[2] = {1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base), dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(h, AXJ_ERR_CUDA, "cuTensorMapEncodeTiled (u8) failed (%d)", (int)r);
  return AXJ_OK;
}

// The Q blocks of the fused z/r filter: 3 planes of doubles, box {ZRK_BZ, ZRK_NR, 3},
// written to shared memory with the 128-byte swizzle.
int make_map_zrq(axj_handle* h, CUtensorMap* m, const double* base) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return fail(h, AXJ_ERR_NODEVICE, "cuTensorMapEncodeTiled is not available from the driver");
  const cuuint64_t dims[3] = {(cuuint64_t)h->Nz, (cuuint64_t)h->Nr, 3};
  const cuuint64_t strides[2] = {(cuuint64_t)h->P * sizeof(double), (cuuint64_t)h->plane * sizeof(double)};
  const cuuint32_t box[3] = {(cuuint32_t)ZRK_BZ, (cuuint32_t)ZRK_NR, 3};
  const cuuint32_t es[3] = {1, 1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double*>(base), dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(h, AXJ_ERR_CUDA, "cuTensorMapEncodeTiled (Q blocks) failed (%d)", (int)r);
  return AXJ_OK;
}

int build_zr_maps(axj_handle* h) {
  const int nb = h->mixed ? NBUF : BUAF;
  int rc = make_map_zrq(h, &h->map_zrQ, h->Q);
  if (rc == AXJ_OK) rc = make_map_u8(h, &h->map_zrZc, h->zcode, ZRK_BZ, ZRK_NR);
  if (rc == AXJ_OK) rc = make_map_u8(h, &h->map_zrRc, h->rcode, ZRK_BZ, ZRK_RB);
  for (int b = 0; b < nb && rc == AXJ_OK; ++b)
    rc = make_map(h, &h->map_zrT[b], buf_ptr(h, b), 5, ZRK_BZ, ZRK_RB, 1, buf_f32(b));
  for (int cls = 0; cls < 2 && rc == AXJ_OK; ++cls) {
    int hw, hh, qh, tw, th, qlh;
    stage_boxes(cls == 1, h->mixed, &hw, &hh, &qh, &tw, &th, &qlh);
    rc = make_map(h, &h->map_coef[cls], h->coef, 3, hw, qlh, 3);
  }
  if (rc == AXJ_OK) {
    int hw, hh, qh, tw, th, qlh;
    stage_boxes(false, h->mixed, &hw, &hh, &qh, &tw, &th, &qlh, TR / 2);
    rc = make_map(h, &h->map_coefH, h->coef, 3, hw, qlh, 3);
  }
  return rc;
}

int build_maps(axj_handle* h) {
  const int nb = h->mixed ? NBUF : BUAF;
  for (int cls = 0; cls < 2; ++cls) {
    int hw, hh, qh, tw, th;
    int qlh;
    stage_boxes(cls == 1, h->mixed, &hw, &hh, &qh, &tw, &th, &qlh);
    for (int b = 0; b < nb; ++b) {
      int rc = make_map(h, &h->map_state[b][cls], buf_ptr(h, b), 5, hw, hh, 5, buf_f32(b));
      if (rc != AXJ_OK) return rc;
    }
    // z-filtered coefficient quantities (never loaded without shock capturing)
    int rc = make_map(h, &h->map_star[cls], h->Qz ? h->Qz : h->star, 3, hw, qh, 3);
    if (rc != AXJ_OK) return rc;
    rc = make_map(h, &h->map_starL[cls], h->star, 3, hw, qlh, 3);
    if (rc != AXJ_OK) return rc;
    int vw, vh, tw2, th2;
    sensor_boxes(cls == 1, h->mixed, &vw, &vh, &tw2, &th2);
    for (int b = 0; b < nb; ++b) {
      rc = make_map(h, &h->map_sens[b][cls], buf_ptr(h, b), 5, vw, vh, 1, buf_f32(b));
      if (rc != AXJ_OK) return rc;
      rc = make_map(h, &h->map_sensT[b][cls], buf_ptr(h, b), 5, tw2, th2, 1, buf_f32(b));
      if (rc != AXJ_OK) return rc;
    }
  }
  int hw, hh, qh, tw, th;
  stage_boxes(false, h->mixed, &hw, &hh, &qh, &tw, &th, nullptr);
  int rc = make_map(h, &h->map_u0_tile, h->U0, 5, tw, th, 5);
  if (rc != AXJ_OK) return rc;
  rc = make_map(h, &h->map_b_tile, h->B, 5, tw, th, 5);
  if (rc != AXJ_OK) return rc;
  rc = make_map(h, &h->map_acc_tile, h->A, 5, tw, th, 5);
  if (rc == AXJ_OK) rc = make_map(h, &h->map_tgt, h->target, 5, tw, th, 5);
  if (rc != AXJ_OK) return rc;
  // the half tiles of the interior class (a handle's int_rows, or a batch's tuning)
  int qlh;
  stage_boxes(false, h->mixed, &hw, &hh, &qh, &tw, &th, &qlh, TR / 2);
  for (int b = 0; b < nb && rc == AXJ_OK; ++b)
    rc = make_map(h, &h->map_stateH[b], buf_ptr(h, b), 5, hw, hh, 5, buf_f32(b));
  if (rc == AXJ_OK) rc = make_map(h, &h->map_starH, h->Qz ? h->Qz : h->star, 3, hw, qh, 3);
  if (rc == AXJ_OK) rc = make_map(h, &h->map_starLH, h->star, 3, hw, qlh, 3);
  if (rc == AXJ_OK) rc = make_map(h, &h->map_u0H, h->U0, 5, tw, th, 5);
  if (rc == AXJ_OK) rc = make_map(h, &h->map_bH, h->B, 5, tw, th, 5);
  if (rc == AXJ_OK) rc = make_map(h, &h->map_accH, h->A, 5, tw, th, 5);
  if (rc == AXJ_OK) rc = make_map(h, &h->map_tgtH, h->target, 5, tw, th, 5);
  return rc;
}

// cm: CM_FILT (z-filtered quantities, r filter in the stage kernel), CM_LRN (learned
// coefficient planes) or CM_PRE (mu_eff, beta, kappa_eff from the fused z/r filter).
StageMaps stage_maps(axj_handle* h, int b, int cls, int cm) {
  StageMaps m;
  if (cls == 0 && h->int_rows != TR) {
    m.state = &h->map_stateH[b];
    m.star = cm == CM_LRN ? &h->map_starLH : (cm == CM_PRE ? &h->map_coefH : &h->map_starH);
    m.u0 = &h->map_u0H;
    m.acc = &h->map_accH;
    m.bt = &h->map_bH;
    m.tg = &h->map_tgtH;
    return m;
  }
  m.state = &h->map_state[b][cls];
  m.star = cm == CM_LRN ? &h->map_starL[cls] : (cm == CM_PRE ? &h->map_coef[cls] : &h->map_star[cls]);
  m.u0 = &h->map_u0_tile;
  m.acc = &h->map_acc_tile;
  m.bt = &h->map_b_tile;
  m.tg = &h->map_tgt;
  return m;
}

int launch_stage_kernels(axj_handle* h, int bin, int bout, int stage, int cm) {
  StageArgs a = stage_args(h, bin, bout, stage);
  a.learned = cm;
  StageMaps mi = stage_maps(h, bin, 0, cm), mg = stage_maps(h, bin, 1, cm);
  AXJ_CUDA(h, launch_stage(a, h->ntiles_int, h->tiles_int, mi, h->ntiles_gen, h->tiles_gen, mg, h->side, h->stream,
                           h->int_rows));
  return AXJ_OK;
}

// The sensor chain of a stage input: the sensor tiles (quantities Q), then the fused
// z filter / r filter / coefficient kernel, which leaves mu_eff, beta, kappa_eff in coef.
ZrArgs zr_args(axj_handle* h, int seg) {
  ZrArgs z;
  std::memset(&z, 0, sizeof(z));
  z.g = grid_of(h);
  z.ramp = h->ramp;
  z.coef = h->coef;
  z.flags = h->flags;
  z.seg = seg;
  z.c = h->c;
  return z;
}

int enqueue_sensor_chain(axj_handle* h, int bin) {
  SensorArgs s = sensor_args(h, bin);
  AXJ_CUDA(h, launch_sensor_tiles_only(s, h->side, h->stream));
  // about three CTAs per SM: segments of a multiple of ZRK_BZ positions, at least 64
  const int nrb = (h->Nr + ZRK_RB - 1) / ZRK_RB;
  const int nseg = std::max(1, (3 * 148) / nrb);
  const int seg = (int)((h->Nz + nseg - 1) / nseg);
  ZrArgs z = zr_args(h, std::max(64, (seg + ZRK_BZ - 1) / ZRK_BZ * ZRK_BZ));
  ZrMaps m{&h->map_zrQ, &h->map_zrZc, &h->map_zrRc, &h->map_zrT[bin]};
  AXJ_CUDA(h, launch_zr(z, m, h->mixed, buf_f32(bin), h->stream));
  return AXJ_OK;
}

// One RK stage: the sensor chain on the stage input (if enabled), then the fused
// stage kernel over both tile classes.
int enqueue_stage(axj_handle* h, int bin, int bout, int stage) {
  if (h->c.shock_capturing) {
    int rc = enqueue_sensor_chain(h, bin);
    if (rc != AXJ_OK) return rc;
    return launch_stage_kernels(h, bin, bout, stage, CM_PRE);
  }
  return launch_stage_kernels(h, bin, bout, stage, CM_FILT);
}

FeatArgs feat_args(axj_handle* h, int b) {
  FeatArgs f;
  f.g = grid_of(h);
  f.U = buf_ptr(h, b);
  f.f32 = buf_f32(b);
  f.desc = h->desc;
  f.dxidz = h->dxidz;
  f.detadr = h->detadr;
  f.rc = h->rc;
  f.dz = h->dzv;
  f.dr = h->drv;
  f.feat = h->feat;
  for (int r = 0; r < 9; ++r)
    for (int m = 0; m < 6; ++m) f.sbp1[r][m] = (float)h->S1[r][m];
  return f;
}

InferArgs infer_args(axj_handle* h, int mode) {
  InferArgs a;
  a.g = grid_of(h);
  a.feat = h->feat;
  a.params = h->mlp;
  a.norm = h->norm;
  a.ramp = h->ramp;
  a.mode = mode;
  a.out = mode == 0 ? h->pred : h->star;
  a.mask = h->mask;
  a.held = h->held;
  a.flags = h->flags;
  a.ntiles_z = (h->Nz + 31) / 32;
  a.ntiles = a.ntiles_z * ((h->Nr + 3) / 4);
  return a;
}

// Learned-sensor stage. judge1: the first stage of a judge step (plain sensor with its
// r filter into the coefficient planes, prediction on the same input, fallback mask and
// held values); plain: a later stage of a judge step (the plain path).
int enqueue_stage_learned(axj_handle* h, int bin, int bout, int stage, bool judge1, bool plain) {
  if (plain) return enqueue_stage(h, bin, bout, stage);
  if (h->held_only) {
    if (judge1) {
      SensorArgs s = sensor_args(h, bin);
      AXJ_CUDA(h, launch_sensor(s, true, h->side, h->stream));
    }
    return launch_stage_kernels(h, bin, bout, stage, CM_LRN);
  }
  // the network runs once per step, on the first stage's input; its coefficients
  // serve the step's four stages, as the judge's plain values serve the steps between
  // judges
  if (stage > 1) return launch_stage_kernels(h, bin, bout, stage, CM_LRN);
  AXJ_CUDA(h, launch_features(feat_args(h, bin), h->stream));
  if (judge1) {
    SensorArgs s = sensor_args(h, bin);
    AXJ_CUDA(h, launch_sensor(s, true, h->side, h->stream));
    AXJ_CUDA(h, launch_mlp_infer(infer_args(h, 0), h->stream));
    JudgeArgs j;
    j.g = grid_of(h);
    j.pred = h->pred;
    j.plain = h->star + h->plane;
    j.thr = h->judge_thr;
    j.mask = h->mask;
    j.held = h->held;
    j.counts = h->counts;
    AXJ_CUDA(h, launch_judge(j, h->stream));
  } else {
    AXJ_CUDA(h, launch_mlp_infer(infer_args(h, 1), h->stream));
  }
  return launch_stage_kernels(h, bin, bout, stage, CM_LRN);
}

// Stage input/output buffers of RK4: U0 -> Ua -> Ub -> Ua -> U0 (FP32 Ua, Ub when mixed).
void rk4_buffers(const axj_handle* h, int b[5]) {
  const int a = h->mixed ? BUAF : BUA, c = h->mixed ? BUBF : BUB;
  b[0] = BU0; b[1] = a; b[2] = c; b[3] = a; b[4] = BU0;
}

// ComputeTimeStep on the device; with advance != 0 the kernel also performs
// time = time + delt for the step this dt is used by (ModRungeKutta.f90:152-155).
DtArgs dt_args(axj_handle* h, int advance) {
  DtArgs d;
  d.g = grid_of(h);
  d.U = h->U0;
  d.desc = h->desc;
  d.dxidz = h->dxidz;
  d.detadr = h->detadr;
  d.staleT = h->staleT;
  d.partial = h->partial;
  d.counter = h->counter;
  d.dt = h->dt;
  d.flags = h->flags;
  d.time = h->time;
  d.advance = advance;
  d.c = h->c;
  return d;
}

int enqueue_dt(axj_handle* h, int advance) {
  AXJ_CUDA(h, launch_dt(dt_args(h, advance), h->dt_blocks, h->stream));
  return AXJ_OK;
}

// RK4 (ModRungeKutta.f90:5-171) on the device dt. With the learned sensor, `judge`
// makes this a judge step.
int enqueue_rk4(axj_handle* h, bool judge = false) {
  int b[5];
  rk4_buffers(h, b);
  if (h->c.control_forcing == 2)
    AXJ_CUDA(h, launch_harmonic_phase(h->time, h->dt, h->c.harm_omega, 0, h->harm, h->stream));
  for (int st = 1; st <= 4; ++st) {
    const int rc = h->learned ? enqueue_stage_learned(h, b[st - 1], b[st], st, judge && st == 1, judge && st > 1 && h->judge_all)
                              : enqueue_stage(h, b[st - 1], b[st], st);
    if (rc != AXJ_OK) return rc;
  }
  return AXJ_OK;
}

// The learned sensor needs a model before any step.
int check_model(axj_handle* h) {
  if (h->learned && !h->held_only && !h->mlp_set) return fail(h, AXJ_ERR_ARG, "learned sensor without a model (axj_mlp_set / axj_mlp_train)");
  return AXJ_OK;
}

// The learned sensor judges on the first step after the state or the model changed
// and every judge_every iterations.
bool judge_due(const axj_handle* h) {
  return h->learned && (!h->judged || (h->judge_every > 0 && h->iteration % h->judge_every == 0));
}

// Captured step graphs: dt + RK4, and (learned sensor) the judge step.
int step_graph(axj_handle* h, bool judge, cudaGraphExec_t* out) {
  cudaGraphExec_t* ge = judge ? &h->graph_judge_exec : &h->graph_exec;
  cudaGraph_t* gr = judge ? &h->graph_judge : &h->graph;
  if (!*ge) {
    AXJ_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_dt(h, 1);
    if (rc == AXJ_OK) rc = enqueue_rk4(h, judge);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    if (rc != AXJ_OK) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) return fail(h, AXJ_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    *gr = g;
    AXJ_CUDA(h, cudaGraphInstantiate(ge, g, 0));
  }
  *out = *ge;
  return AXJ_OK;
}

// The captured graphs hold the model's normalisation by value: a new model (or new
// statistics) drops them, and the next step captures them again.
void drop_graphs(axj_handle* h) {
  cudaStreamSynchronize(h->stream);
  cudaGraphExec_t* ex[4] = {&h->graph_exec, &h->graph_judge_exec, &h->graph_rk4_exec[0], &h->graph_rk4_exec[1]};
  cudaGraph_t* gr[4] = {&h->graph, &h->graph_judge, &h->graph_rk4[0], &h->graph_rk4[1]};
  for (int k = 0; k < 4; ++k) {
    if (*ex[k]) cudaGraphExecDestroy(*ex[k]);
    if (*gr[k]) cudaGraphDestroy(*gr[k]);
    *ex[k] = nullptr;
    *gr[k] = nullptr;
  }
}

// Captured RK4 stages alone (the dt the host passed to axj_rk4_step is on the device).
int rk4_graph(axj_handle* h, bool judge, cudaGraphExec_t* out) {
  const int k = judge ? 1 : 0;
  if (!h->graph_rk4_exec[k]) {
    AXJ_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_rk4(h, judge);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    if (rc != AXJ_OK) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) return fail(h, AXJ_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    h->graph_rk4[k] = g;
    AXJ_CUDA(h, cudaGraphInstantiate(&h->graph_rk4_exec[k], g, 0));
  }
  *out = h->graph_rk4_exec[k];
  return AXJ_OK;
}

// One graph-launched step; advances the iteration counter.
int launch_step(axj_handle* h) {
  if (int rc = check_model(h)) return rc;
  const bool judge = judge_due(h);
  cudaGraphExec_t ge = nullptr;
  int rc = step_graph(h, judge, &ge);
  if (rc != AXJ_OK) return rc;
  AXJ_CUDA(h, cudaGraphLaunch(ge, h->stream));
  if (judge) {
    h->judged = true;
    h->njudges += 1;
  }
  h->iteration += 1;
  return AXJ_OK;
}

int flags_status(axj_handle* h, int f) {
  if (f & 4) return fail(h, AXJ_ERR_TIMEOUT, "a bounded wait on a TMA transfer gave up");
  if (f & 2) return fail(h, AXJ_ERR_DT_BLOWUP, "Time step blow up (every point blanked, dt == 100)");
  if (f & 1) return fail(h, AXJ_ERR_NONFINITE, "non-finite value in the solution or time step");
  return AXJ_OK;
}

int check_flags(axj_handle* h) {
  int f = 0;
  AXJ_CUDA(h, cudaMemcpyAsync(&f, h->flags, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  AXJ_CUDA(h, cudaStreamSynchronize(h->stream));
  if (f & 4) return fail(h, AXJ_ERR_TIMEOUT, "a bounded wait on a TMA transfer gave up");
  if (f & 2) return fail(h, AXJ_ERR_DT_BLOWUP, "Time step blow up (every point blanked, dt == 100)");
  if (f & 1) return fail(h, AXJ_ERR_NONFINITE, "non-finite value in the solution or time step");
  return AXJ_OK;
}

}  // namespace

namespace axj {
// Message returned by axj_last_error(NULL) (used by entry points without a handle).
void set_global_error(const char* msg) { g_create_error = msg; }
}  // namespace axj

// The per-point descriptors of one block holding the grid (CreateAllPatches,
// ModPatch.f90:214-242: the last patch of a direction wins a point) with pitch P, and the
// face-operation lists in patch order (the BoundaryConditions loop, ModBC.f90:25-274):
// faces[0] = 0, then per face point its count and 0-based patch indices, referenced from
// the descriptor. iT, jT (1-based): the last face point the loop visits, else the last
// point of the RHS loops (ModRHS.f90:76,145), where the stale scalar T is taken.
static int build_point_maps(const axj_patch* patches, int64_t npatch, int64_t Nz, int64_t Nr, int64_t P,
                            const double* ibval, std::vector<uint32_t>& desc, std::vector<int>& faces, int64_t& iT,
                            int64_t& jT, std::string& msg) {
  const size_t npt = (size_t)Nz * Nr;
  std::vector<int> which_i(npt, 0), which_j(npt, 0);  // 1-based patch number, 0 = none
  for (int64_t k = 0; k < npatch; ++k) {
    const axj_patch& p = patches[k];
    for (int64_t i = std::max<int64_t>(p.i_start, 1); i <= std::min<int64_t>(p.i_end, Nz); ++i)
      for (int64_t j = std::max<int64_t>(p.j_start, 1); j <= std::min<int64_t>(p.j_end, Nr); ++j) {
        const size_t x = (size_t)(i - 1) + (size_t)(j - 1) * Nz;
        if (p.bc_dir == 1 || p.bc_dir == -1) which_i[x] = (int)k + 1;
        if (p.bc_dir == 2 || p.bc_dir == -2) which_j[x] = (int)k + 1;
      }
  }
  // face-operation lists in patch order (BoundaryConditions loop, ModBC.f90:25-274)
  std::vector<std::vector<int>> ops(npt);
  iT = Nz;
  jT = Nr;
  for (int64_t k = 0; k < npatch; ++k) {
    const axj_patch& p = patches[k];
    if (p.bc == AXJ_BC_AXIS) continue;
    int64_t is, ie, js, je;
    if (p.bc_dir == 1) { is = ie = p.i_start; js = p.j_start; je = p.j_end; }
    else if (p.bc_dir == -1) { is = ie = p.i_end; js = p.j_start; je = p.j_end; }
    else if (p.bc_dir == 2) { is = p.i_start; ie = p.i_end; js = je = p.j_start; }
    else { is = p.i_start; ie = p.i_end; js = je = p.j_end; }
    for (int64_t i = is; i <= ie; ++i)
      for (int64_t j = js; j <= je; ++j) {
        if (i < 1 || i > Nz || j < 1 || j > Nr) continue;
        const bool j1 = (j == 1);
        const int adir = (int)(p.bc_dir < 0 ? -p.bc_dir : p.bc_dir);
        bool active = false;
        if (p.bc == AXJ_BC_SAT_FARFIELD) active = !j1 && adir == 1;
        else if (p.bc == AXJ_BC_SAT_NOSLIP_WALL || p.bc == AXJ_BC_NSCBC_NOSLIP_WALL) active = true;
        else if (p.bc == AXJ_BC_NSCBC_NONREFLECTING) active = !j1;
        if (!active) continue;
        const size_t x = (size_t)(i - 1) + (size_t)(j - 1) * Nz;
        ops[x].push_back((int)k);
        if ((int)ops[x].size() > MAX_FACE_OPS) {
          char b[128];
          std::snprintf(b, sizeof(b), "more than %d face operations at (%lld,%lld)", MAX_FACE_OPS, (long long)i,
                        (long long)j);
          msg = b;
          return AXJ_ERR_BADPATCH;
        }
        iT = i;
        jT = j;
      }
  }
  faces.assign(1, 0);
  desc.assign((size_t)P * Nr, make_desc(ROW_NONE, ROW_NONE, false, 0));
  for (int64_t j = 1; j <= Nr; ++j)
    for (int64_t i = 1; i <= Nz; ++i) {
      const size_t x = (size_t)(i - 1) + (size_t)(j - 1) * Nz;
      int zr = 4, rw = 4;
      if (which_i[x]) {
        const axj_patch& p = patches[which_i[x] - 1];
        zr = p.bc_dir == 1 ? (int)(i - p.i_start) : (int)(8 + i - p.i_end);
      }
      if (which_j[x]) {
        const axj_patch& p = patches[which_j[x] - 1];
        rw = p.bc_dir == 2 ? (int)(j - p.j_start) : (int)(8 + j - p.j_end);
      }
      uint32_t f = 0;
      if (!ops[x].empty()) {
        f = (uint32_t)faces.size();
        faces.push_back((int)ops[x].size());
        for (int id : ops[x]) faces.push_back(id);
      }
      desc[(size_t)(j - 1) * P + (i - 1)] = make_desc(zr, rw, ibval[x] == 0.0, f);
    }
  if (faces.size() >= (1u << 20)) {
    msg = "too many face points";
    return AXJ_ERR_BADPATCH;
  }
  return AXJ_OK;
}

// The tiles of the stage and sensor kernels, in launch order: r bands [0, 8), then bands
// of TR rows up to 8 rows short of the top, then the rest in bands of at most TR rows;
// per band the tiles along z. Interior tiles need a full band; the thin bands along r = 0
// and r = r_max (closure rows, the axis, faces) hold general tiles that own only their
// band's rows (the row count is packed into the tile's j0: bits 24-31 hold TR - rows).
// Entries (i0, j0, rows).
static std::vector<int64_t> tile_candidates(int64_t Nz, int64_t Nr) {
  std::vector<std::pair<int64_t, int64_t>> bands;
  int64_t j = 0;
  if (Nr > 24) {
    bands.push_back({0, 8});
    j = 8;
  }
  while (j + TR <= Nr - 8) {
    bands.push_back({j, TR});
    j += TR;
  }
  while (j < Nr) {
    const int64_t rows = std::min<int64_t>(TR, Nr - j);
    bands.push_back({j, rows});
    j += rows;
  }
  std::vector<int64_t> c;
  for (const auto& band : bands)
    for (int64_t i0 = 0; i0 < Nz; i0 += TZ) {
      c.push_back(i0);
      c.push_back(band.first);
      c.push_back(band.second);
    }
  return c;
}

// The tile lists from the classes of the candidates (bit 0 interior stage tile, bit 1
// interior sensor tile).
static void tile_lists(const std::vector<int64_t>& cand, const std::vector<unsigned char>& flags,
                       std::vector<int2>& tint, std::vector<int2>& tgen, std::vector<int2>& sti,
                       std::vector<int2>& stg) {
  tint.clear(); tgen.clear(); sti.clear(); stg.clear();
  for (size_t t = 0; t < flags.size(); ++t) {
    const int64_t i0 = cand[3 * t], j0 = cand[3 * t + 1], brows = cand[3 * t + 2];
    const int ytile = (int)j0 | (int)((TR - brows) << 24);
    const bool interior = flags[t] & 1, sint = (flags[t] >> 1) & 1;
    (interior ? tint : tgen).push_back(make_int2((int)i0, interior ? (int)j0 : ytile));
    (sint ? sti : stg).push_back(make_int2((int)i0, sint ? (int)j0 : ytile));
  }
}

// Classes of every candidate tile from the descriptors (pitch P), on the host.
static std::vector<unsigned char> classify_tiles(const std::vector<uint32_t>& desc, int64_t P, int64_t Nz,
                                                 int64_t Nr, const std::vector<int64_t>& cand) {
  std::vector<unsigned char> flags(cand.size() / 3);
  auto dsc = [&](int64_t i, int64_t j) { return desc[(size_t)j * P + i]; };
  for (size_t t = 0; t < flags.size(); ++t) {
    const int64_t i0 = cand[3 * t], j0 = cand[3 * t + 1], brows = cand[3 * t + 2];
    bool interior = brows == TR && i0 - H_INT >= 0 && i0 + TZ + H_INT <= Nz && j0 - H_INT >= 0 &&
                    j0 + TR + H_INT <= Nr;
    for (int64_t j = j0; interior && j < j0 + TR; ++j)
      for (int64_t i = i0; interior && i < i0 + TZ; ++i) {
        uint32_t d = dsc(i, j);
        if (desc_zrow(d) != 4 || desc_rrow(d) != 4 || desc_blank(d) || desc_face(d) != 0) interior = false;
      }
    // r-halo points on the tile columns: dV/dz there feeds the mixed derivatives, and
    // the r filter of the coefficients runs there with the centred row
    for (int64_t j = j0 - H_INT; interior && j < j0 + TR + H_INT; ++j) {
      if (j >= j0 && j < j0 + TR) continue;
      for (int64_t i = i0; interior && i < i0 + TZ; ++i) {
        uint32_t d = dsc(i, j);
        if (desc_zrow(d) != 4 || desc_rrow(d) != 4 || desc_blank(d)) interior = false;
      }
    }
    // z-halo points on the tile rows: the r filter of the coefficients
    for (int64_t j = j0; interior && j < j0 + TR; ++j)
      for (int64_t i = i0 - H_INT; interior && i < i0 + TZ + H_INT; ++i) {
        if (i >= i0 && i < i0 + TZ) continue;
        uint32_t d = dsc(i, j);
        if (desc_rrow(d) != 4 || desc_blank(d)) interior = false;
      }
    // sensor classes: S, T and the dilatation are formed on a cross of halo
    // SENS_HS_INT from V_r, V_z stencils of reach H_INT, so every point within
    // SENS_HS_INT of the tile must use centred rows, and the V region must lie inside.
    const int64_t hv = SENS_HS_INT + H_INT, hs = SENS_HS_INT;
    bool sint = brows == TR && i0 - hz_of((int)hv) >= 0 && i0 + TZ + hz_of((int)hv) <= Nz && j0 - hv >= 0 &&
                j0 + TR + hv <= Nr;
    for (int64_t j = j0 - hs; sint && j < j0 + TR + hs; ++j)
      for (int64_t i = i0 - hs; sint && i < i0 + TZ + hs; ++i) {
        uint32_t d = dsc(i, j);
        if (desc_zrow(d) != 4 || desc_rrow(d) != 4 || desc_blank(d)) sint = false;
      }
    flags[t] = (unsigned char)((interior ? 1 : 0) | (sint ? 2 : 0));
  }
  return flags;
}

// The point where the stale scalar T is taken (1-based): the last face point of the bc
// loop that acts, else the last point of the RHS loops (ModRHS.f90:76,145).
static void stale_T_point(const axj_patch* patches, int64_t npatch, int64_t Nz, int64_t Nr, int64_t& iT,
                          int64_t& jT) {
  iT = Nz;
  jT = Nr;
  for (int64_t k = 0; k < npatch; ++k) {
    const axj_patch& p = patches[k];
    if (p.bc == AXJ_BC_AXIS) continue;
    int64_t is, ie, js, je;
    if (p.bc_dir == 1) { is = ie = p.i_start; js = p.j_start; je = p.j_end; }
    else if (p.bc_dir == -1) { is = ie = p.i_end; js = p.j_start; je = p.j_end; }
    else if (p.bc_dir == 2) { is = p.i_start; ie = p.i_end; js = je = p.j_start; }
    else { is = p.i_start; ie = p.i_end; js = je = p.j_end; }
    const int adir = (int)(p.bc_dir < 0 ? -p.bc_dir : p.bc_dir);
    for (int64_t i = is; i <= ie; ++i)
      for (int64_t j = js; j <= je; ++j) {
        if (i < 1 || i > Nz || j < 1 || j > Nr) continue;
        const bool j1 = (j == 1);
        bool active = false;
        if (p.bc == AXJ_BC_SAT_FARFIELD) active = !j1 && adir == 1;
        else if (p.bc == AXJ_BC_SAT_NOSLIP_WALL || p.bc == AXJ_BC_NSCBC_NOSLIP_WALL) active = true;
        else if (p.bc == AXJ_BC_NSCBC_NONREFLECTING) active = !j1;
        if (!active) continue;
        iT = i;
        jT = j;
      }
  }
}

// The host algorithm: build_point_maps, the z / r codes and the tile classes.
static int host_patch_maps(const axj_patch* patches, int64_t npatch, int64_t Nz, int64_t Nr, int64_t P,
                           const double* ibval, std::vector<uint32_t>& desc, std::vector<unsigned char>& zcode,
                           std::vector<unsigned char>& rcode, std::vector<int>& faces, std::vector<int2>& tint,
                           std::vector<int2>& tgen, std::vector<int2>& sti, std::vector<int2>& stg, int64_t& iT,
                           int64_t& jT, std::string& msg) {
  const int rc = build_point_maps(patches, npatch, Nz, Nr, P, ibval, desc, faces, iT, jT, msg);
  if (rc != AXJ_OK) return rc;
  zcode.resize(desc.size());
  rcode.resize(desc.size());
  for (size_t x = 0; x < desc.size(); ++x) {
    zcode[x] = (unsigned char)(desc_blank(desc[x]) ? ROW_NONE : (uint32_t)desc_zrow(desc[x]));
    rcode[x] = (unsigned char)(desc_blank(desc[x]) ? ROW_NONE : (uint32_t)desc_rrow(desc[x]));
  }
  const std::vector<int64_t> cand = tile_candidates(Nz, Nr);
  tile_lists(cand, classify_tiles(desc, P, Nz, Nr, cand), tint, tgen, sti, stg);
  return AXJ_OK;
}

// The device algorithm (axj_prep.cuh, one thread per row and per tile), or with
// emulate the same per-row and per-tile functions run on the host.
static int device_patch_maps(const axj_patch* patches, int64_t npatch, int64_t Nz, int64_t Nr, int64_t P,
                             const double* ibval, std::vector<uint32_t>& desc, std::vector<unsigned char>& zcode,
                             std::vector<unsigned char>& rcode, std::vector<int>& faces, std::vector<int2>& tint,
                             std::vector<int2>& tgen, std::vector<int2>& sti, std::vector<int2>& stg, int64_t& iT,
                             int64_t& jT, std::string& msg, bool emulate = false) {
  const PrepArgs a{patches, (int)npatch, Nz, Nr, P, ibval};
  const std::vector<int64_t> cand = tile_candidates(Nz, Nr);
  const int64_t ncand = (int64_t)cand.size() / 3;
  desc.assign((size_t)P * Nr, 0);
  zcode.assign(desc.size(), 0);
  rcode.assign(desc.size(), 0);
  std::vector<unsigned char> flags((size_t)ncand);
  if (emulate) {
    std::vector<int64_t> off((size_t)Nr);
    int64_t total = 1;
    for (int64_t j = 1; j <= Nr; ++j) {
      const int64_t sz = prep_row_size(a, j);
      if (sz < 0) {
        msg = "more than " + std::to_string(MAX_FACE_OPS) + " face operations at a point of row " + std::to_string(j);
        return AXJ_ERR_BADPATCH;
      }
      off[j - 1] = total;
      total += sz;
    }
    if (total >= (1 << 20)) {
      msg = "too many face points";
      return AXJ_ERR_BADPATCH;
    }
    faces.assign((size_t)total, 0);
    for (int64_t j = 1; j <= Nr; ++j) prep_row(a, j, off[j - 1], desc.data(), zcode.data(), rcode.data(), faces.data());
    for (int64_t t = 0; t < ncand; ++t)
      flags[t] = (unsigned char)prep_tile_flags(desc.data(), P, Nz, Nr, cand[3 * t], cand[3 * t + 1], cand[3 * t + 2]);
  } else {
    char b[256] = {0};
    const int rc = prep_on_device(a, cand.data(), ncand, desc.data(), zcode.data(), rcode.data(), faces, flags.data(),
                                  b, (int)sizeof(b));
    if (rc != AXJ_OK) {
      msg = b;
      return rc;
    }
  }
  tile_lists(cand, flags, tint, tgen, sti, stg);
  stale_T_point(patches, npatch, Nz, Nr, iT, jT);
  return AXJ_OK;
}

extern "C" {

int axj_operator_tables(double* sbp1, double* sbp2, double* tgfilt) {
  if (!sbp1 || !sbp2 || !tgfilt) return fail(nullptr, AXJ_ERR_ARG, "null argument");
  double S1[9][6], S2[9][6], G[9][11];
  build_tables(S1, S2, G);
  std::memcpy(sbp1, S1, sizeof(S1));
  std::memcpy(sbp2, S2, sizeof(S2));
  std::memcpy(tgfilt, G, sizeof(G));
  return AXJ_OK;
}

int axj_point_maps(const axj_patch* patches, int64_t npatch, int64_t Nz, int64_t Nr, const double* ibval,
                   uint8_t* zrow, uint8_t* rrow, uint8_t* blank, uint8_t* nfaceops, uint64_t* faceop_ids) {
  if ((npatch > 0 && !patches) || !ibval || !zrow || !rrow || !blank || !nfaceops || !faceop_ids)
    return fail(nullptr, AXJ_ERR_ARG, "null argument");
  if (Nz < 1 || Nr < 1) return fail(nullptr, AXJ_ERR_ARG, "grid %lld x %lld", (long long)Nz, (long long)Nr);
  if (npatch < 0 || npatch > MAX_PATCHES) return fail(nullptr, AXJ_ERR_BADPATCH, "%lld patches", (long long)npatch);
  for (int64_t k = 0; k < npatch; ++k) {
    const int64_t d = patches[k].bc_dir;
    if (d != 1 && d != -1 && d != 2 && d != -2)
      return fail(nullptr, AXJ_ERR_BADPATCH, "patch %lld: bc_dir %lld", (long long)k + 1, (long long)d);
  }
  std::vector<uint32_t> desc;
  std::vector<int> faces;
  int64_t iT = 0, jT = 0;
  std::string msg;
  const int rc = build_point_maps(patches, npatch, Nz, Nr, Nz, ibval, desc, faces, iT, jT, msg);
  if (rc != AXJ_OK) return fail(nullptr, rc, "%s", msg.c_str());
  for (size_t x = 0; x < (size_t)Nz * Nr; ++x) {
    const uint32_t d = desc[x];
    zrow[x] = (uint8_t)desc_zrow(d);
    rrow[x] = (uint8_t)desc_rrow(d);
    blank[x] = desc_blank(d) ? 1 : 0;
    const uint32_t f = desc_face(d);
    nfaceops[x] = f ? (uint8_t)faces[f] : 0;
    uint64_t ids = 0;
    for (int k = 0; f && k < faces[f]; ++k) ids |= (uint64_t)(faces[f + 1 + k] + 1) << (8 * k);
    faceop_ids[x] = ids;
  }
  return AXJ_OK;
}

int axj_prep_maps(const axj_patch* patches, int64_t npatch, int64_t Nz, int64_t Nr, const double* ibval,
                  int64_t algorithm, uint32_t* desc, int32_t* faces, int64_t faces_cap, int64_t* nfaces,
                  int32_t* tiles, int64_t tiles_cap, int64_t* counts, int64_t* stale) {
  if ((npatch > 0 && !patches) || !ibval || !desc || !nfaces || !counts || !stale)
    return fail(nullptr, AXJ_ERR_ARG, "null argument");
  if (Nz < 1 || Nr < 1) return fail(nullptr, AXJ_ERR_ARG, "grid %lld x %lld", (long long)Nz, (long long)Nr);
  if (npatch < 0 || npatch > MAX_PATCHES) return fail(nullptr, AXJ_ERR_BADPATCH, "%lld patches", (long long)npatch);
  for (int64_t k = 0; k < npatch; ++k) {
    const int64_t d = patches[k].bc_dir;
    if (d != 1 && d != -1 && d != 2 && d != -2)
      return fail(nullptr, AXJ_ERR_BADPATCH, "patch %lld: bc_dir %lld", (long long)k + 1, (long long)d);
  }
  if (algorithm < 0 || algorithm > 2) return fail(nullptr, AXJ_ERR_ARG, "algorithm %lld", (long long)algorithm);
  const int64_t P = (Nz + 31) / 32 * 32;
  std::vector<uint32_t> dv;
  std::vector<unsigned char> zc, rc_;
  std::vector<int> fv;
  std::vector<int2> lists[4];
  int64_t iT = 0, jT = 0;
  std::string msg;
  const int rc = algorithm == 0
                     ? host_patch_maps(patches, npatch, Nz, Nr, P, ibval, dv, zc, rc_, fv, lists[0], lists[1], lists[2],
                                       lists[3], iT, jT, msg)
                     : device_patch_maps(patches, npatch, Nz, Nr, P, ibval, dv, zc, rc_, fv, lists[0], lists[1],
                                         lists[2], lists[3], iT, jT, msg, algorithm == 1);
  if (rc != AXJ_OK) return fail(nullptr, rc, "%s", msg.c_str());
  std::memcpy(desc, dv.data(), dv.size() * sizeof(uint32_t));
  *nfaces = (int64_t)fv.size();
  if (faces && (int64_t)fv.size() <= faces_cap) std::memcpy(faces, fv.data(), fv.size() * sizeof(int32_t));
  int64_t n = 0;
  for (int c = 0; c < 4; ++c) {
    counts[c] = (int64_t)lists[c].size();
    for (const int2& t : lists[c]) {
      if (tiles && n < tiles_cap) {
        tiles[2 * n] = t.x;
        tiles[2 * n + 1] = t.y;
      }
      ++n;
    }
  }
  stale[0] = iT;
  stale[1] = jT;
  if ((faces && (int64_t)fv.size() > faces_cap) || (tiles && n > tiles_cap))
    return fail(nullptr, AXJ_ERR_ARG, "output capacity: %lld face entries, %lld tiles", (long long)fv.size(),
                (long long)n);
  return AXJ_OK;
}

void axj_default_params(axj_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->gam = 1.4;
  p->Re = 1000.0;
  p->Pr = 0.72;
  p->CFL = 0.5;
  p->sponge_start_top = 12.5;
  p->sponge_A_top = 0.5;
  p->sponge_end_left = 6.0;
  p->sponge_A_left = 5.0;
  p->C_mu = 0.0;
  p->C_beta = 0.0;
  p->C_kappa = 0.0;
  p->forcing_alpha = 6.0;
  p->forcing_lz = 1.0;
  p->forcing_lr = 1.0;
  p->do_viscous_terms = 1;
  p->shock_capturing = 0;
  p->control_forcing = 0;
  p->dt_mode = AXJ_DT_REFERENCE;
  p->precision = AXJ_FP64;
  p->sensor = AXJ_SENSOR_PLAIN;
  p->judge_every = 50;
  p->judge_threshold = 0.1;
}

const char* axj_version(void) { return "axj 0.2 sm_100a fp64 mixed"; }

double axj_mu_of_T(double T) {
  static const std::vector<double> tab = [] {
    std::vector<double> t(POW_TAB);
    pow0666_fill(t.data());
    return t;
  }();
  return pow0666(T, tab.data());
}

int axj_read_bc_file(const char* path, axj_bc_record* rec, int64_t max_records, int64_t* nrecords) {
  if (!path || !nrecords) return fail(nullptr, AXJ_ERR_ARG, "null argument");
  FILE* f = std::fopen(path, "r");
  if (!f) return fail(nullptr, AXJ_ERR_ARG, "cannot open bc file %s", path);
  int64_t n = 0;
  char line[1024];
  int rc = AXJ_OK;
  while (std::fgets(line, sizeof(line), f)) {
    long long v[9];
    int k = std::sscanf(line, "%lld %lld %lld %lld %lld %lld %lld %lld %lld", &v[0], &v[1], &v[2], &v[3], &v[4],
                        &v[5], &v[6], &v[7], &v[8]);
    if (k <= 0) continue;  // blank line: list-directed input skips it
    // a record is 9 integers (ModPatch.f90:48); the reference's list-directed READ would
    // take the missing values from the next line, so a short record is an error here
    if (k < 9) { rc = fail(nullptr, AXJ_ERR_BADPATCH, "bc file %s: short record %lld", path, (long long)n + 1); break; }
    if (n < max_records && rec) {
      rec[n].bc = v[1];
      rec[n].bc_dir = v[2];
      rec[n].istart = v[3];
      rec[n].iend = v[4];
      rec[n].jstart = v[5];
      rec[n].jend = v[6];
    }
    ++n;
  }
  std::fclose(f);
  *nrecords = n;
  if (rc == AXJ_OK && rec && n > max_records)
    return fail(nullptr, AXJ_ERR_ARG, "bc file has %lld records, buffer holds %lld", (long long)n,
                (long long)max_records);
  return rc;
}

int axj_patches_from_records(const axj_bc_record* rec, int64_t nrec, int64_t Nzg, int64_t Nrg, axj_patch* out,
                             int64_t* npatch) {
  if (!rec || !out || !npatch) return fail(nullptr, AXJ_ERR_ARG, "null argument");
  int64_t n = 0;
  for (int64_t k = 0; k < nrec; ++k) {
    int64_t is = rec[k].istart, ie = rec[k].iend, js = rec[k].jstart, je = rec[k].jend, dir = rec[k].bc_dir;
    if (is == -1) is = Nzg;
    if (js == -1) js = Nrg;
    if (ie == -1) ie = Nzg;
    if (je == -1) je = Nrg;
    int64_t pis, pie, pjs, pje;  // the 4-wide strip (ModPatch.f90:159-179)
    if (dir == 1) { pis = is; pie = is + 3; pjs = js; pje = je; }
    else if (dir == -1) { pis = ie - 3; pie = ie; pjs = js; pje = je; }
    else if (dir == 2) { pis = is; pie = ie; pjs = js; pje = js + 3; }
    else if (dir == -2) { pis = is; pie = ie; pjs = je - 3; pje = je; }
    else return fail(nullptr, AXJ_ERR_BADPATCH, "record %lld: bc_dir %lld", (long long)k + 1, (long long)dir);
    // the first/last block point inside the strip in the i-outer, j-inner scan
    // (CreateAllPatches :154-197), for one block holding the whole grid
    int64_t ci0 = std::max<int64_t>(pis, 1), ci1 = std::min<int64_t>(pie, Nzg);
    int64_t cj0 = std::max<int64_t>(pjs, 1), cj1 = std::min<int64_t>(pje, Nrg);
    if (pis > pie || pjs > pje || ci0 > ci1 || cj0 > cj1) continue;  // no point of this block: patch dropped
    const int64_t sI = ci0, sJ = cj0, eI = ci1, eJ = cj1;
    axj_patch p;
    p.bc = rec[k].bc;
    p.bc_dir = dir;
    // PatchCreation (:264-309)
    if (dir == 1) { p.i_start = sI; p.i_end = sI + 3; p.j_start = sJ; p.j_end = eJ; }
    else if (dir == -1) { p.i_start = eI - 3; p.i_end = eI; p.j_start = sJ; p.j_end = eJ; }
    else if (dir == 2) { p.i_start = sI; p.i_end = eI; p.j_start = sJ; p.j_end = sJ + 3; }
    else { p.i_start = sI; p.i_end = eI; p.j_start = eJ - 3; p.j_end = eJ; }
    out[n++] = p;
  }
  *npatch = n;
  return AXJ_OK;
}

const char* axj_last_error(const axj_handle* h) { return h ? h->err.c_str() : g_create_error.c_str(); }

int axj_set_wait_limit(axj_handle* h, int64_t tries) {
  if (!h) return fail(h, AXJ_ERR_ARG, "null handle");
  if (tries > (int64_t)INT32_MAX) return fail(h, AXJ_ERR_ARG, "wait limit %lld too large", (long long)tries);
  AXJ_CUDA(h, cudaSetDevice(h->device));
  AXJ_CUDA(h, cudaStreamSynchronize(h->stream));
  AXJ_CUDA(h, set_wait_tries((int)tries));
  AXJ_CUDA(h, cudaDeviceSynchronize());
  return AXJ_OK;
}

void axj_destroy(axj_handle* h) {
  if (!h) return;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->out_stream) {
    cudaStreamSynchronize(h->out_stream);
    cudaStreamDestroy(h->out_stream);
  }
  if (h->out_snapped) cudaEventDestroy(h->out_snapped);
  if (h->out_copied) cudaEventDestroy(h->out_copied);
  if (h->out_snap) cudaFree(h->out_snap);
  if (h->out_host) cudaFreeHost(h->out_host);
  if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
  if (h->graph) cudaGraphDestroy(h->graph);
  if (h->graph_judge_exec) cudaGraphExecDestroy(h->graph_judge_exec);
  if (h->graph_judge) cudaGraphDestroy(h->graph_judge);
  for (int k = 0; k < 2; ++k) {
    if (h->graph_rk4_exec[k]) cudaGraphExecDestroy(h->graph_rk4_exec[k]);
    if (h->graph_rk4[k]) cudaGraphDestroy(h->graph_rk4[k]);
  }
  for (void* p : h->allocs) cudaFree(p);
  if (h->ds_feat) cudaFree(h->ds_feat);
  if (h->ds_targ) cudaFree(h->ds_targ);
  if (h->side.stream) cudaStreamSynchronize(h->side.stream);
  if (h->side.fork) cudaEventDestroy(h->side.fork);
  if (h->side.join) cudaEventDestroy(h->side.join);
  if (h->side.stream) cudaStreamDestroy(h->side.stream);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

int axj_create(const axj_params* prm, int64_t Nz, int64_t Nr, const double* zvec, const double* rvec,
               const double* ibval, const axj_patch* patches, int64_t npatch, axj_handle** out) {
  if (!prm || !zvec || !rvec || !ibval || !out || (npatch > 0 && !patches))
    return fail(nullptr, AXJ_ERR_ARG, "null argument");
  *out = nullptr;
  if (Nz < 12 || Nr < 12 || Nz > (1 << 20) || Nr > (1 << 20))
    return fail(nullptr, AXJ_ERR_BADGRID, "grid %lld x %lld outside 12..2^20", (long long)Nz, (long long)Nr);
  if (npatch > MAX_PATCHES) return fail(nullptr, AXJ_ERR_BADPATCH, "more than %d patches", MAX_PATCHES);
  if (prm->precision != AXJ_FP64 && prm->precision != AXJ_MIXED)
    return fail(nullptr, AXJ_ERR_UNSUPPORTED, "precision %lld not built", (long long)prm->precision);
  if (prm->sensor != AXJ_SENSOR_PLAIN && prm->sensor != AXJ_SENSOR_LEARNED && prm->sensor != AXJ_SENSOR_HELD)
    return fail(nullptr, AXJ_ERR_ARG, "sensor %lld unknown", (long long)prm->sensor);
  if (prm->patch_prep != 0 && prm->patch_prep != 1)
    return fail(nullptr, AXJ_ERR_ARG, "patch_prep %lld unknown", (long long)prm->patch_prep);
  if (prm->stage_rows != 0 && prm->stage_rows != TR && prm->stage_rows != TR / 2)
    return fail(nullptr, AXJ_ERR_ARG, "stage_rows %lld is not 0, %d or %d", (long long)prm->stage_rows, TR, TR / 2);
  if (prm->sensor != AXJ_SENSOR_PLAIN && !prm->shock_capturing)
    return fail(nullptr, AXJ_ERR_ARG, "the learned sensor needs shock_capturing = 1");
  if (prm->sensor != AXJ_SENSOR_PLAIN && (prm->judge_every < 1 || !(prm->judge_threshold >= 0.0)))
    return fail(nullptr, AXJ_ERR_ARG, "judge_every must be >= 1 and judge_threshold >= 0");
  if (prm->judge_stages != 0 && prm->judge_stages != 1 && prm->judge_stages != 4)
    return fail(nullptr, AXJ_ERR_ARG, "judge_stages %lld is not 0, 1 or 4", (long long)prm->judge_stages);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(nullptr, AXJ_ERR_NODEVICE, "no CUDA device available");
  if (prm->device < 0 || prm->device >= ndev)
    return fail(nullptr, AXJ_ERR_ARG, "device %lld not in 0..%d", (long long)prm->device, ndev - 1);
  {
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, (int)prm->device) != cudaSuccess || prop.major != 10)
      return fail(nullptr, AXJ_ERR_NODEVICE, "device %lld is not an sm_100 (B200) GPU", (long long)prm->device);
    if (cudaSetDevice((int)prm->device) != cudaSuccess)
      return fail(nullptr, AXJ_ERR_NODEVICE, "cudaSetDevice(%lld) failed", (long long)prm->device);
  }
  // tensor-product grid: z depends on i only, r on j only (the reference only
  // carries dxi/dz and deta/dr, ModDeriv.f90:57,108)
  for (int64_t j = 0; j < Nr; ++j)
    for (int64_t i = 0; i < Nz; ++i) {
      if (zvec[i + j * Nz] != zvec[i]) return fail(nullptr, AXJ_ERR_BADGRID, "z varies with j at (%lld,%lld)", (long long)i + 1, (long long)j + 1);
      if (rvec[i + j * Nz] != rvec[j * Nz]) return fail(nullptr, AXJ_ERR_BADGRID, "r varies with i at (%lld,%lld)", (long long)i + 1, (long long)j + 1);
    }
  for (int64_t k = 0; k < npatch; ++k) {
    const axj_patch& p = patches[k];
    if (p.bc_dir != 1 && p.bc_dir != -1 && p.bc_dir != 2 && p.bc_dir != -2)
      return fail(nullptr, AXJ_ERR_BADPATCH, "patch %lld: bc_dir %lld", (long long)k + 1, (long long)p.bc_dir);
    if (p.i_start > p.i_end || p.j_start > p.j_end)
      return fail(nullptr, AXJ_ERR_BADPATCH, "patch %lld: empty range", (long long)k + 1);
    if (p.bc < 90 || p.bc > 95) return fail(nullptr, AXJ_ERR_BADPATCH, "patch %lld: bc %lld", (long long)k + 1, (long long)p.bc);
  }

  axj_handle* h = new axj_handle();
  cudaGetDevice(&h->device);
  h->Nz = (int)Nz;
  h->Nr = (int)Nr;
  h->P = (Nz + 31) / 32 * 32;
  h->plane = h->P * Nr;
  h->params = *prm;
  Consts& c = h->c;
  c.gam = prm->gam; c.Re = prm->Re; c.Pr = prm->Pr; c.CFL = prm->CFL;
  c.sponge_start_top = prm->sponge_start_top; c.sponge_A_top = prm->sponge_A_top;
  c.sponge_end_left = prm->sponge_end_left; c.sponge_A_left = prm->sponge_A_left;
  c.C_mu_Re = prm->C_mu * prm->Re;
  c.C_beta_Re = prm->C_beta * prm->Re;
  c.C_kappa_Re_Pr = prm->C_kappa * prm->Re * prm->Pr;
  c.forcing_alpha = prm->forcing_alpha; c.forcing_z0 = prm->forcing_z0; c.forcing_r0 = prm->forcing_r0;
  c.forcing_lz = prm->forcing_lz; c.forcing_lr = prm->forcing_lr;
  c.r_top = rvec[(Nr - 1) * Nz];
  c.inv_gam = 1.0 / prm->gam;
  c.inv_Re = 1.0 / prm->Re;
  c.gam_RePr = prm->gam / (prm->Re * prm->Pr);
  c.gg1_Re = prm->gam * (prm->gam - 1.0) / prm->Re;
  c.do_viscous = prm->do_viscous_terms == 1;
  c.shock_capturing = prm->shock_capturing == 1;
  c.control_forcing = (prm->control_forcing == 1 || prm->control_forcing == 2) ? (int)prm->control_forcing : 0;
  c.harm_amp = prm->harmonic_amp;
  c.harm_omega = 2.0 * 3.141592653589793 * prm->harmonic_st * prm->harmonic_uj;
  c.dt_mode = (int)prm->dt_mode;
  c.npatch = (int)npatch;

  // ---- operator tables and 1-D metrics (ModSolver.f90:57-76)
  double S1[9][6], S2[9][6], G[9][11];
  build_tables(S1, S2, G);
  std::memcpy(h->S1, S1, sizeof(S1));
  std::vector<double> z(Nz), r(Nr);
  for (int64_t i = 0; i < Nz; ++i) z[i] = zvec[i];
  for (int64_t j = 0; j < Nr; ++j) r[j] = rvec[j * Nz];
  std::vector<double> dzdxi, drdeta, dxidz(Nz), detadr(Nr), ddxidxidz, ddetadetadr;
  metric_1d(S1, z, dzdxi);
  metric_1d(S1, r, drdeta);
  for (int64_t i = 0; i < Nz; ++i) dxidz[i] = 1.0 / dzdxi[i];
  for (int64_t j = 0; j < Nr; ++j) detadr[j] = 1.0 / drdeta[j];
  metric_1d(S1, dxidz, ddxidxidz);
  metric_1d(S1, detadr, ddetadetadr);
  // deltaz, deltar and the z ramp of the sensor (ModShockCapturing.f90:171-189, :85)
  std::vector<double> dzv(Nz), drv(Nr), ramp(Nz);
  for (int64_t i = 0; i < Nz; ++i) {
    if (i >= 1 && i <= Nz - 2) dzv[i] = (z[i + 1] - z[i - 1]) / 2.0;
    if (i == 0) dzv[i] = z[1] - z[0];
    if (i == Nz - 1) dzv[i] = z[Nz - 1] - z[Nz - 2];
    ramp[i] = (1.0 + std::tanh(5.0 * (z[i] - 10.0))) / 2.0;
  }
  for (int64_t j = 0; j < Nr; ++j) {
    if (j >= 1 && j <= Nr - 2) drv[j] = (r[j + 1] - r[j - 1]) / 2.0;
    if (j == 0) drv[j] = r[1] - r[0];
    if (j == Nr - 1) drv[j] = r[Nr - 1] - r[Nr - 2];
  }

  // ---- stencil maps (CreateAllPatches, ModPatch.f90:214-242) -> per-point descriptors,
  // face-operation lists and tile classes, on the host or on the device
  std::vector<uint32_t> desc;
  std::vector<int> faces;
  std::vector<unsigned char> zcode, rcode;
  std::vector<int2> tint, tgen, sti, stg;
  int64_t iT = Nz, jT = Nr;
  {
    std::string msg;
    const int prc = prm->patch_prep == 1
                        ? device_patch_maps(patches, npatch, Nz, Nr, h->P, ibval, desc, zcode, rcode, faces, tint, tgen,
                                            sti, stg, iT, jT, msg)
                        : host_patch_maps(patches, npatch, Nz, Nr, h->P, ibval, desc, zcode, rcode, faces, tint, tgen,
                                          sti, stg, iT, jT, msg);
    if (prc != AXJ_OK) {
      delete h;
      return fail(nullptr, prc, "%s", msg.c_str());
    }
  }
  h->iT = (int)(iT - 1);
  h->jT = (int)(jT - 1);
  h->ntiles_int = (int)tint.size();
  h->ntiles_gen = (int)tgen.size();
  h->nstiles_int = (int)sti.size();
  h->nstiles_gen = (int)stg.size();

  // ---- device buffers
  cudaError_t ce = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (ce != cudaSuccess) { delete h; return fail(nullptr, AXJ_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(ce)); }
  if (cudaStreamCreateWithFlags(&h->side.stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->side.fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->side.join, cudaEventDisableTiming) != cudaSuccess) {
    g_create_error = "side stream / event creation failed";
    axj_destroy(h);
    return AXJ_ERR_CUDA;
  }
  int rc = AXJ_OK;
  const size_t pl = (size_t)h->plane;
  h->U0 = dalloc<double>(h, 5 * pl, &rc);
  h->Ua = dalloc<double>(h, 5 * pl, &rc);
  h->Ub = dalloc<double>(h, 5 * pl, &rc);
  h->mixed = prm->precision == AXJ_MIXED;
  h->int_rows = prm->stage_rows == 0 ? AXJ_DEFAULT_STAGE_ROWS : (int)prm->stage_rows;
  h->learned = prm->sensor != AXJ_SENSOR_PLAIN;
  h->held_only = prm->sensor == AXJ_SENSOR_HELD;
  h->judge_every = prm->judge_every;
  h->judge_all = prm->judge_stages != 1;
  h->judge_thr = prm->judge_threshold;
  if (c.shock_capturing) {
    // learned-sensor buffers (also used by the feature/prediction entry points)
    h->mlp = dalloc<float>(h, MLP_NPARAM, &rc);
    h->feat = dalloc<float4>(h, pl, &rc);
    h->pred = dalloc<double>(h, 2 * pl, &rc);
    h->held = dalloc<double>(h, 2 * pl, &rc);
    h->mask = dalloc<unsigned char>(h, pl, &rc);
    h->counts = dalloc<unsigned long long>(h, 2, &rc);
  }
  if (h->mixed) {
    h->Uaf = reinterpret_cast<float*>(h->Ua);
    h->Ubf = reinterpret_cast<float*>(h->Ub);
  }
  h->A = dalloc<double>(h, 5 * pl, &rc);
  h->B = dalloc<double>(h, 5 * pl, &rc);
  h->target = dalloc<double>(h, 5 * pl, &rc);
  h->star = dalloc<double>(h, 3 * pl, &rc);
  if (c.shock_capturing) {
    h->Q = dalloc<double>(h, 3 * pl, &rc);
    h->Qz = dalloc<double>(h, 3 * pl, &rc);
    h->coef = dalloc<double>(h, 3 * pl, &rc);
    h->rcode = dalloc<unsigned char>(h, pl, &rc);
  }
  h->desc = dalloc<uint32_t>(h, pl, &rc);
  h->zcode = dalloc<unsigned char>(h, pl, &rc);
  h->faces = dalloc<int>(h, faces.size(), &rc);
  h->dxidz = dalloc<double>(h, Nz, &rc);
  h->ddxidxidz = dalloc<double>(h, Nz, &rc);
  h->detadr = dalloc<double>(h, Nr, &rc);
  h->ddetadetadr = dalloc<double>(h, Nr, &rc);
  h->zc = dalloc<double>(h, Nz, &rc);
  h->rc = dalloc<double>(h, Nr, &rc);
  h->invr = dalloc<double>(h, Nr, &rc);
  h->dzv = dalloc<double>(h, Nz, &rc);
  h->drv = dalloc<double>(h, Nr, &rc);
  h->ramp = dalloc<double>(h, Nz, &rc);
  h->forcing = dalloc<double>(h, 25, &rc);
  h->dt = dalloc<double>(h, 1, &rc);
  h->staleT = dalloc<double>(h, 1, &rc);
  h->time = dalloc<double>(h, 1, &rc);
  h->harm = dalloc<double>(h, 5, &rc);
  h->flags = dalloc<int>(h, 1, &rc);

  h->counter = dalloc<unsigned int>(h, 1, &rc);
  h->dt_blocks = dt_grid_blocks();
  h->partial = dalloc<double>(h, h->dt_blocks, &rc);
  h->tiles_int = dalloc<int2>(h, std::max<size_t>(tint.size(), 1), &rc);
  h->tiles_gen = dalloc<int2>(h, std::max<size_t>(tgen.size(), 1), &rc);
  h->stiles_int = dalloc<int2>(h, std::max<size_t>(sti.size(), 1), &rc);
  h->stiles_gen = dalloc<int2>(h, std::max<size_t>(stg.size(), 1), &rc);
  if (rc != AXJ_OK) {
    g_create_error = h->err;
    axj_destroy(h);
    return rc;
  }
  auto up = [&](void* dst, const void* src, size_t bytes) {
    if (rc == AXJ_OK && bytes) {
      cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, h->stream);
      if (e != cudaSuccess) rc = fail(h, AXJ_ERR_CUDA, "upload: %s", cudaGetErrorString(e));
    }
  };
  up(h->desc, desc.data(), desc.size() * sizeof(uint32_t));
  up(h->zcode, zcode.data(), zcode.size());
  if (h->rcode) up(h->rcode, rcode.data(), rcode.size());
  up(h->faces, faces.data(), faces.size() * sizeof(int));
  up(h->dxidz, dxidz.data(), Nz * sizeof(double));
  up(h->ddxidxidz, ddxidxidz.data(), Nz * sizeof(double));
  up(h->detadr, detadr.data(), Nr * sizeof(double));
  up(h->ddetadetadr, ddetadetadr.data(), Nr * sizeof(double));
  up(h->zc, z.data(), Nz * sizeof(double));
  up(h->rc, r.data(), Nr * sizeof(double));
  std::vector<double> invr(Nr, 0.0);
  for (int64_t j = 1; j < Nr; ++j) invr[j] = 1.0 / r[j];
  up(h->invr, invr.data(), Nr * sizeof(double));
  up(h->dzv, dzv.data(), Nz * sizeof(double));
  up(h->drv, drv.data(), Nr * sizeof(double));
  up(h->ramp, ramp.data(), Nz * sizeof(double));
  up(h->forcing, prm->forcing_mat, 25 * sizeof(double));
  up(h->tiles_int, tint.data(), tint.size() * sizeof(int2));
  up(h->tiles_gen, tgen.data(), tgen.size() * sizeof(int2));
  up(h->stiles_int, sti.data(), sti.size() * sizeof(int2));
  up(h->stiles_gen, stg.data(), stg.size() * sizeof(int2));
  std::vector<PatchDev> pd(npatch > 0 ? npatch : 1);
  for (int64_t k = 0; k < npatch; ++k) { pd[k].bc = (int)patches[k].bc; pd[k].dir = (int)patches[k].bc_dir; }
  upload_tables(S1, S2, G, pd.data(), (int)npatch, h->stream);
  if (rc == AXJ_OK) {
    cudaError_t e = init_kernel_attributes();
    if (e == cudaSuccess) e = mlp_init_attributes();
    if (e != cudaSuccess) rc = fail(h, AXJ_ERR_NODEVICE, "kernel set-up failed (no sm_100a device?): %s", cudaGetErrorString(e));
  }
  if (rc == AXJ_OK) rc = build_maps(h);
  if (rc == AXJ_OK && c.shock_capturing) rc = build_zr_maps(h);
  if (rc == AXJ_OK) {
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) rc = fail(h, AXJ_ERR_CUDA, "set-up: %s", cudaGetErrorString(e));
  }
  if (rc != AXJ_OK) {
    g_create_error = h->err;
    axj_destroy(h);
    return rc;
  }
  *out = h;
  return AXJ_OK;
}

int axj_set_state(axj_handle* h, const double* pv, const double* pv_target, int64_t iteration, double time) {
  if (!h || !pv || !pv_target) return fail(h, AXJ_ERR_ARG, "null argument");
  AXJ_CUDA(h, cudaSetDevice(h->device));
  // a new state starts without the error flags of the previous one
  AXJ_CUDA(h, cudaMemsetAsync(h->flags, 0, sizeof(int), h->stream));
  AXJ_CUDA(h, h2d(h, h->U0, pv, 5));
  AXJ_CUDA(h, h2d(h, h->target, pv_target, 5));
  AXJ_CUDA(h, cudaMemcpyAsync(h->time, &time, sizeof(double), cudaMemcpyHostToDevice, h->stream));
  AXJ_CUDA(h, cudaStreamSynchronize(h->stream));
  h->iteration = iteration;
  h->time_host = time;
  h->state_set = true;
  h->judged = false;
  return AXJ_OK;
}

int axj_get_state(axj_handle* h, double* pv) {
  if (!h || !pv) return fail(h, AXJ_ERR_ARG, "null argument");
  AXJ_CUDA(h, cudaSetDevice(h->device));
  AXJ_CUDA(h, d2h(h, pv, h->U0, 5));
  AXJ_CUDA(h, cudaStreamSynchronize(h->stream));
  return AXJ_OK;
}

int axj_get_time(axj_handle* h, int64_t* iteration, double* time) {
  if (!h) return fail(h, AXJ_ERR_ARG, "null handle");
  if (iteration) *iteration = h->iteration;
  if (time) *time = h->time_host;
  return AXJ_OK;
}

int axj_compute_dt(axj_handle* h, double* delt) {
  if (!h) return fail(h, AXJ_ERR_ARG, "null handle");
  if (!h->state_set) return fail(h, AXJ_ERR_ARG, "axj_set_state has not been called");
  AXJ_CUDA(h, cudaSetDevice(h->device));
  int rc = enqueue_dt(h, 0);
  if (rc != AXJ_OK) return rc;
  double d = 0.0;
  AXJ_CUDA(h, cudaMemcpyAsync(&d, h->dt, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  rc = check_flags(h);
  if (delt) *delt = d;
  return rc;
}

int axj_rk4_step(axj_handle* h, double delt) {
  if (!h) return fail(h, AXJ_ERR_ARG, "null handle");
  if (!h->state_set) return fail(h, AXJ_ERR_ARG, "axj_set_state has not been called");
  AXJ_CUDA(h, cudaSetDevice(h->device));
  AXJ_CUDA(h, cudaMemcpyAsync(h->dt, &delt, sizeof(double), cudaMemcpyHostToDevice, h->stream));
  if (int rc0 = check_model(h)) return rc0;
  // the stages read the step's end time t_n + delt, as after the dt kernel of axj_run
  h->time_end = h->time_host + delt;
  AXJ_CUDA(h, cudaMemcpyAsync(h->time, &h->time_end, sizeof(double), cudaMemcpyHostToDevice, h->stream));
  const bool judge = judge_due(h);
  // the stages replay a captured graph (one launch instead of some thirty)
  cudaGraphExec_t ge = nullptr;
  int rc = rk4_graph(h, judge, &ge);
  if (rc != AXJ_OK) return rc;
  AXJ_CUDA(h, cudaGraphLaunch(ge, h->stream));
  if (judge) {
    h->judged = true;
    h->njudges += 1;
  }
  rc = check_flags(h);
  h->time_host = h->time_host + delt;
  h->iteration += 1;
  AXJ_CUDA(h, cudaMemcpyAsync(h->time, &h->time_host, sizeof(double), cudaMemcpyHostToDevice, h->stream));
  AXJ_CUDA(h, cudaStreamSynchronize(h->stream));
  return rc;
}

namespace {
// Output of axj_run, first use: snapshot, pinned staging, copy stream and events.
int out_setup(axj_handle* h) {
  if (h->out_snap) return AXJ_OK;
  const size_t n = (size_t)h->Nz * h->Nr * 5;
  AXJ_CUDA(h, cudaMalloc(&h->out_snap, (5 * (size_t)h->plane + 2) * sizeof(double)));
  AXJ_CUDA(h, cudaHostAlloc(&h->out_host, (n + 2) * sizeof(double), cudaHostAllocDefault));
  AXJ_CUDA(h, cudaStreamCreateWithFlags(&h->out_stream, cudaStreamNonBlocking));
  AXJ_CUDA(h, cudaEventCreateWithFlags(&h->out_snapped, cudaEventDisableTiming));
  AXJ_CUDA(h, cudaEventCreateWithFlags(&h->out_copied, cudaEventDisableTiming));
  return AXJ_OK;
}

// Snapshot of the state, time and flags after the step just enqueued (device copies in
// stream order), then the copy to pinned host memory on the output stream.
int out_snapshot(axj_handle* h) {
  const size_t n = (size_t)h->Nz * h->Nr * 5;
  double* aux = h->out_snap + 5 * (size_t)h->plane;
  AXJ_CUDA(h, cudaMemcpyAsync(h->out_snap, h->U0, 5 * (size_t)h->plane * sizeof(double), cudaMemcpyDeviceToDevice,
                              h->stream));
  AXJ_CUDA(h, cudaMemcpyAsync(aux, h->time, sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  AXJ_CUDA(h, cudaMemcpyAsync(aux + 1, h->flags, sizeof(int), cudaMemcpyDeviceToDevice, h->stream));
  AXJ_CUDA(h, cudaEventRecord(h->out_snapped, h->stream));
  AXJ_CUDA(h, cudaStreamWaitEvent(h->out_stream, h->out_snapped, 0));
  AXJ_CUDA(h, cudaMemcpy2DAsync(h->out_host, (size_t)h->Nz * sizeof(double), h->out_snap,
                                (size_t)h->P * sizeof(double), (size_t)h->Nz * sizeof(double), (size_t)h->Nr * 5,
                                cudaMemcpyDeviceToHost, h->out_stream));
  AXJ_CUDA(h, cudaMemcpyAsync(h->out_host + n, aux, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->out_stream));
  AXJ_CUDA(h, cudaEventRecord(h->out_copied, h->out_stream));
  h->out_pending = true;
  h->out_iter = h->iteration;
  return AXJ_OK;
}

// Hands the pending snapshot to the callback once its copy is complete (or reports the
// error flags it recorded).
int out_deliver(axj_handle* h, axj_output_cb cb, void* user) {
  if (!h->out_pending) return AXJ_OK;
  h->out_pending = false;
  AXJ_CUDA(h, cudaEventSynchronize(h->out_copied));
  const size_t n = (size_t)h->Nz * h->Nr * 5;
  int f = 0;
  std::memcpy(&f, h->out_host + n + 1, sizeof(int));
  if (int rc = flags_status(h, f)) return rc;
  cb(user, h->out_iter, h->out_host[n], h->out_host);
  return AXJ_OK;
}
}  // namespace

int axj_run(axj_handle* h, int64_t nsteps, int64_t out_every, axj_output_cb cb, void* user, double* last_dt) {
  if (!h) return fail(h, AXJ_ERR_ARG, "null handle");
  if (!h->state_set) return fail(h, AXJ_ERR_ARG, "axj_set_state has not been called");
  if (nsteps < 0) return fail(h, AXJ_ERR_ARG, "nsteps < 0");
  AXJ_CUDA(h, cudaSetDevice(h->device));
  {
    if (int rc = check_model(h)) return rc;
    cudaGraphExec_t ge = nullptr;
    int rc = step_graph(h, false, &ge);  // capture outside the step loop
    if (rc != AXJ_OK) return rc;
  }
  h->out_pending = false;
  for (int64_t s = 0; s < nsteps; ++s) {
    int rc = launch_step(h);
    if (rc != AXJ_OK) return rc;
    if (out_every > 0 && cb && (h->iteration % out_every == 0)) {
      // the previous output reaches the callback now (its copy ran beside the steps
      // since); this one is snapshot and copied while the next steps run
      rc = out_deliver(h, cb, user);
      if (rc == AXJ_OK) rc = out_setup(h);
      if (rc == AXJ_OK) rc = out_snapshot(h);
      if (rc != AXJ_OK) return rc;
    }
  }
  if (cb) {
    int rc = out_deliver(h, cb, user);
    if (rc != AXJ_OK) return rc;
  }
  double dlast = 0.0;
  AXJ_CUDA(h, cudaMemcpyAsync(&dlast, h->dt, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  AXJ_CUDA(h, cudaMemcpyAsync(&h->time_host, h->time, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  int rc = check_flags(h);
  if (last_dt) *last_dt = dlast;
  return rc;
}

int axj_run_timed(axj_handle* h, int64_t nsteps, double* ms) {
  if (!h || !ms) return fail(h, AXJ_ERR_ARG, "null argument");
  AXJ_CUDA(h, cudaSetDevice(h->device));
  int rc = axj_run(h, 0, 0, nullptr, nullptr, nullptr);  // builds the graph
  if (rc != AXJ_OK) return rc;
  cudaEvent_t e0, e1;
  AXJ_CUDA(h, cudaEventCreate(&e0));
  AXJ_CUDA(h, cudaEventCreate(&e1));
  if (judge_due(h)) {  // the judge graph is captured outside the timed region
    cudaGraphExec_t ge = nullptr;
    rc = step_graph(h, true, &ge);
    if (rc != AXJ_OK) return rc;
  }
  AXJ_CUDA(h, cudaEventRecord(e0, h->stream));
  for (int64_t s = 0; s < nsteps; ++s) {
    rc = launch_step(h);
    if (rc != AXJ_OK) return rc;
  }
  AXJ_CUDA(h, cudaEventRecord(e1, h->stream));
  AXJ_CUDA(h, cudaEventSynchronize(e1));
  float t = 0.f;
  AXJ_CUDA(h, cudaEventElapsedTime(&t, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = t;
  AXJ_CUDA(h, cudaMemcpyAsync(&h->time_host, h->time, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  return check_flags(h);
}

int axj_profile_steps(axj_handle* h, int64_t nsteps, double* ms, int64_t* launches) {
  if (!h || !ms) return fail(h, AXJ_ERR_ARG, "null argument");
  if (!h->state_set) return fail(h, AXJ_ERR_ARG, "axj_set_state has not been called");
  AXJ_CUDA(h, cudaSetDevice(h->device));
  cudaEvent_t ev[2];
  AXJ_CUDA(h, cudaEventCreate(&ev[0]));
  AXJ_CUDA(h, cudaEventCreate(&ev[1]));
  double acc[4] = {0, 0, 0, 0};
  int64_t nl[3] = {0, 0, 0};
  auto timed = [&](int slot, auto&& body) -> int {
    AXJ_CUDA(h, cudaEventRecord(ev[0], h->stream));
    int rc = body();
    if (rc != AXJ_OK) return rc;
    AXJ_CUDA(h, cudaEventRecord(ev[1], h->stream));
    AXJ_CUDA(h, cudaEventSynchronize(ev[1]));
    float t = 0.f;
    AXJ_CUDA(h, cudaEventElapsedTime(&t, ev[0], ev[1]));
    acc[slot] += t;
    return AXJ_OK;
  };
  const int stage_launches = (h->ntiles_gen > 0) + (h->ntiles_int > 0);
  int bufs[5];
  rk4_buffers(h, bufs);
  int rc = AXJ_OK;
  if (rc == AXJ_OK) rc = check_model(h);
  for (int64_t s = 0; s < nsteps && rc == AXJ_OK; ++s) {
    const bool judge = judge_due(h);
    rc = timed(0, [&]() -> int {
      int r = enqueue_dt(h, 1);
      if (r == AXJ_OK && h->c.control_forcing == 2)
        AXJ_CUDA(h, launch_harmonic_phase(h->time, h->dt, h->c.harm_omega, 0, h->harm, h->stream));
      return r;
    });
    nl[0] += 1 + (h->c.control_forcing == 2);
    for (int st = 1; st <= 4 && rc == AXJ_OK; ++st) {
      const bool lrn_plain = h->learned && judge && st > 1 && h->judge_all;
      const bool lrn = h->learned && !lrn_plain;
      if (lrn && h->held_only) {
        if (judge && st == 1) {
          rc = timed(1, [&]() -> int {
            SensorArgs sa = sensor_args(h, bufs[st - 1]);
            AXJ_CUDA(h, launch_sensor(sa, true, h->side, h->stream));
            return AXJ_OK;
          });
          nl[1] += (h->nstiles_int > 0) + (h->nstiles_gen > 0) + 2;
        }
      } else if (lrn && st > 1) {
        // the step's coefficients come from its first stage
      } else if (lrn) {
        // features + inference (+ plain sensor and judge at the first stage of a judge step)
        rc = timed(1, [&]() -> int {
          AXJ_CUDA(h, launch_features(feat_args(h, bufs[st - 1]), h->stream));
          if (judge && st == 1) {
            SensorArgs sa = sensor_args(h, bufs[st - 1]);
            AXJ_CUDA(h, launch_sensor(sa, true, h->side, h->stream));
            AXJ_CUDA(h, launch_mlp_infer(infer_args(h, 0), h->stream));
            JudgeArgs j{grid_of(h), h->pred, h->star + h->plane, h->judge_thr, h->mask, h->held, h->counts};
            AXJ_CUDA(h, launch_judge(j, h->stream));
          } else {
            AXJ_CUDA(h, launch_mlp_infer(infer_args(h, 1), h->stream));
          }
          return AXJ_OK;
        });
        nl[1] += 2 + ((judge && st == 1) ? (h->nstiles_int > 0) + (h->nstiles_gen > 0) + 4 : 0);
      } else if (h->c.shock_capturing) {
        rc = timed(1, [&]() -> int { return enqueue_sensor_chain(h, bufs[st - 1]); });
        nl[1] += (h->nstiles_int > 0) + (h->nstiles_gen > 0) + 1;
      }
      if (rc != AXJ_OK) break;
      const int cm = lrn ? CM_LRN : (h->c.shock_capturing ? CM_PRE : CM_FILT);
      rc = timed(2, [&]() -> int { return launch_stage_kernels(h, bufs[st - 1], bufs[st], st, cm); });
      nl[2] += stage_launches;
    }
    if (judge) {
      h->judged = true;
      h->njudges += 1;
    }
    h->iteration += 1;
  }
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  if (rc != AXJ_OK) return rc;
  acc[3] = acc[0] + acc[1] + acc[2];
  for (int k = 0; k < 4; ++k) ms[k] = acc[k];
  if (launches)
    for (int k = 0; k < 3; ++k) launches[k] = nl[k];
  AXJ_CUDA(h, cudaMemcpyAsync(&h->time_host, h->time, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  return check_flags(h);
}

int axj_rhs(axj_handle* h, const double* pv, double* rhs) {
  if (!h || !pv || !rhs) return fail(h, AXJ_ERR_ARG, "null argument");
  if (!h->state_set) return fail(h, AXJ_ERR_ARG, "axj_set_state has not been called (the target is needed)");
  AXJ_CUDA(h, cudaSetDevice(h->device));
  AXJ_CUDA(h, h2d(h, h->Ua, pv, 5));
  if (h->c.control_forcing == 2)
    AXJ_CUDA(h, launch_harmonic_phase(h->time, h->dt, h->c.harm_omega, 1, h->harm, h->stream));
  int rc = enqueue_stage(h, BUA, BUB, 0);
  if (rc != AXJ_OK) return rc;
  AXJ_CUDA(h, d2h(h, rhs, h->Ub, 5));
  AXJ_CUDA(h, cudaStreamSynchronize(h->stream));
  return AXJ_OK;
}

int axj_deriv1(axj_handle* h, const double* var, int64_t dirn, double* out) {
  if (!h || !var || !out || (dirn != 1 && dirn != 2)) return fail(h, AXJ_ERR_ARG, "bad argument");
  AXJ_CUDA(h, cudaSetDevice(h->device));
  AXJ_CUDA(h, h2d(h, h->Ua, var, 1));
  AXJ_CUDA(h, launch_deriv(grid_of(h), h->desc, h->Ua, nullptr, dirn == 1 ? h->dxidz : h->detadr, nullptr, (int)dirn,
                           1, h->Ub, h->stream));
  AXJ_CUDA(h, d2h(h, out, h->Ub, 1));
  AXJ_CUDA(h, cudaStreamSynchronize(h->stream));
  return AXJ_OK;
}

int axj_deriv2(axj_handle* h, const double* var, int64_t dirn, const double* first, double* out) {
  if (!h || !var || !out || !first || (dirn != 1 && dirn != 2)) return fail(h, AXJ_ERR_ARG, "bad argument");
  AXJ_CUDA(h, cudaSetDevice(h->device));
  AXJ_CUDA(h, h2d(h, h->Ua, var, 1));
  AXJ_CUDA(h, h2d(h, h->Ua + h->plane, first, 1));
  AXJ_CUDA(h, launch_deriv(grid_of(h), h->desc, h->Ua, h->Ua + h->plane, dirn == 1 ? h->dxidz : h->detadr,
                           dirn == 1 ? h->ddxidxidz : h->ddetadetadr, (int)dirn, 2, h->Ub, h->stream));
  AXJ_CUDA(h, d2h(h, out, h->Ub, 1));
  AXJ_CUDA(h, cudaStreamSynchronize(h->stream));
  return AXJ_OK;
}

int axj_tgfilter(axj_handle* h, const double* var, int64_t dirn, int64_t inplace, double* out) {
  if (!h || !out || (dirn != 1 && dirn != 2) || (!inplace && !var)) return fail(h, AXJ_ERR_ARG, "bad argument");
  if (inplace && dirn != 1) return fail(h, AXJ_ERR_UNSUPPORTED, "in-place filtering is only defined along z");
  AXJ_CUDA(h, cudaSetDevice(h->device));
  AXJ_CUDA(h, h2d(h, h->Ub, out, 1));
  if (inplace) {
    AXJ_CUDA(h, launch_tgfilter_z_inplace(grid_of(h), h->desc, h->zcode, h->Ub, h->Ua, 1, h->flags, h->stream));
    AXJ_CUDA(h, d2h(h, out, h->Ua, 1));
  } else {
    AXJ_CUDA(h, h2d(h, h->Ua, var, 1));
    AXJ_CUDA(h, launch_tgfilter(grid_of(h), h->desc, h->Ua, (int)dirn, h->Ub, h->stream));
    AXJ_CUDA(h, d2h(h, out, h->Ub, 1));
  }
  AXJ_CUDA(h, cudaStreamSynchronize(h->stream));
  return AXJ_OK;
}

int axj_sensor(axj_handle* h, const double* pv, double* mustar, double* betastar, double* kappastar) {
  if (!h || !pv || !mustar || !betastar || !kappastar) return fail(h, AXJ_ERR_ARG, "null argument");
  if (!h->c.shock_capturing) return fail(h, AXJ_ERR_ARG, "handle created with shock_capturing = 0");
  AXJ_CUDA(h, cudaSetDevice(h->device));
  AXJ_CUDA(h, h2d(h, h->Ua, pv, 5));
  SensorArgs s = sensor_args(h, BUA);
  AXJ_CUDA(h, launch_sensor(s, true, h->side, h->stream));
  h->judged = false;  // the coefficient planes (the learned sensor's held mu*) were overwritten
  AXJ_CUDA(h, d2h(h, mustar, h->star, 1));
  AXJ_CUDA(h, d2h(h, betastar, h->star + h->plane, 1));
  AXJ_CUDA(h, d2h(h, kappastar, h->star + 2 * h->plane, 1));
  AXJ_CUDA(h, cudaStreamSynchronize(h->stream));
  return AXJ_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Learned sensor: model, data set, training, checks
// ---------------------------------------------------------------------------
namespace {

void mlp_to_flat(const axj_mlp* m, std::vector<float>& flat, MlpNorm* norm) {
  flat.assign(MLP_NPARAM, 0.0f);
  for (int n = 0; n < MLP_HID; ++n)
    for (int k = 0; k < MLP_IN; ++k) flat[MLP_OFF_W1 + n * MLP_K1 + k] = m->w1[n * MLP_IN + k];
  for (int n = 0; n < MLP_HID; ++n) flat[MLP_OFF_B1 + n] = m->b1[n];
  for (int e = 0; e < MLP_HID * MLP_HID; ++e) flat[MLP_OFF_W2 + e] = m->w2[e];
  for (int n = 0; n < MLP_HID; ++n) flat[MLP_OFF_B2 + n] = m->b2[n];
  for (int e = 0; e < MLP_OUT * MLP_HID; ++e) flat[MLP_OFF_W3 + e] = m->w3[e];
  for (int n = 0; n < MLP_OUT; ++n) flat[MLP_OFF_B3 + n] = m->b3[n];
  if (norm) {
    for (int c = 0; c < MLP_CH; ++c) {
      norm->feat_mean[c] = m->feat_mean[c];
      norm->feat_inv_scale[c] = 1.0f / m->feat_scale[c];
    }
    for (int k = 0; k < MLP_OUT; ++k) norm->out_scale[k] = m->out_scale[k];
  }
}

void flat_to_mlp(const std::vector<float>& flat, const MlpNorm* norm, axj_mlp* m) {
  std::memset(m, 0, sizeof(*m));
  for (int n = 0; n < MLP_HID; ++n)
    for (int k = 0; k < MLP_IN; ++k) m->w1[n * MLP_IN + k] = flat[MLP_OFF_W1 + n * MLP_K1 + k];
  for (int n = 0; n < MLP_HID; ++n) m->b1[n] = flat[MLP_OFF_B1 + n];
  for (int e = 0; e < MLP_HID * MLP_HID; ++e) m->w2[e] = flat[MLP_OFF_W2 + e];
  for (int n = 0; n < MLP_HID; ++n) m->b2[n] = flat[MLP_OFF_B2 + n];
  for (int e = 0; e < MLP_OUT * MLP_HID; ++e) m->w3[e] = flat[MLP_OFF_W3 + e];
  for (int n = 0; n < MLP_OUT; ++n) m->b3[n] = flat[MLP_OFF_B3 + n];
  if (norm) {
    for (int c = 0; c < MLP_CH; ++c) {
      m->feat_mean[c] = norm->feat_mean[c];
      m->feat_scale[c] = 1.0f / norm->feat_inv_scale[c];
    }
    for (int k = 0; k < MLP_OUT; ++k) m->out_scale[k] = norm->out_scale[k];
  }
}

int need_mlp_buffers(axj_handle* h) {
  if (!h->mlp) return fail(h, AXJ_ERR_ARG, "handle created with shock_capturing = 0 (no sensor to learn)");
  return AXJ_OK;
}

// Forward and backward workspace of one batch (row-major, batch-major).
struct TrainWs {
  int B = 0;
  float *X = nullptr, *T = nullptr, *Z1 = nullptr, *H1 = nullptr, *Z2 = nullptr, *H2 = nullptr, *Y = nullptr,
        *dY = nullptr, *dH2 = nullptr, *dH1 = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr, *loss = nullptr;
  int* step = nullptr;
  std::vector<void*> mem;
  ~TrainWs() {
    for (void* p : mem) cudaFree(p);
  }
  template <typename T_>
  T_* get(size_t n, cudaError_t* e) {
    void* p = nullptr;
    if (*e == cudaSuccess) *e = cudaMalloc(&p, n * sizeof(T_) + 16);
    if (*e == cudaSuccess) {
      mem.push_back(p);
      *e = cudaMemset(p, 0, n * sizeof(T_) + 16);
    }
    return static_cast<T_*>(p);
  }
  cudaError_t alloc(int B_, int nloss) {
    B = B_;
    cudaError_t e = cudaSuccess;
    const size_t b = (size_t)B;
    X = get<float>(b * MLP_K1, &e);
    T = get<float>(b * MLP_OUT, &e);
    Z1 = get<float>(b * MLP_HID, &e);
    H1 = get<float>(b * MLP_HID, &e);
    Z2 = get<float>(b * MLP_HID, &e);
    H2 = get<float>(b * MLP_HID, &e);
    Y = get<float>(b * MLP_OUT, &e);
    dY = get<float>(b * MLP_OUT, &e);
    dH2 = get<float>(b * MLP_HID, &e);
    dH1 = get<float>(b * MLP_HID, &e);
    grad = get<float>(MLP_NPARAM, &e);
    m = get<float>(MLP_NPARAM, &e);
    v = get<float>(MLP_NPARAM, &e);
    loss = get<float>((size_t)(nloss > 0 ? nloss : 1), &e);
    step = get<int>(1, &e);
    return e;
  }
};

// Forward and backward pass over ws.X / ws.T; gradients (all parameters) into ws.grad,
// the batch loss added to ws.loss[*ws.step].
int forward_backward(axj_handle* h, TrainWs& w) {
  const int B = w.B;
  const float* P = h->mlp;
  float* G = w.grad;
  cudaStream_t s = h->stream;
  const int ks = B >= 2048 ? B / 1024 : 1;
  AXJ_CUDA(h, launch_gemm(false, true, B, MLP_HID, MLP_K1, w.X, MLP_K1, P + MLP_OFF_W1, MLP_K1, w.Z1, MLP_HID, 1, s));
  AXJ_CUDA(h, launch_bias_gelu(w.Z1, P + MLP_OFF_B1, w.H1, B, MLP_HID, s));
  AXJ_CUDA(h, launch_gemm(false, true, B, MLP_HID, MLP_HID, w.H1, MLP_HID, P + MLP_OFF_W2, MLP_HID, w.Z2, MLP_HID, 1, s));
  AXJ_CUDA(h, launch_bias_gelu(w.Z2, P + MLP_OFF_B2, w.H2, B, MLP_HID, s));
  AXJ_CUDA(h, launch_gemm(false, true, B, MLP_OUT, MLP_HID, w.H2, MLP_HID, P + MLP_OFF_W3, MLP_HID, w.Y, MLP_OUT, 1, s));
  AXJ_CUDA(h, launch_bias(w.Y, P + MLP_OFF_B3, B, MLP_OUT, s));
  AXJ_CUDA(h, launch_loss(w.Y, w.T, w.dY, w.loss, w.step, B, s));
  AXJ_CUDA(h, cudaMemsetAsync(G, 0, sizeof(float) * MLP_NPARAM, s));
  AXJ_CUDA(h, launch_gemm(true, false, MLP_OUT, MLP_HID, B, w.dY, MLP_OUT, w.H2, MLP_HID, G + MLP_OFF_W3, MLP_HID, ks, s));
  AXJ_CUDA(h, launch_colsum(w.dY, G + MLP_OFF_B3, B, MLP_OUT, s));
  AXJ_CUDA(h, launch_gemm(false, false, B, MLP_HID, MLP_OUT, w.dY, MLP_OUT, P + MLP_OFF_W3, MLP_HID, w.dH2, MLP_HID, 1, s));
  AXJ_CUDA(h, launch_gelu_bwd(w.dH2, w.Z2, B * MLP_HID, s));
  AXJ_CUDA(h, launch_gemm(true, false, MLP_HID, MLP_HID, B, w.dH2, MLP_HID, w.H1, MLP_HID, G + MLP_OFF_W2, MLP_HID, ks, s));
  AXJ_CUDA(h, launch_colsum(w.dH2, G + MLP_OFF_B2, B, MLP_HID, s));
  AXJ_CUDA(h, launch_gemm(false, false, B, MLP_HID, MLP_HID, w.dH2, MLP_HID, P + MLP_OFF_W2, MLP_HID, w.dH1, MLP_HID, 1, s));
  AXJ_CUDA(h, launch_gelu_bwd(w.dH1, w.Z1, B * MLP_HID, s));
  AXJ_CUDA(h, launch_gemm(true, false, MLP_HID, MLP_K1, B, w.dH1, MLP_HID, w.X, MLP_K1, G + MLP_OFF_W1, MLP_K1, ks, s));
  AXJ_CUDA(h, launch_colsum(w.dH1, G + MLP_OFF_B1, B, MLP_HID, s));
  return AXJ_OK;
}

Dataset dataset_of(axj_handle* h) {
  Dataset d;
  d.feat = h->ds_feat;
  d.targ = h->ds_targ;
  d.S = (int)h->ds_n;
  d.g = grid_of(h);
  return d;
}

uint64_t host_mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

}  // namespace

extern "C" {

void axj_default_train_cfg(axj_train_cfg* c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->steps = 2000;
  c->batch = 65536;
  c->lr = 1e-3;
  c->beta1 = 0.9;
  c->beta2 = 0.999;
  c->eps = 1e-8;
  c->seed = 1;
  c->fit_normalization = 1;
}

void axj_mlp_init(axj_mlp* m, int64_t seed) {
  if (!m) return;
  std::memset(m, 0, sizeof(*m));
  uint64_t state = (uint64_t)seed;
  auto uni = [&](double bound) {
    state = host_mix64(state);
    const double u = (double)(state >> 11) * (1.0 / 9007199254740992.0);
    return (float)((2.0 * u - 1.0) * bound);
  };
  const double b1 = 1.0 / std::sqrt((double)MLP_IN), b2 = 1.0 / std::sqrt((double)MLP_HID);
  for (int e = 0; e < MLP_HID * MLP_IN; ++e) m->w1[e] = uni(b1);
  for (int e = 0; e < MLP_HID; ++e) m->b1[e] = uni(b1);
  for (int e = 0; e < MLP_HID * MLP_HID; ++e) m->w2[e] = uni(b2);
  for (int e = 0; e < MLP_HID; ++e) m->b2[e] = uni(b2);
  for (int e = 0; e < MLP_OUT * MLP_HID; ++e) m->w3[e] = uni(b2);
  for (int e = 0; e < MLP_OUT; ++e) m->b3[e] = uni(b2);
  for (int c = 0; c < MLP_CH; ++c) m->feat_scale[c] = 1.0f;
  for (int k = 0; k < MLP_OUT; ++k) m->out_scale[k] = 1.0f;
}

int axj_mlp_set(axj_handle* h, const axj_mlp* m) {
  if (!h || !m) return fail(h, AXJ_ERR_ARG, "null argument");
  if (int rc = need_mlp_buffers(h)) return rc;
  for (int c = 0; c < MLP_CH; ++c)
    if (!(m->feat_scale[c] > 0.0f) || !std::isfinite(m->feat_mean[c]))
      return fail(h, AXJ_ERR_ARG, "feature normalisation of channel %d is not positive and finite", c);
  for (int k = 0; k < MLP_OUT; ++k)
    if (!std::isfinite(m->out_scale[k])) return fail(h, AXJ_ERR_ARG, "out_scale[%d] is not finite", k);
  AXJ_CUDA(h, cudaSetDevice(h->device));
  std::vector<float> flat;
  drop_graphs(h);
  mlp_to_flat(m, flat, &h->norm);
  AXJ_CUDA(h, cudaMemcpyAsync(h->mlp, flat.data(), sizeof(float) * MLP_NPARAM, cudaMemcpyHostToDevice, h->stream));
  AXJ_CUDA(h, cudaStreamSynchronize(h->stream));
  h->mlp_set = true;
  h->judged = false;
  return AXJ_OK;
}

int axj_mlp_get(axj_handle* h, axj_mlp* m) {
  if (!h || !m) return fail(h, AXJ_ERR_ARG, "null argument");
  if (int rc = need_mlp_buffers(h)) return rc;
  AXJ_CUDA(h, cudaSetDevice(h->device));
  std::vector<float> flat(MLP_NPARAM);
  AXJ_CUDA(h, cudaMemcpyAsync(flat.data(), h->mlp, sizeof(float) * MLP_NPARAM, cudaMemcpyDeviceToHost, h->stream));
  AXJ_CUDA(h, cudaStreamSynchronize(h->stream));
  flat_to_mlp(flat, &h->norm, m);
  return AXJ_OK;
}

int axj_dataset_reserve(axj_handle* h, int64_t nsnapshots) {
  if (!h || nsnapshots < 1) return fail(h, AXJ_ERR_ARG, "bad argument");
  if (int rc = need_mlp_buffers(h)) return rc;
  AXJ_CUDA(h, cudaSetDevice(h->device));
  AXJ_CUDA(h, cudaStreamSynchronize(h->stream));
  if (h->ds_feat) cudaFree(h->ds_feat);
  if (h->ds_targ) cudaFree(h->ds_targ);
  h->ds_feat = nullptr;
  h->ds_targ = nullptr;
  h->ds_cap = h->ds_n = 0;
  const size_t n = (size_t)nsnapshots * (size_t)h->plane;
  cudaError_t e = cudaMalloc(&h->ds_feat, n * sizeof(float4));
  if (e == cudaSuccess) e = cudaMalloc(&h->ds_targ, n * sizeof(float2));
  if (e != cudaSuccess) {
    if (h->ds_feat) cudaFree(h->ds_feat);
    h->ds_feat = nullptr;
    h->ds_targ = nullptr;
    return fail(h, AXJ_ERR_NOMEM, "data set of %lld snapshots: %s", (long long)nsnapshots, cudaGetErrorString(e));
  }
  h->ds_cap = nsnapshots;
  return AXJ_OK;
}

int axj_dataset_add(axj_handle* h) {
  if (!h) return fail(h, AXJ_ERR_ARG, "null handle");
  if (int rc = need_mlp_buffers(h)) return rc;
  if (!h->state_set) return fail(h, AXJ_ERR_ARG, "axj_set_state has not been called");
  if (h->ds_n >= h->ds_cap) return fail(h, AXJ_ERR_ARG, "data set full (%lld snapshots)", (long long)h->ds_cap);
  AXJ_CUDA(h, cudaSetDevice(h->device));
  const size_t off = (size_t)h->ds_n * (size_t)h->plane;
  FeatArgs f = feat_args(h, BU0);
  f.feat = h->ds_feat + off;
  AXJ_CUDA(h, launch_features(f, h->stream));
  SensorArgs sa = sensor_args(h, BU0);
  sa.ramp_off = 1;  // the network predicts the coefficients before the z ramp
  AXJ_CUDA(h, launch_sensor(sa, true, h->side, h->stream));
  AXJ_CUDA(h, launch_pack_targets(grid_of(h), h->star, h->ds_targ + off, h->stream));
  AXJ_CUDA(h, cudaStreamSynchronize(h->stream));
  h->ds_n += 1;
  h->judged = false;  // the coefficient planes were overwritten
  return check_flags(h);
}

int axj_dataset_size(axj_handle* h, int64_t* n) {
  if (!h || !n) return fail(h, AXJ_ERR_ARG, "null argument");
  *n = h->ds_n;
  return AXJ_OK;
}

int axj_dataset_sample(axj_handle* h, int64_t batch, int64_t seed, int64_t step, float* X, float* T) {
  if (!h || !X || !T || batch < 1 || step < 0) return fail(h, AXJ_ERR_ARG, "bad argument");
  if (h->ds_n < 1) return fail(h, AXJ_ERR_ARG, "empty data set");
  AXJ_CUDA(h, cudaSetDevice(h->device));
  TrainWs w;
  AXJ_CUDA(h, w.alloc((int)batch, 1));
  const int st = (int)step;
  AXJ_CUDA(h, cudaMemcpyAsync(w.step, &st, sizeof(int), cudaMemcpyHostToDevice, h->stream));
  AXJ_CUDA(h, launch_sample(dataset_of(h), h->norm, (unsigned long long)seed, w.step, (int)batch, w.X, w.T, h->stream));
  std::vector<float> xb((size_t)batch * MLP_K1);
  AXJ_CUDA(h, cudaMemcpyAsync(xb.data(), w.X, xb.size() * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  AXJ_CUDA(h, cudaMemcpyAsync(T, w.T, (size_t)batch * MLP_OUT * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  AXJ_CUDA(h, cudaStreamSynchronize(h->stream));
  for (int64_t b = 0; b < batch; ++b)
    for (int k = 0; k < MLP_IN; ++k) X[b * MLP_IN + k] = xb[b * MLP_K1 + k];
  return AXJ_OK;
}

int axj_mlp_grad(axj_handle* h, const float* X, const float* T, int64_t batch, axj_mlp* grad, float* loss) {
  if (!h || !X || !T || !grad || batch < 1) return fail(h, AXJ_ERR_ARG, "bad argument");
  if (int rc = need_mlp_buffers(h)) return rc;
  AXJ_CUDA(h, cudaSetDevice(h->device));
  TrainWs w;
  AXJ_CUDA(h, w.alloc((int)batch, 1));
  std::vector<float> xb((size_t)batch * MLP_K1, 0.0f);
  for (int64_t b = 0; b < batch; ++b)
    for (int k = 0; k < MLP_IN; ++k) xb[b * MLP_K1 + k] = X[b * MLP_IN + k];
  AXJ_CUDA(h, cudaMemcpyAsync(w.X, xb.data(), xb.size() * sizeof(float), cudaMemcpyHostToDevice, h->stream));
  AXJ_CUDA(h, cudaMemcpyAsync(w.T, T, (size_t)batch * MLP_OUT * sizeof(float), cudaMemcpyHostToDevice, h->stream));
  int rc = forward_backward(h, w);
  if (rc != AXJ_OK) return rc;
  std::vector<float> g(MLP_NPARAM);
  float l = 0.0f;
  AXJ_CUDA(h, cudaMemcpyAsync(g.data(), w.grad, sizeof(float) * MLP_NPARAM, cudaMemcpyDeviceToHost, h->stream));
  AXJ_CUDA(h, cudaMemcpyAsync(&l, w.loss, sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  AXJ_CUDA(h, cudaStreamSynchronize(h->stream));
  flat_to_mlp(g, nullptr, grad);
  if (loss) *loss = l;
  return AXJ_OK;
}

int axj_mlp_train(axj_handle* h, const axj_train_cfg* cfg, float* loss) {
  if (!h || !cfg || cfg->steps < 0 || cfg->batch < 1 || cfg->batch > (1 << 24))
    return fail(h, AXJ_ERR_ARG, "bad argument");
  if (int rc = need_mlp_buffers(h)) return rc;
  if (h->ds_n < 1) return fail(h, AXJ_ERR_ARG, "empty data set (axj_dataset_add)");
  if (!h->mlp_set) return fail(h, AXJ_ERR_ARG, "no initial model (axj_mlp_set)");
  AXJ_CUDA(h, cudaSetDevice(h->device));
  if (cfg->fit_normalization) {
    double* acc = nullptr;
    AXJ_CUDA(h, cudaMalloc(&acc, 11 * sizeof(double)));
    cudaMemsetAsync(acc, 0, 11 * sizeof(double), h->stream);
    cudaError_t e = launch_dataset_stats(dataset_of(h), acc, h->stream);
    double a[11];
    if (e == cudaSuccess) e = cudaMemcpyAsync(a, acc, sizeof(a), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(acc);
    if (e != cudaSuccess) return fail(h, AXJ_ERR_CUDA, "data set statistics: %s", cudaGetErrorString(e));
    const double n = a[10];
    for (int c = 0; c < MLP_CH; ++c) {
      const double mean = a[c] / n;
      const double var = std::max(a[4 + c] / n - mean * mean, 0.0);
      const double sd = std::sqrt(var);
      h->norm.feat_mean[c] = (float)mean;
      h->norm.feat_inv_scale[c] = (float)(sd > 1e-30 ? 1.0 / sd : 1.0);
    }
    for (int k = 0; k < MLP_OUT; ++k) {
      const double rms = std::sqrt(a[8 + k] / n);
      h->norm.out_scale[k] = (float)(rms > 1e-30 ? rms : 1.0);
    }
    drop_graphs(h);
  }
  TrainWs w;
  AXJ_CUDA(h, w.alloc((int)cfg->batch, (int)std::max<int64_t>(cfg->steps, 1)));
  const Dataset d = dataset_of(h);
  for (int64_t it = 0; it < cfg->steps; ++it) {
    AXJ_CUDA(h, launch_sample(d, h->norm, (unsigned long long)cfg->seed, w.step, w.B, w.X, w.T, h->stream));
    int rc = forward_backward(h, w);
    if (rc != AXJ_OK) return rc;
    AXJ_CUDA(h, launch_adam(h->mlp, w.grad, w.m, w.v, MLP_NPARAM, w.step, (float)cfg->lr, (float)cfg->beta1,
                            (float)cfg->beta2, (float)cfg->eps, h->stream));
    AXJ_CUDA(h, launch_step_inc(w.step, h->stream));
  }
  if (loss && cfg->steps > 0)
    AXJ_CUDA(h, cudaMemcpyAsync(loss, w.loss, sizeof(float) * cfg->steps, cudaMemcpyDeviceToHost, h->stream));
  AXJ_CUDA(h, cudaStreamSynchronize(h->stream));
  h->judged = false;
  return AXJ_OK;
}

int axj_mlp_features(axj_handle* h, const double* pv, float* feat) {
  if (!h || !pv || !feat) return fail(h, AXJ_ERR_ARG, "null argument");
  if (int rc = need_mlp_buffers(h)) return rc;
  AXJ_CUDA(h, cudaSetDevice(h->device));
  AXJ_CUDA(h, h2d(h, h->Ua, pv, 5));
  AXJ_CUDA(h, launch_features(feat_args(h, BUA), h->stream));
  std::vector<float4> f((size_t)h->plane);
  AXJ_CUDA(h, cudaMemcpyAsync(f.data(), h->feat, f.size() * sizeof(float4), cudaMemcpyDeviceToHost, h->stream));
  AXJ_CUDA(h, cudaStreamSynchronize(h->stream));
  const size_t np = (size_t)h->Nz * h->Nr;
  for (int j = 0; j < h->Nr; ++j)
    for (int i = 0; i < h->Nz; ++i) {
      const float4 v = f[(size_t)j * h->P + i];
      const size_t o = (size_t)j * h->Nz + i;
      feat[o] = v.x;
      feat[np + o] = v.y;
      feat[2 * np + o] = v.z;
      feat[3 * np + o] = v.w;
    }
  return AXJ_OK;
}

int axj_mlp_predict(axj_handle* h, const double* pv, double* betastar, double* kappastar) {
  if (!h || !pv || !betastar || !kappastar) return fail(h, AXJ_ERR_ARG, "null argument");
  if (int rc = need_mlp_buffers(h)) return rc;
  if (!h->mlp_set) return fail(h, AXJ_ERR_ARG, "no model (axj_mlp_set)");
  AXJ_CUDA(h, cudaSetDevice(h->device));
  AXJ_CUDA(h, h2d(h, h->Ua, pv, 5));
  AXJ_CUDA(h, launch_features(feat_args(h, BUA), h->stream));
  AXJ_CUDA(h, launch_mlp_infer(infer_args(h, 0), h->stream));
  AXJ_CUDA(h, d2h(h, betastar, h->pred, 1));
  AXJ_CUDA(h, d2h(h, kappastar, h->pred + h->plane, 1));
  AXJ_CUDA(h, cudaStreamSynchronize(h->stream));
  return check_flags(h);
}

int axj_learned_stats(axj_handle* h, int64_t* judged, int64_t* fallback, int64_t* njudges) {
  if (!h) return fail(h, AXJ_ERR_ARG, "null handle");
  if (int rc = need_mlp_buffers(h)) return rc;
  AXJ_CUDA(h, cudaSetDevice(h->device));
  unsigned long long c[2] = {0, 0};
  AXJ_CUDA(h, cudaMemcpyAsync(c, h->counts, sizeof(c), cudaMemcpyDeviceToHost, h->stream));
  AXJ_CUDA(h, cudaStreamSynchronize(h->stream));
  if (judged) *judged = (int64_t)c[0];
  if (fallback) *fallback = (int64_t)c[1];
  if (njudges) *njudges = h->njudges;
  return AXJ_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batches: many solver instances advanced together, every kernel of the step launched
// once for all of them (persistent grid-stride kernels over per-instance tile tables,
// per-instance arguments and tensor maps in device tables), the step captured in a
// CUDA graph.
// ---------------------------------------------------------------------------
struct axj_batch {
  int n = 0;
  int device = 0;
  std::vector<axj_handle*> h;
  cudaStream_t stream = nullptr;
  SideStream side{nullptr, nullptr, nullptr};
  std::string err;
  std::vector<void*> mem;
  bool mixed = false, learned = false, held_only = false, sc = false, any_harm = false, judge_all = true;
  int64_t iteration = 0, judge_every = 50, njudges = 0;
  // device tables
  CUtensorMap* maps = nullptr;
  StageArgs* stage_argv[3][5] = {};  // coefficient box CM_FILT, CM_LRN, CM_PRE
  SensorArgs* sens_argv[5] = {};
  FeatArgs* feat_argv = nullptr;
  InferArgs* infer_argv[2] = {};
  JudgeArgs* judge_argv = nullptr;
  DtArgs* dt_argv = nullptr;
  HarmArgs* harm_argv = nullptr;
  // host copies of instance 0's arguments (dispatch decisions, model pointer)
  StageArgs a0_stage[3][5];
  // the fused z/r filter of the plain sensor: per-instance arguments, (segment, row block,
  // instance) work items
  ZrArgs* zr_argv = nullptr;
  int4* zr_items = nullptr;
  int nzr_items = 0;
  SensorArgs a0_sens[5];
  InferArgs a0_infer[2];
  // host tile lists (i0, j0, instance) and their device copies
  std::vector<int4> h_st_int, h_st_gen, h_se_int, h_se_gen, h_ft, h_mt, h_st_half;
  int4 *st_int = nullptr, *st_gen = nullptr, *se_int = nullptr, *se_gen = nullptr, *ft = nullptr, *mt = nullptr;
  int4* st_half = nullptr;  // the interior stage tiles as half tiles of TR / 2 rows
  int2* zrows = nullptr;
  int nzrows = 0, zthreads = 32;
  size_t zsmem = 0;
  long long max_pts = 0;
  int dt_blocks = 1, nsm = 148;
  axj_batch_tuning tune{};
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};  // normal step, judge step
  cudaGraph_t graph[2] = {nullptr, nullptr};
};

namespace {

int bfail(axj_batch* b, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (b) b->err = buf;
  else g_create_error = buf;
  return code;
}

#define BATCH_CUDA(b, call)                                                                                \
  do {                                                                                                     \
    cudaError_t e_ = (call);                                                                               \
    if (e_ != cudaSuccess) return bfail((b), AXJ_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

template <typename T>
int bupload(axj_batch* b, T** dst, const std::vector<T>& v) {
  void* p = nullptr;
  const size_t bytes = std::max<size_t>(v.size(), 1) * sizeof(T);
  BATCH_CUDA(b, cudaMalloc(&p, bytes));
  b->mem.push_back(p);
  if (!v.empty()) BATCH_CUDA(b, cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  *dst = static_cast<T*>(p);
  return AXJ_OK;
}

template <typename T>
int bupdate(axj_batch* b, T* dst, const std::vector<T>& v) {
  if (!v.empty()) BATCH_CUDA(b, cudaMemcpy(dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return AXJ_OK;
}

std::vector<int2> download_tiles(const int2* d, int n) {
  std::vector<int2> v((size_t)std::max(n, 0));
  if (n > 0) cudaMemcpy(v.data(), d, v.size() * sizeof(int2), cudaMemcpyDeviceToHost);
  return v;
}

// Tile list of all instances in the tuning's order: instance after instance, or
// round-robin over the instances (tile k of every instance in turn).
std::vector<int4> order_tiles(const std::vector<std::vector<int2>>& per, int order) {
  std::vector<int4> out;
  size_t total = 0, mx = 0;
  for (const auto& v : per) {
    total += v.size();
    mx = std::max(mx, v.size());
  }
  out.reserve(total);
  if (order == 0) {
    for (size_t k = 0; k < per.size(); ++k)
      for (const int2& t : per[k]) out.push_back(make_int4(t.x, t.y, (int)k, 0));
  } else {
    for (size_t q = 0; q < mx; ++q)
      for (size_t k = 0; k < per.size(); ++k)
        if (q < per[k].size()) out.push_back(make_int4(per[k][q].x, per[k][q].y, (int)k, 0));
  }
  return out;
}

std::vector<std::vector<int2>> block_tiles(const axj_batch* b, int tz, int tr) {
  std::vector<std::vector<int2>> per(b->n);
  for (int k = 0; k < b->n; ++k)
    for (int j = 0; j < b->h[k]->Nr; j += tr)
      for (int i = 0; i < b->h[k]->Nz; i += tz) per[k].push_back(make_int2(i, j));
  return per;
}

// (Re)build the ordered tile tables of the batch for its tuning.
int batch_tiles(axj_batch* b, bool first) {
  std::vector<std::vector<int2>> si(b->n), sg(b->n), ei(b->n), eg(b->n);
  for (int k = 0; k < b->n; ++k) {
    axj_handle* h = b->h[k];
    si[k] = download_tiles(h->tiles_int, h->ntiles_int);
    sg[k] = download_tiles(h->tiles_gen, h->ntiles_gen);
    ei[k] = download_tiles(h->stiles_int, h->nstiles_int);
    eg[k] = download_tiles(h->stiles_gen, h->nstiles_gen);
  }
  const int o = (int)b->tune.tile_order;
  b->h_st_int = order_tiles(si, o);
  std::vector<std::vector<int2>> sh(b->n);
  for (int k = 0; k < b->n; ++k)
    for (const int2& t : si[k]) {
      sh[k].push_back(t);
      sh[k].push_back(make_int2(t.x, t.y + TR / 2));
    }
  b->h_st_half = order_tiles(sh, o);
  b->h_st_gen = order_tiles(sg, o);
  b->h_se_int = order_tiles(ei, o);
  b->h_se_gen = order_tiles(eg, o);
  b->h_ft = order_tiles(block_tiles(b, FEAT_TILE_Z, FEAT_TILE_R), o);
  b->h_mt = order_tiles(block_tiles(b, MLP_TILE_Z, MLP_TILE_R), o);
  int rc = AXJ_OK;
  if (first) {
    if (rc == AXJ_OK) rc = bupload(b, &b->st_int, b->h_st_int);
    if (rc == AXJ_OK) rc = bupload(b, &b->st_half, b->h_st_half);
    if (rc == AXJ_OK) rc = bupload(b, &b->st_gen, b->h_st_gen);
    if (rc == AXJ_OK) rc = bupload(b, &b->se_int, b->h_se_int);
    if (rc == AXJ_OK) rc = bupload(b, &b->se_gen, b->h_se_gen);
    if (rc == AXJ_OK) rc = bupload(b, &b->ft, b->h_ft);
    if (rc == AXJ_OK) rc = bupload(b, &b->mt, b->h_mt);
  } else {
    if (rc == AXJ_OK) rc = bupdate(b, b->st_int, b->h_st_int);
    if (rc == AXJ_OK) rc = bupdate(b, b->st_half, b->h_st_half);
    if (rc == AXJ_OK) rc = bupdate(b, b->st_gen, b->h_st_gen);
    if (rc == AXJ_OK) rc = bupdate(b, b->se_int, b->h_se_int);
    if (rc == AXJ_OK) rc = bupdate(b, b->se_gen, b->h_se_gen);
    if (rc == AXJ_OK) rc = bupdate(b, b->ft, b->h_ft);
    if (rc == AXJ_OK) rc = bupdate(b, b->mt, b->h_mt);
  }
  return rc;
}

BatchTiles btiles(const axj_batch* b, const int4* d, const std::vector<int4>& hv, int64_t per_sm) {
  BatchTiles t;
  t.tiles = d;
  t.ntiles = (int)hv.size();
  const long long g = (long long)std::max<int64_t>(per_sm, 1) * b->nsm;
  t.grid = (int)std::max<long long>(1, std::min<long long>(g, t.ntiles));
  return t;
}

// One batched RK stage (mirrors enqueue_stage / enqueue_stage_learned of a handle).
int batch_stage(axj_batch* b, int bin, int bout, int stage, bool judge) {
  (void)bout;
  const bool lrn_plain = b->learned && judge && stage > 1 && b->judge_all;
  const bool lrn = b->learned && !lrn_plain;
  const int rows = (int)b->tune.stage_rows;
  const BatchTiles sti = rows == TR / 2 ? btiles(b, b->st_half, b->h_st_half, b->tune.stage_ctas_per_sm)
                                        : btiles(b, b->st_int, b->h_st_int, b->tune.stage_ctas_per_sm);
  const BatchTiles stg = btiles(b, b->st_gen, b->h_st_gen, std::max<int64_t>(1, b->tune.general_ctas_per_sm));
  const BatchTiles sei = btiles(b, b->se_int, b->h_se_int, b->tune.sensor_ctas_per_sm);
  const BatchTiles seg = btiles(b, b->se_gen, b->h_se_gen, 2);
  // general tiles beside the interior launches (side stream) or on the batch's stream
  const SideStream gside = b->tune.general_serial ? SideStream{nullptr, nullptr, nullptr} : b->side;
  auto sensor = [&](bool rfilter) -> int {
    BATCH_CUDA(b, launch_sensor_batch(b->sens_argv[bin], b->a0_sens[bin], sei, seg, b->maps, bin, b->zrows, b->nzrows,
                                      b->zthreads, b->zsmem, rfilter, b->n, b->max_pts, gside, b->stream));
    return AXJ_OK;
  };
  if (lrn) {
    if (b->held_only) {
      if (judge && stage == 1)
        if (int rc = sensor(true)) return rc;
    } else if (stage == 1) {
      const BatchTiles ft = btiles(b, b->ft, b->h_ft, 4);
      BATCH_CUDA(b, launch_features_batch(b->feat_argv, ft.tiles, ft.ntiles, ft.grid, b->stream));
      if (judge) {
        if (int rc = sensor(true)) return rc;
        BATCH_CUDA(b, launch_mlp_infer_batch(b->a0_infer[0], b->infer_argv[0], b->mt, (int)b->h_mt.size(), b->stream));
        BATCH_CUDA(b, launch_judge_batch(b->judge_argv, b->n, b->max_pts, b->stream));
      } else {
        BATCH_CUDA(b, launch_mlp_infer_batch(b->a0_infer[1], b->infer_argv[1], b->mt, (int)b->h_mt.size(), b->stream));
      }
    }
  } else if (b->sc) {
    // the plain sensor: sensor tiles, then the fused z/r filter into the coefficient planes
    BATCH_CUDA(b, launch_sensor_batch(b->sens_argv[bin], b->a0_sens[bin], sei, seg, b->maps, bin, nullptr, 0,
                                      b->zthreads, b->zsmem, false, b->n, b->max_pts, gside, b->stream));
    BATCH_CUDA(b, launch_zr_batch(b->zr_argv, b->zr_items, b->nzr_items, b->maps, bin, b->mixed, buf_f32(bin),
                                  b->stream));
  }
  const int L = lrn ? CM_LRN : (b->sc ? CM_PRE : CM_FILT);
  BATCH_CUDA(b, launch_stage_batch(b->stage_argv[L][stage], b->a0_stage[L][stage], sti, stg, b->maps, bin, gside,
                                   b->stream, rows));
  return AXJ_OK;
}

int batch_enqueue_step(axj_batch* b, bool judge) {
  BATCH_CUDA(b, launch_dt_batch(b->dt_argv, b->n, b->dt_blocks, b->stream));
  if (b->any_harm) BATCH_CUDA(b, launch_harmonic_phase_batch(b->harm_argv, b->n, b->stream));
  int bufs[5];
  rk4_buffers(b->h[0], bufs);
  for (int st = 1; st <= 4; ++st)
    if (int rc = batch_stage(b, bufs[st - 1], bufs[st], st, judge)) return rc;
  return AXJ_OK;
}

void batch_drop_graphs(axj_batch* b) {
  for (int k = 0; k < 2; ++k) {
    if (b->gexec[k]) cudaGraphExecDestroy(b->gexec[k]);
    if (b->graph[k]) cudaGraphDestroy(b->graph[k]);
    b->gexec[k] = nullptr;
    b->graph[k] = nullptr;
  }
}

int batch_graph(axj_batch* b, bool judge, cudaGraphExec_t* out) {
  const int k = judge ? 1 : 0;
  if (!b->gexec[k]) {
    BATCH_CUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int rc = batch_enqueue_step(b, judge);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (rc != AXJ_OK) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return bfail(b, AXJ_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    b->graph[k] = g;
    BATCH_CUDA(b, cudaGraphInstantiate(&b->gexec[k], g, 0));
  }
  *out = b->gexec[k];
  return AXJ_OK;
}

bool batch_judge_due(const axj_batch* b) {
  if (!b->learned) return false;
  for (const axj_handle* h : b->h)
    if (!h->judged) return true;
  return b->judge_every > 0 && b->iteration % b->judge_every == 0;
}

int batch_launch_step(axj_batch* b) {
  const bool judge = batch_judge_due(b);
  cudaGraphExec_t ge = nullptr;
  if (int rc = batch_graph(b, judge, &ge)) return rc;
  BATCH_CUDA(b, cudaGraphLaunch(ge, b->stream));
  if (judge) {
    for (axj_handle* h : b->h) {
      h->judged = true;
      h->njudges += 1;
    }
    b->njudges += 1;
  }
  b->iteration += 1;
  for (axj_handle* h : b->h) h->iteration += 1;
  return AXJ_OK;
}

// After the batch's stream has run: host times and the error flags of every instance.
int batch_finish(axj_batch* b) {
  BATCH_CUDA(b, cudaStreamSynchronize(b->stream));
  for (int k = 0; k < b->n; ++k) {
    axj_handle* h = b->h[k];
    BATCH_CUDA(b, cudaMemcpy(&h->time_host, h->time, sizeof(double), cudaMemcpyDeviceToHost));
    int f = 0;
    BATCH_CUDA(b, cudaMemcpy(&f, h->flags, sizeof(int), cudaMemcpyDeviceToHost));
    if (f & 4) return bfail(b, AXJ_ERR_TIMEOUT, "instance %d: a bounded wait on a TMA transfer gave up", k);
    if (f & 2) return bfail(b, AXJ_ERR_DT_BLOWUP, "instance %d: Time step blow up", k);
    if (f & 1) return bfail(b, AXJ_ERR_NONFINITE, "instance %d: non-finite value in the solution or time step", k);
  }
  return AXJ_OK;
}

int batch_build_tables(axj_batch* b) {
  const int n = b->n;
  // tensor maps: every instance's maps at the fixed batch indices
  std::vector<CUtensorMap> maps((size_t)n * NM_BATCH);
  for (int k = 0; k < n; ++k) {
    axj_handle* h = b->h[k];
    CUtensorMap* m = maps.data() + (size_t)k * NM_BATCH;
    const int nb = h->mixed ? NBUF : BUAF;
    for (int bf = 0; bf < NBUF; ++bf)
      for (int cls = 0; cls < 2; ++cls) {
        const int src = bf < nb ? bf : 0;  // unused FP32 slots of an FP64 batch repeat buffer 0
        m[bmap_state(bf, cls)] = h->map_state[src][cls];
        m[bmap_sens(bf, cls)] = h->map_sens[src][cls];
        m[bmap_sensT(bf, cls)] = h->map_sensT[src][cls];
      }
    for (int cls = 0; cls < 2; ++cls) {
      m[bmap_star(cls, false)] = h->map_star[cls];
      m[bmap_star(cls, true)] = h->map_starL[cls];
    }
    m[14] = h->map_u0_tile;
    m[15] = h->map_acc_tile;
    for (int bf = 0; bf < NBUF; ++bf) m[bmap_stateH(bf)] = h->map_stateH[bf < nb ? bf : 0];
    m[bmap_starH(false)] = h->map_starH;
    m[bmap_starH(true)] = h->map_starLH;
    m[bmap_u0H] = h->map_u0H;
    m[bmap_accH] = h->map_accH;
    if (h->c.shock_capturing) {
      m[bmap_zrQ] = h->map_zrQ;
      m[bmap_zrZc] = h->map_zrZc;
      m[bmap_zrRc] = h->map_zrRc;
      for (int bf = 0; bf < NBUF; ++bf) m[bmap_zrT(bf)] = h->map_zrT[bf < nb ? bf : 0];
      m[bmap_coef(0)] = h->map_coef[0];
      m[bmap_coef(1)] = h->map_coef[1];
      m[bmap_coef(2)] = h->map_coefH;
    }
  }
  {
    void* p = nullptr;
    BATCH_CUDA(b, cudaMalloc(&p, maps.size() * sizeof(CUtensorMap)));
    b->mem.push_back(p);
    BATCH_CUDA(b, cudaMemcpy(p, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice));
    b->maps = static_cast<CUtensorMap*>(p);
  }
  // per-instance arguments
  int bufs[5];
  rk4_buffers(b->h[0], bufs);
  for (int L = 0; L < 3; ++L)
    for (int st = 1; st <= 4; ++st) {
      std::vector<StageArgs> v(n);
      for (int k = 0; k < n; ++k) {
        v[k] = stage_args(b->h[k], bufs[st - 1], bufs[st], st);
        v[k].learned = L;  // CM_FILT, CM_LRN, CM_PRE
      }
      b->a0_stage[L][st] = v[0];
      if (int rc = bupload(b, &b->stage_argv[L][st], v)) return rc;
    }
  for (int bf = 0; bf < NBUF; ++bf) {
    std::vector<SensorArgs> v(n);
    for (int k = 0; k < n; ++k) v[k] = sensor_args(b->h[k], (b->mixed || bf < BUAF) ? bf : BU0);
    b->a0_sens[bf] = v[0];
    if (int rc = bupload(b, &b->sens_argv[bf], v)) return rc;
  }
  if (b->sc) {
    std::vector<FeatArgs> fv(n);
    std::vector<InferArgs> i0(n), i1(n);
    std::vector<JudgeArgs> jv(n);
    for (int k = 0; k < n; ++k) {
      axj_handle* h = b->h[k];
      fv[k] = feat_args(h, BU0);
      i0[k] = infer_args(h, 0);
      i1[k] = infer_args(h, 1);
      jv[k] = JudgeArgs{grid_of(h), h->pred, h->star + h->plane, h->judge_thr, h->mask, h->held, h->counts};
    }
    b->a0_infer[0] = i0[0];
    b->a0_infer[1] = i1[0];
    if (int rc = bupload(b, &b->feat_argv, fv)) return rc;
    if (int rc = bupload(b, &b->infer_argv[0], i0)) return rc;
    if (int rc = bupload(b, &b->infer_argv[1], i1)) return rc;
    if (int rc = bupload(b, &b->judge_argv, jv)) return rc;
  }
  std::vector<DtArgs> dv(n);
  std::vector<HarmArgs> hv(n);
  for (int k = 0; k < n; ++k) {
    axj_handle* h = b->h[k];
    dv[k] = dt_args(h, 1);
    hv[k] = HarmArgs{h->time, h->dt, h->c.harm_omega, h->harm};
    if (h->c.control_forcing == 2) b->any_harm = true;
  }
  if (int rc = bupload(b, &b->dt_argv, dv)) return rc;
  if (int rc = bupload(b, &b->harm_argv, hv)) return rc;
  // z-filter rows (instance, j)
  if (b->sc) {
    std::vector<int2> rows;
    int bs = 32;
    for (int k = 0; k < n; ++k) {
      for (int j = 0; j < b->h[k]->Nr; ++j) rows.push_back(make_int2(k, j));
      bs = std::max(bs, zrows_threads(b->h[k]->Nz));
    }
    size_t sm = 0;
    for (int k = 0; k < n; ++k) sm = std::max(sm, zrows_smem(b->h[k]->Nz, b->h[k]->P, bs));
    b->nzrows = (int)rows.size();
    b->zthreads = bs;
    b->zsmem = sm;
    if (int rc = bupload(b, &b->zrows, rows)) return rc;
    // the fused z/r filter over all instances: one segment length for the batch, about
    // three CTAs per SM in all (segments of a multiple of ZRK_BZ, at least 64 positions)
    long long work = 0;
    for (int k = 0; k < n; ++k) work += (long long)b->h[k]->Nz * ((b->h[k]->Nr + ZRK_RB - 1) / ZRK_RB);
    long long seg = std::max<long long>(64, (work + 3 * b->nsm - 1) / (3 * b->nsm));
    seg = (seg + ZRK_BZ - 1) / ZRK_BZ * ZRK_BZ;
    std::vector<ZrArgs> zv(n);
    std::vector<int4> items;
    for (int k = 0; k < n; ++k) {
      axj_handle* h = b->h[k];
      zv[k] = zr_args(h, (int)seg);
      const int nx = (int)((h->Nz + seg - 1) / seg), ny = (h->Nr + ZRK_RB - 1) / ZRK_RB;
      for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) items.push_back(make_int4(x, y, k, 0));
    }
    b->nzr_items = (int)items.size();
    if (int rc = bupload(b, &b->zr_argv, zv)) return rc;
    if (int rc = bupload(b, &b->zr_items, items)) return rc;
  }
  // dt: the same number of blocks for every instance (the handles' partial arrays hold 592)
  b->dt_blocks = (int)std::min<long long>(592, std::max<long long>(1, b->max_pts / (DT_THREADS * 8)));
  return batch_tiles(b, true);
}

// Device copies of the instances' solutions, times and stale T (autotuning trials
// advance the batch and are undone).
struct BatchSave {
  std::vector<void*> u0;
  std::vector<double> time_host, stale;
  std::vector<int64_t> it;
};

int batch_save(axj_batch* b, BatchSave& s) {
  for (axj_handle* h : b->h) {
    void* p = nullptr;
    const size_t bytes = sizeof(double) * 5 * (size_t)h->plane;
    BATCH_CUDA(b, cudaMalloc(&p, bytes));
    s.u0.push_back(p);
    BATCH_CUDA(b, cudaMemcpy(p, h->U0, bytes, cudaMemcpyDeviceToDevice));
    double st = 0.0, t = 0.0;
    BATCH_CUDA(b, cudaMemcpy(&st, h->staleT, sizeof(double), cudaMemcpyDeviceToHost));
    BATCH_CUDA(b, cudaMemcpy(&t, h->time, sizeof(double), cudaMemcpyDeviceToHost));
    s.stale.push_back(st);
    s.time_host.push_back(t);
    s.it.push_back(h->iteration);
  }
  return AXJ_OK;
}

int batch_restore(axj_batch* b, BatchSave& s) {
  for (int k = 0; k < b->n; ++k) {
    axj_handle* h = b->h[k];
    const size_t bytes = sizeof(double) * 5 * (size_t)h->plane;
    BATCH_CUDA(b, cudaMemcpy(h->U0, s.u0[k], bytes, cudaMemcpyDeviceToDevice));
    BATCH_CUDA(b, cudaMemcpy(h->staleT, &s.stale[k], sizeof(double), cudaMemcpyHostToDevice));
    BATCH_CUDA(b, cudaMemcpy(h->time, &s.time_host[k], sizeof(double), cudaMemcpyHostToDevice));
    h->time_host = s.time_host[k];
    h->iteration = s.it[k];
    h->judged = false;  // the held coefficients are rebuilt by the next judge step
    cudaFree(s.u0[k]);
  }
  s.u0.clear();
  b->iteration = b->h[0]->iteration;
  return AXJ_OK;
}

}  // namespace

extern "C" {

void axj_batch_default_tuning(axj_batch_tuning* t) {
  if (!t) return;
  std::memset(t, 0, sizeof(*t));
  t->tile_order = 0;
  t->stage_ctas_per_sm = 2;
  t->sensor_ctas_per_sm = 4;
  t->stage_rows = TR;
  t->general_ctas_per_sm = 1;
  t->general_serial = 0;
}

int axj_batch_create(axj_handle* const* handles, int64_t n, axj_batch** out) {
  if (!handles || !out || n < 1) return bfail(nullptr, AXJ_ERR_ARG, "bad argument");
  *out = nullptr;
  axj_handle* h0 = handles[0];
  for (int64_t k = 0; k < n; ++k) {
    const axj_handle* h = handles[k];
    if (!h) return bfail(nullptr, AXJ_ERR_ARG, "null handle %lld", (long long)k);
    if (!h->state_set) return bfail(nullptr, AXJ_ERR_ARG, "instance %lld: axj_set_state has not been called", (long long)k);
    if (h->device != h0->device || h->mixed != h0->mixed || h->learned != h0->learned ||
        h->held_only != h0->held_only || (h->c.shock_capturing != 0) != (h0->c.shock_capturing != 0) ||
        h->judge_all != h0->judge_all)
      return bfail(nullptr, AXJ_ERR_UNSUPPORTED,
                   "instance %lld: every instance needs the same device, precision, sensor, judge stages and shock "
                   "capturing",
                   (long long)k);
    if (h->learned && !h->held_only && !h->mlp_set)
      return bfail(nullptr, AXJ_ERR_ARG, "instance %lld: learned sensor without a model", (long long)k);
    if (h->c.shock_capturing && h->Nz > 10240)
      return bfail(nullptr, AXJ_ERR_UNSUPPORTED, "instance %lld: batched z filter takes Nz <= 10240", (long long)k);
  }
  axj_batch* b = new axj_batch();
  b->n = (int)n;
  b->device = h0->device;
  b->h.assign(handles, handles + n);
  b->mixed = h0->mixed;
  b->learned = h0->learned;
  b->held_only = h0->held_only;
  b->sc = h0->c.shock_capturing != 0;
  b->judge_every = h0->judge_every;
  b->judge_all = h0->judge_all;
  b->iteration = h0->iteration;
  axj_batch_default_tuning(&b->tune);
  int rc = AXJ_OK;
  if (cudaSetDevice(b->device) != cudaSuccess) rc = bfail(b, AXJ_ERR_CUDA, "cudaSetDevice failed");
  // the batch runs the model of instance 0 for every instance: they must agree
  if (rc == AXJ_OK && b->learned && !b->held_only) {
    std::vector<float> w0(MLP_NPARAM), wk(MLP_NPARAM);
    cudaMemcpy(w0.data(), h0->mlp, sizeof(float) * MLP_NPARAM, cudaMemcpyDeviceToHost);
    for (int64_t k = 1; k < n && rc == AXJ_OK; ++k) {
      cudaMemcpy(wk.data(), handles[k]->mlp, sizeof(float) * MLP_NPARAM, cudaMemcpyDeviceToHost);
      if (std::memcmp(w0.data(), wk.data(), sizeof(float) * MLP_NPARAM) != 0 ||
          std::memcmp(&h0->norm, &handles[k]->norm, sizeof(MlpNorm)) != 0)
        rc = bfail(b, AXJ_ERR_UNSUPPORTED, "instance %lld has a different model than instance 0", (long long)k);
    }
  }
  for (int64_t k = 0; k < n; ++k) {
    b->max_pts = std::max<long long>(b->max_pts, (long long)handles[k]->Nz * handles[k]->Nr);
    cudaStreamSynchronize(handles[k]->stream);
  }
  cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, b->device);
  if (rc == AXJ_OK && (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
                       cudaStreamCreateWithFlags(&b->side.stream, cudaStreamNonBlocking) != cudaSuccess ||
                       cudaEventCreateWithFlags(&b->side.fork, cudaEventDisableTiming) != cudaSuccess ||
                       cudaEventCreateWithFlags(&b->side.join, cudaEventDisableTiming) != cudaSuccess))
    rc = bfail(b, AXJ_ERR_CUDA, "stream / event creation failed");
  if (rc == AXJ_OK) rc = batch_build_tables(b);
  if (rc != AXJ_OK) {
    g_create_error = b->err;
    axj_batch_destroy(b);
    return rc;
  }
  *out = b;
  return AXJ_OK;
}

int axj_batch_set_tuning(axj_batch* b, const axj_batch_tuning* t) {
  if (!b || !t) return bfail(b, AXJ_ERR_ARG, "null argument");
  if (t->tile_order < 0 || t->tile_order > 1 || t->stage_ctas_per_sm < 1 || t->stage_ctas_per_sm > 8 ||
      t->sensor_ctas_per_sm < 1 || t->sensor_ctas_per_sm > 8 || (t->stage_rows != TR && t->stage_rows != TR / 2) ||
      t->general_ctas_per_sm < 0 || t->general_ctas_per_sm > 2 || t->general_serial < 0 || t->general_serial > 1)
    return bfail(b, AXJ_ERR_ARG, "tuning out of range");
  BATCH_CUDA(b, cudaSetDevice(b->device));
  BATCH_CUDA(b, cudaStreamSynchronize(b->stream));
  const bool reorder = t->tile_order != b->tune.tile_order;
  b->tune = *t;
  if (reorder)
    if (int rc = batch_tiles(b, false)) return rc;
  batch_drop_graphs(b);
  return AXJ_OK;
}

int axj_batch_get_tuning(axj_batch* b, axj_batch_tuning* t) {
  if (!b || !t) return bfail(b, AXJ_ERR_ARG, "null argument");
  *t = b->tune;
  return AXJ_OK;
}

int axj_batch_run(axj_batch* b, int64_t nsteps) {
  if (!b || nsteps < 0) return bfail(b, AXJ_ERR_ARG, "bad argument");
  BATCH_CUDA(b, cudaSetDevice(b->device));
  for (axj_handle* h : b->h) BATCH_CUDA(b, cudaStreamSynchronize(h->stream));
  for (int64_t s = 0; s < nsteps; ++s)
    if (int rc = batch_launch_step(b)) return rc;
  return batch_finish(b);
}

int axj_batch_run_timed(axj_batch* b, int64_t nsteps, double* ms) {
  if (!b || !ms || nsteps < 0) return bfail(b, AXJ_ERR_ARG, "bad argument");
  BATCH_CUDA(b, cudaSetDevice(b->device));
  for (axj_handle* h : b->h) BATCH_CUDA(b, cudaStreamSynchronize(h->stream));
  // both step graphs are captured outside the timed region
  cudaGraphExec_t ge = nullptr;
  if (int rc = batch_graph(b, false, &ge)) return rc;
  if (b->learned)
    if (int rc = batch_graph(b, true, &ge)) return rc;
  cudaEvent_t e0, e1;
  BATCH_CUDA(b, cudaEventCreate(&e0));
  BATCH_CUDA(b, cudaEventCreate(&e1));
  BATCH_CUDA(b, cudaEventRecord(e0, b->stream));
  int rc = AXJ_OK;
  for (int64_t s = 0; s < nsteps && rc == AXJ_OK; ++s) rc = batch_launch_step(b);
  BATCH_CUDA(b, cudaEventRecord(e1, b->stream));
  BATCH_CUDA(b, cudaEventSynchronize(e1));
  float t = 0.f;
  BATCH_CUDA(b, cudaEventElapsedTime(&t, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = t;
  if (rc != AXJ_OK) return rc;
  return batch_finish(b);
}

int axj_batch_autotune(axj_batch* b, int64_t steps_per_trial, axj_batch_tuning* chosen, double* trial_ms,
                       int64_t* ntrials) {
  if (!b || steps_per_trial < 1) return bfail(b, AXJ_ERR_ARG, "bad argument");
  BATCH_CUDA(b, cudaSetDevice(b->device));
  BatchSave save;
  if (int rc = batch_save(b, save)) return rc;
  // candidates: tile order x interior stage tile shape (32 x 16, or 32 x 8 half tiles)
  // with its persistent CTAs per SM (1 or 2 of 256 threads; 2 or 4 of 128) x persistent
  // CTAs per SM of the interior sensor kernel (4 or 6 of 128 threads: four fit an SM with
  // FP64 boxes, six with FP32 ones)
  std::vector<axj_batch_tuning> cands;
  for (int o = 0; o < 2; ++o)
    for (int rows : {TR, TR / 2})
      for (int sc = 1; sc <= 2; ++sc)
        for (int se = 1; se <= 2; ++se) {
          axj_batch_tuning t;
          axj_batch_default_tuning(&t);
          t.tile_order = o;
          t.stage_rows = rows;
          // half tiles: two or four CTAs per SM (FP64), three or six (FP32 stencils)
          t.stage_ctas_per_sm = rows == TR ? sc : (b->mixed ? 3 : 2) * sc;
          t.sensor_ctas_per_sm = 2 + 2 * se;
          if (!b->sc && se > 1) continue;
          cands.push_back(t);
        }
  double best = 1e300;
  axj_batch_tuning best_t = b->tune;
  int k = 0;
  // one trial: set t, warm up (captures the graphs), time, undo the steps
  auto trial = [&](const axj_batch_tuning& t) -> int {
    int rc = axj_batch_set_tuning(b, &t);
    double ms = 0.0;
    if (rc == AXJ_OK) rc = axj_batch_run(b, 1);
    if (rc == AXJ_OK) rc = axj_batch_run_timed(b, steps_per_trial, &ms);
    if (rc != AXJ_OK) {
      batch_restore(b, save);
      return rc;
    }
    if (trial_ms) trial_ms[k] = ms;
    ++k;
    if (ms < best) {
      best = ms;
      best_t = t;
    }
    if (int r2 = batch_restore(b, save)) return r2;
    return batch_save(b, save);
  };
  for (const axj_batch_tuning& t : cands)
    if (int rc = trial(t)) return rc;
  // then the fastest with the general stage tiles at two CTAs per SM and / or on the
  // batch's stream after the interior tiles
  const axj_batch_tuning main_best = best_t;
  for (int g = 1; g < 4; ++g) {
    axj_batch_tuning t = main_best;
    t.general_ctas_per_sm = (g & 1) ? 2 : 1;
    t.general_serial = (g & 2) ? 1 : 0;
    if (int rc = trial(t)) return rc;
  }
  for (void* p : save.u0) cudaFree(p);
  save.u0.clear();
  if (ntrials) *ntrials = k;
  if (int rc = axj_batch_set_tuning(b, &best_t)) return rc;
  if (chosen) *chosen = best_t;
  return AXJ_OK;
}

const char* axj_batch_last_error(const axj_batch* b) { return b ? b->err.c_str() : g_create_error.c_str(); }

void axj_batch_destroy(axj_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  batch_drop_graphs(b);
  for (void* p : b->mem) cudaFree(p);
  if (b->side.stream) cudaStreamSynchronize(b->side.stream);
  if (b->side.fork) cudaEventDestroy(b->side.fork);
  if (b->side.join) cudaEventDestroy(b->side.join);
  if (b->side.stream) cudaStreamDestroy(b->side.stream);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

}  // extern "C"
