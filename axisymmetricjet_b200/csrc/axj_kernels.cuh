// axj_kernels.cuh -- kernel argument blocks and launch entry points shared by the
// C-ABI layer (axj_api.cu) and the kernels (axj_kernels.cu).
#pragma once

#include <cuda.h>  // CUtensorMap (the encoding call is resolved at run time)
#include <cuda_runtime.h>

#include "axj_common.cuh"

namespace axj {

// TMA descriptors of one fused-stage launch: the stage input with its halo box for
// the tile class, the shock-capturing coefficient planes with the same box, and
// the tile-sized boxes of pv_old and the running RK sum.
struct StageMaps {
  const CUtensorMap* state;
  const CUtensorMap* star;
  const CUtensorMap* u0;
  const CUtensorMap* acc;
  const CUtensorMap* bt;  // tile box of k2 (prefetched into L2 for stage 3)
  const CUtensorMap* tg;  // tile box of pv_target (prefetched into L2 where sponges or faces read it)
};

// Device view of one solver instance.
struct Grid {
  int Nz, Nr;
  long long P;       // row pitch (doubles) of every device field
  long long plane;   // P * Nr
};

// Content of the stage kernel's coefficient box (StageArgs::learned):
//   CM_FILT: the z-filtered sensor quantities; the kernel applies the r filter, so the
//            box reaches the filter's rows beyond the state box;
//   CM_LRN:  the final mu*, beta*, kappa* planes (learned sensor), on the state box;
//   CM_PRE:  mu_eff, beta (0.6 mu + beta*) and kappa_eff, formed by the fused z/r filter
//            kernel, on the state box (the stage kernel evaluates no T**0.666).
constexpr int CM_FILT = 0, CM_LRN = 1, CM_PRE = 2;

// Arguments of the fused RK-stage kernel.
struct StageArgs {
  Grid g;
  const double* Uin;     // stage input state (5 planes)
  const double* U0;      // pv_old (5 planes)
  double* A;             // running sum  pv_old + k1/6 (+ (k2+k3)/3)
  double* B;             // k2
  double* Uout;          // stage output (5 planes); rhs (5 planes) in stage 0
  float* Uout_f;         // FP32 stage output (mixed precision, stages 1-3)
  const double* target;  // pv_target (5 planes)
  const double* mustar;  // shock-capturing coefficients (planes), or null
  const double* betastar;
  const double* kappastar;
  const uint32_t* desc;  // per-point stencil descriptors (pitch P)
  const int* faces;      // face-operation lists: faces[f] = n, faces[f+1..f+n] = patch ids
  const int2* tiles;     // tile origins (i0, j0)
  const double* dxidz;   // 1-D metrics and coordinates
  const double* ddxidxidz;
  const double* detadr;
  const double* ddetadetadr;
  const double* zc;
  const double* rc;
  const double* invr;     // 1/r_j (0 on the axis row)
  const double* forcing;  // 25 doubles, row-major F(eqn,k)
  const double* ramp;     // shock-capturing z ramp (1+tanh(5(z-10)))/2
  const double* dt;       // device dt (read by stages 1-4)
  double* staleT;         // stage 4: T(i*, j*) of its input, the next ComputeTimeStep's stale T
  const double* harm;     // cos(omega t_s) of the harmonic forcing: [0] at t_n (stage 0), [s] at stage s
  int* flags;             // bit 0: non-finite value produced
  int stage;              // 0: write rhs only; 1..4: RK4 stage
  int iT, jT;             // stale-T point (0-based)
  int mixed;              // 1: FP32 stencils and interior pointwise terms
  int in_f32;             // 1: the stage input (maps) is FP32
  int out_f32;            // 1: stages 1-3 write Uout_f instead of Uout
  int learned;            // coefficient box content: CM_FILT, CM_LRN or CM_PRE
  Consts c;
};

struct DtArgs {
  Grid g;
  const double* U;
  const uint32_t* desc;
  const double* dxidz;
  const double* detadr;
  const double* staleT;
  double* partial;       // one per block
  unsigned int* counter; // last-block-done counter, left at 0
  double* dt;            // result
  int* flags;            // bit 1: dt blow-up (every point blanked), bit 0: non-finite dt
  double* time;          // solution time, advanced by dt when advance != 0
  int advance;
  Consts c;
};

// Shock-capturing sensor chain (ModShockCapturing.f90:5-106).
struct SensorArgs {
  Grid g;
  const double* U;       // stage input state (FP64 inputs; else null)
  const float* Uf;       // stage input state (FP32 inputs; else null)
  const uint32_t* desc;
  const double* dxidz;
  const double* detadr;
  const double* zc;
  const double* rc;
  const double* invr;    // 1/r_j (0 on the axis row)
  const double* dz;      // deltaz(i) (:171-179)
  const double* dr;      // deltar(j) (:181-189)
  const double* ramp;    // (1+tanh(5(z-10)))/2 (:85)
  const int2* tiles_int; // sensor tile classes: centred rows within reach 6 of the tile
  const int2* tiles_gen; // everything else (closure rows, blanked points, domain edges)
  int ntiles_int, ntiles_gen;
  const CUtensorMap* mv_int;   // TMA maps of the stage input for the two sensor tile classes:
  const CUtensorMap* mv_gen;   //   V_r / V_z boxes,
  const CUtensorMap* mt_int;   //   temperature boxes,
  const CUtensorMap* mt_gen;   // (rho is read from the stage input: U / Uf)
  const unsigned char* zcode;  // z stencil code per point (9 = blanked), pitch P
  int* flags;
  double* Q;             // 3 planes: mustarQuantity, betastarQuantity, kappastarQuantity
  double* Qz;            // 3 planes: Q after the in-place z filter
  double* star;          // 3 planes: mustar, betastar, kappastar
  int mixed;             // 1: FP32 stencils
  int in_f32;            // 1: the stage input (maps) is FP32
  int ramp_off;          // 1: the r filter leaves out the z ramp (training targets)
  Consts c;
};

cudaError_t init_kernel_attributes();
cudaError_t set_wait_tries(int tries);
void upload_tables(const double sbp1[9][6], const double sbp2[9][6], const double tg[9][11],
                   const PatchDev* patches, int npatch, cudaStream_t s);

// Optional side stream for the general-tile launches (stream == null: one stream).
struct SideStream {
  cudaStream_t stream;
  cudaEvent_t fork, join;
};

// int_rows: rows of the interior tiles' CTAs, TR (one CTA per tile) or TR / 2 (two CTAs per
// tile; mint then holds the half-tile boxes).
cudaError_t launch_stage(const StageArgs& a, int ntiles_int, const int2* tiles_int, const StageMaps& mint,
                         int ntiles_gen, const int2* tiles_gen, const StageMaps& mgen, const SideStream& side,
                         cudaStream_t s, int int_rows);

// Box sizes (elements) the stage kernel expects in its tensor maps: state halo box
// halo_w x halo_h, z-filtered coefficient box halo_w x q_h, tile box tile_w x tile_h.
// The mixed path uses one set of box sizes for its FP64 and FP32 stage inputs.
// qlrn_h (nullable): box height of the final-coefficient planes of the learned sensor.
// rows: TR, or TR / 2 for the half tiles of the interior class (gen = false).
void stage_boxes(bool gen, bool mixed, int* halo_w, int* halo_h, int* q_h, int* tile_w, int* tile_h, int* qlrn_h,
                 int rows = TR);
// Boxes (elements, one plane deep) the sensor tile kernel expects for the stage input:
// V_r / V_z box vw x vh, temperature box tw x th (rho uses the stage tile box).
void sensor_boxes(bool gen, bool mixed, int* vw, int* vh, int* tw, int* th);
cudaError_t launch_dt(const DtArgs& a, int nblocks, cudaStream_t s);
int dt_grid_blocks();
// cos(omega t_s) of the harmonic forcing: rhs_mode != 0: out[0] at t = *time; else
// out[s], s = 1..4, at t_s = (*time - *dt) + c_s * *dt (the device time is t_n + dt).
cudaError_t launch_harmonic_phase(const double* time, const double* dt, double omega, int rhs_mode, double* out,
                                  cudaStream_t s);
// rfilter: also run the r filter into a.star (the stage kernel applies it itself; the
// unit entry point axj_sensor needs the coefficients as output).
cudaError_t launch_sensor(const SensorArgs& a, bool rfilter, const SideStream& side, cudaStream_t s);

// Sensor tile kernels only (the quantities Q), for the fused z/r filter path.
cudaError_t launch_sensor_tiles_only(const SensorArgs& a, const SideStream& side, cudaStream_t s);

// Fused z filter + r filter + transport coefficients (zr_kernel): from Q to the planes
// mu_eff, beta = 0.6 mu + beta*, kappa_eff of the stage input. A CTA of ZRK_THREADS
// threads owns seg z positions (a multiple of ZRK_BZ) and ZRK_RB rows.
constexpr int ZRK_BZ = 16;                    // z positions per block (one 128-byte row of doubles)
constexpr int ZRK_RB = 30;                    // rows per CTA (30 x 16 points: three per thread)
constexpr int ZRK_HR = 10;                    // r reach of the TG boundary rows
constexpr int ZRK_NR = ZRK_RB + 2 * ZRK_HR;   // rows of the z recurrence per CTA
constexpr int ZRK_THREADS = 160;
struct ZrArgs {
  Grid g;
  const double* ramp;  // (1+tanh(5(z-10)))/2 per i
  double* coef;        // 3 planes: mu_eff, beta, kappa_eff
  int* flags;          // bit 2: a bounded wait gave up
  int seg;             // z positions per CTA (multiple of ZRK_BZ)
  Consts c;
};
// TMA maps: q = Q (3 planes of doubles, box {ZRK_BZ, ZRK_NR, 3}, 128-byte swizzle);
// zc / rc = z / r row codes (uint8, 9 = blanked; boxes {ZRK_BZ, ZRK_NR} / {ZRK_BZ, ZRK_RB});
// t = the stage input's planes (box {ZRK_BZ, ZRK_RB, 1}, FP32 when in_f32).
struct ZrMaps {
  const CUtensorMap* q;
  const CUtensorMap* zc;
  const CUtensorMap* rc;
  const CUtensorMap* t;
};
cudaError_t launch_zr(const ZrArgs& a, const ZrMaps& m, bool mixed, bool in_f32, cudaStream_t s);
// Batched fused z/r filter: items (segment, row block, instance, 0), per-instance arguments
// and the maps of the batch table (kin = stage-input buffer id).
cudaError_t launch_zr_batch(const ZrArgs* argv, const int4* items, int nitems, const CUtensorMap* mapv, int kin,
                            bool mixed, bool in_f32, cudaStream_t s);

// Unit entry points (one operator on one field, host-facing).
cudaError_t launch_deriv(const Grid& g, const uint32_t* desc, const double* var, const double* first,
                         const double* met, const double* met2, int dirn, int order, double* out, cudaStream_t s);
cudaError_t launch_tgfilter(const Grid& g, const uint32_t* desc, const double* var, int dirn, double* out,
                            cudaStream_t s);
// In-place z filter of nfield planes (q -> out). zcode: per-point z row code bytes
// (9 = no filtering: blanked), pitch P; flags bit 2 is set if a bounded wait gives up.
cudaError_t launch_tgfilter_z_inplace(const Grid& g, const uint32_t* desc, const unsigned char* zcode,
                                      const double* q, double* out, int nfield, int* flags, cudaStream_t s);

constexpr int DT_THREADS = 256;

// ---- batched launches: many solver instances per launch ----
// Per-instance TMA maps of a batch, NM_BATCH per instance, at these indices:
//   state box of stage buffer b, tile class cls:  b * 2 + cls         (0..9)
//   z-filtered coefficient box of class cls:      10 + cls
//   final-coefficient box of class cls:           12 + cls
//   pv_old tile box, running-sum tile box:         14, 15
//   sensor V box of buffer b, class cls:           16 + b * 2 + cls  (16..25)
//   sensor temperature box of buffer b, class cls: 26 + b * 2 + cls  (26..35)
//   interior half tiles (TR / 2 rows): state box of buffer b 36 + b (36..40), z-filtered
//   coefficient box 41, final-coefficient box 42, pv_old and running-sum tile boxes 43, 44
//   fused z/r filter: Q blocks 45, z and r code blocks 46, 47, temperature blocks of
//   buffer b 48 + b (48..52); its coefficient planes as boxes of the interior, general and
//   half tiles 53, 54, 55
constexpr int NM_BATCH = 56;
inline int bmap_state(int b, int cls) { return b * 2 + cls; }
inline int bmap_star(int cls, bool lrn) { return (lrn ? 12 : 10) + cls; }
inline int bmap_sens(int b, int cls) { return 16 + b * 2 + cls; }
inline int bmap_sensT(int b, int cls) { return 26 + b * 2 + cls; }
inline int bmap_stateH(int b) { return 36 + b; }
inline int bmap_starH(bool lrn) { return lrn ? 42 : 41; }
constexpr int bmap_u0H = 43, bmap_accH = 44;
constexpr int bmap_zrQ = 45, bmap_zrZc = 46, bmap_zrRc = 47;
inline int bmap_zrT(int b) { return 48 + b; }
inline int bmap_coef(int cls) { return 53 + cls; }  // cls 0 interior, 1 general, 2 half tiles

struct BatchTiles {
  const int4* tiles;  // (i0, j0, instance, 0)
  int ntiles;
  int grid;           // persistent CTAs
};

// Fused stage over the interior and general tiles of all instances (general on the
// side stream). argv: per-instance arguments of this stage (all with the same stage,
// precision flags and learned flag); kin = stage-input buffer id.
// int_rows: TR, or TR / 2 with tint holding the interior half tiles.
cudaError_t launch_stage_batch(const StageArgs* argv, const StageArgs& a0, const BatchTiles& tint, const BatchTiles& tgen,
                               const CUtensorMap* mapv, int kin, const SideStream& side, cudaStream_t s, int int_rows);
// Sensor chain over all instances: sensor tiles, the row-staged z filter of every row
// (zrows: (instance, j)), and with rfilter the r filter (grid y = instance, max_pts
// points per instance at most).
cudaError_t launch_sensor_batch(const SensorArgs* argv, const SensorArgs& a0, const BatchTiles& tint,
                                const BatchTiles& tgen, const CUtensorMap* mapv, int kin, const int2* zrows,
                                int nzrows, int zthreads, size_t zsmem, bool rfilter, int ninst, long long max_pts,
                                const SideStream& side, cudaStream_t s);
cudaError_t launch_dt_batch(const DtArgs* argv, int ninst, int nblocks, cudaStream_t s);
struct HarmArgs {
  const double* time;
  const double* dt;
  double omega;
  double* out;
};
cudaError_t launch_harmonic_phase_batch(const HarmArgs* argv, int ninst, cudaStream_t s);
// z-filter smem for a row of Nz points with pitch P and bs threads.
size_t zrows_smem(int Nz, long long P, int bs);
int zrows_threads(int Nz);

// Sets the message axj_last_error(NULL) returns.
void set_global_error(const char* msg);

}  // namespace axj
