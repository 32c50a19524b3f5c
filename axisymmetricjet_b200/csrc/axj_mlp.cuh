// axj_mlp.cuh -- learned artificial-diffusivity sensor: feature maps, BF16 tensor-core
// inference (tcgen05), the plain-sensor judge, and FP32 training kernels. Shared by
// the C-ABI layer (axj_api.cu) and the kernels (axj_mlp.cu).
#pragma once

#include <cuda_runtime.h>

#include "axj_common.cuh"
#include "axj_kernels.cuh"

namespace axj {

constexpr int MLP_CH = 4;       // dilatation, |grad rho|, |vorticity|, sqrt(deltaz*deltar)
constexpr int MLP_IN = 100;     // 4 channels x 5 x 5 window
constexpr int MLP_K1 = 112;     // MLP_IN padded to a multiple of the MMA K step (16)
constexpr int MLP_HID = 64;
constexpr int MLP_OUT = 2;      // betastar, kappastar before the z ramp
// flat FP32 parameter vector (training layout, W1 padded to MLP_K1 columns)
constexpr int MLP_OFF_W1 = 0;
constexpr int MLP_OFF_B1 = MLP_OFF_W1 + MLP_HID * MLP_K1;
constexpr int MLP_OFF_W2 = MLP_OFF_B1 + MLP_HID;
constexpr int MLP_OFF_B2 = MLP_OFF_W2 + MLP_HID * MLP_HID;
constexpr int MLP_OFF_W3 = MLP_OFF_B2 + MLP_HID;
constexpr int MLP_OFF_B3 = MLP_OFF_W3 + MLP_OUT * MLP_HID;
constexpr int MLP_NPARAM = MLP_OFF_B3 + MLP_OUT;

// Normalisation constants of the model (host copy uploaded with the weights).
struct MlpNorm {
  float feat_mean[MLP_CH];
  float feat_inv_scale[MLP_CH];
  float out_scale[MLP_OUT];
};

// Feature channels of one state: float4 per point, pitch P.
struct FeatArgs {
  Grid g;
  const void* U;        // stage state (5 planes), double or float
  int f32;              // 1: U is float
  const uint32_t* desc;
  const double* dxidz;
  const double* detadr;
  const double* rc;
  const double* dz;     // deltaz(i), deltar(j) of the sensor (ModShockCapturing.f90:171-189)
  const double* dr;
  float4* feat;
  float sbp1[9][6];     // SBP first-derivative rows
};

// Inference: features -> MLP -> (betastar, kappastar) * ramp(z).
// mode 0: write pred (2 planes, double). mode 1: write star planes 1, 2 with the
// judge's fallback: where mask bit k is set, the held plain value is kept.
struct InferArgs {
  Grid g;
  const float4* feat;
  const float* params;  // flat FP32 parameters (MLP_NPARAM)
  MlpNorm norm;
  const double* ramp;
  int mode;
  double* out;                 // mode 0: 2 planes; mode 1: star (planes 1 and 2 written)
  const unsigned char* mask;   // mode 1
  const double* held;          // mode 1: 2 planes
  int* flags;                  // bit 4: a bounded wait gave up
  int ntiles_z, ntiles;        // tiles of 32 (z) x 4 (r) points
};

// Judge: compare pred with the plain sensor's (ramped) betastar/kappastar, set the
// fallback mask where |pred - plain| > thr * (max |plain| over the 5 x 5 window),
// keep the plain values as the held values, count judged and fallback points.
struct JudgeArgs {
  Grid g;
  const double* pred;    // 2 planes
  const double* plain;   // 2 planes (star planes 1, 2)
  double thr;
  unsigned char* mask;
  double* held;          // 2 planes
  unsigned long long* counts;  // [0] judged point-outputs, [1] fallbacks
};

cudaError_t launch_features(const FeatArgs& a, cudaStream_t s);
// Batched forms (tiles (i0, j0, instance, 0); features tiles 32 x 8, inference tiles
// 32 x 4 points; judge: grid y = instance, max_pts points per instance at most).
cudaError_t launch_features_batch(const FeatArgs* argv, const int4* tiles, int ntiles, int grid, cudaStream_t s);
cudaError_t launch_mlp_infer_batch(const InferArgs& a0, const InferArgs* argv, const int4* tiles, int ntiles,
                                   cudaStream_t s);
cudaError_t launch_judge_batch(const JudgeArgs* argv, int ninst, long long max_pts, cudaStream_t s);
constexpr int FEAT_TILE_Z = 32, FEAT_TILE_R = 16;
constexpr int MLP_TILE_Z = 32, MLP_TILE_R = 4;
cudaError_t launch_mlp_infer(const InferArgs& a, cudaStream_t s);
cudaError_t launch_judge(const JudgeArgs& a, cudaStream_t s);
cudaError_t mlp_init_attributes();

// ---- training (FP32, CUDA cores) ----
struct Dataset {
  const float4* feat;    // [S][plane]
  const float2* targ;    // [S][plane] betastar, kappastar before the ramp
  int S;
  Grid g;
};

// X [B x MLP_K1] normalised features (pad columns zero), T [B x 2] normalised targets
// of B points drawn from the data set by a counter-based hash of (seed, step, b).
cudaError_t launch_sample(const Dataset& d, MlpNorm norm, unsigned long long seed, const int* step, int B, float* X,
                          float* T, cudaStream_t s);
// C[M x N] (ldc) = opA(A) * opB(B), opA(m,k) = TA ? A[k*lda+m] : A[m*lda+k], opB(k,n) =
// TB ? B[n*ldb+k] : B[k*ldb+n]. ksplit > 1 adds partial sums atomically (C zeroed first).
cudaError_t launch_gemm(bool TA, bool TB, int M, int N, int K, const float* A, int lda, const float* B, int ldb,
                        float* C, int ldc, int ksplit, cudaStream_t s);
// H = gelu(Z + b) in place of Z's copy: Z += b (kept for the backward pass), H = gelu(Z).
cudaError_t launch_bias_gelu(float* Z, const float* b, float* H, int B, int N, cudaStream_t s);
cudaError_t launch_bias(float* Z, const float* b, int B, int N, cudaStream_t s);
// dY = 2 (Y - T) / B, loss[step] = sum (Y - T)^2 / B (accumulated atomically).
cudaError_t launch_loss(const float* Y, const float* T, float* dY, float* loss, const int* step, int B,
                        cudaStream_t s);
// dZ = dH * gelu'(Z) (in place on dH).
cudaError_t launch_gelu_bwd(float* dH, const float* Z, int n, cudaStream_t s);
// db[n] += sum_b dZ[b][n]
cudaError_t launch_colsum(const float* dZ, float* db, int B, int N, cudaStream_t s);
// Adam on the flat parameter vector; step counter read from *step (0-based) and then
// advanced by launch_step_inc.
cudaError_t launch_adam(float* p, const float* g, float* m, float* v, int n, const int* step, float lr, float b1,
                        float b2, float eps, cudaStream_t s);
cudaError_t launch_step_inc(int* step, cudaStream_t s);
// Per-channel sums / sums of squares of the data set's features and targets
// (acc: 4 x (sum, sumsq) features, 2 x sumsq targets, count), for the normalisation.
cudaError_t launch_dataset_stats(const Dataset& d, double* acc, cudaStream_t s);
// Pack the plain targets (star planes 1, 2) as float2 into the data set.
cudaError_t launch_pack_targets(const Grid& g, const double* star, float2* targ, cudaStream_t s);

}  // namespace axj
