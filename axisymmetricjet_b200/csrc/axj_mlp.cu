// axj_mlp.cu -- learned artificial-diffusivity sensor.
//
// An MLP (100 -> 64 -> 64 -> 2, tanh-form GELU) stands in for the evaluation of
// betastar and kappastar (ModShockCapturing.f90:18-92) between plain-sensor judge
// steps. Its inputs are 5 x 5 (z, r) windows of four channels per point: the
// dilatation, |grad rho|, the vorticity magnitude and the local grid spacing
// sqrt(deltaz*deltar). Inference runs on the 5th-generation tensor cores: BF16
// operands staged in shared memory, FP32 accumulators in tensor memory (tcgen05.mma
// issued by one thread, tcgen05.ld for the epilogues). Training runs in FP32 on the
// CUDA cores: tiled GEMMs for the forward and backward passes and Adam.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "axj_mlp.cuh"

namespace axj {

namespace {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---- mbarrier (one arrival: the tcgen05.commit of the MMA-issuing thread) ----
__device__ __forceinline__ void bar_init(uint64_t* b) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(b)));
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool bar_try(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: gives up after about 1 << 20 polls (a fraction of a second).
__device__ __forceinline__ bool bar_wait(uint64_t* b, uint32_t parity) {
  for (int it = 0; it < (1 << 20); ++it) {
    if (bar_try(b, parity)) return true;
    if (it > 64) __nanosleep(128);
  }
  return false;
}

// ---- tcgen05 ----
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Generic-proxy shared-memory writes become visible to the tensor core (async proxy).
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// Shared-memory matrix descriptor, no swizzle, K-major canonical layout: 8-row x
// 16-byte core matrices; lbo = byte distance of the two K halves of one MMA step,
// sbo = byte distance of consecutive 8-row groups; version 1 (bit 46).
__device__ __forceinline__ uint64_t mdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
         (1ull << 46);
}
// Instruction descriptor of kind::f16: BF16 A and B (K-major), FP32 accumulator,
// M = 128, N = 64.
constexpr uint32_t IDESC_BF16_M128_N64 =
    (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* b) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(b))
               : "memory");
}
// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Two floats to a BF16 pair (a in the low half), one packed conversion.
__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  uint32_t r;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(b), "f"(a));
  return r;
}

}  // namespace

// GELU, tanh form: 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))), and its derivative.
// Inference uses the hardware tanh approximation (one MUFU operation, relative error
// about 2^-11, below the BF16 rounding of the activations it feeds); training uses tanhf.
__device__ __forceinline__ float tanh_fast(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float gelu_fast(float x) {
  const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
  const float hx = 0.5f * x;
  return fmaf(hx, tanh_fast(u), hx);
}
__device__ __forceinline__ float gelu_f(float x) {
  const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
  return 0.5f * x * (1.0f + tanhf(u));
}
__device__ __forceinline__ float gelu_grad_f(float x) {
  const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
  const float t = tanhf(u);
  return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * 0.7978845608028654f * (1.0f + 3.0f * 0.044715f * x * x);
}

// ---------------------------------------------------------------------------
// Feature channels
// ---------------------------------------------------------------------------
// Tile of 32 (z) x 16 (r) points per CTA (256 threads, two points per thread: rows
// tr and tr + 8). rho, V_r, V_z of the tile and a halo of 5 (the widest SBP boundary row
// reaches 5 points) are staged in shared memory as FP32 (zero outside the grid, the
// never-written halo), one box row per warp and pass; each thread forms its six first
// derivatives in FP32 on differences from its own value: every SBP row sums to zero, so
// sum c_m (f_m - f_0) equals sum c_m f_m, and the differences of nearby values are exact
// in FP32 (the network reads its inputs in BF16).
constexpr int FT_Z = FEAT_TILE_Z, FT_R = FEAT_TILE_R, FT_H = 5;
constexpr int FB_Z = FT_Z + 2 * FT_H, FB_R = FT_R + 2 * FT_H;

__device__ __forceinline__ float fd1s(const FeatArgs& a, const float* box, int row, int bz, int br, int dirn) {
  if (row >= 9) return 0.0f;
  const int st = dirn == 1 ? 1 : FB_Z;
  const float* p = box + br * FB_Z + bz;
  const float f0 = p[0];
  if (row == 4) {  // centred row
    float s = a.sbp1[4][0] * (p[-2 * st] - f0);
#pragma unroll
    for (int m = 1; m < 5; ++m) s = s + a.sbp1[4][m] * (p[(m - 2) * st] - f0);
    return s;
  }
  const int w0 = sbp_w0(row);
  float s = a.sbp1[row][0] * (p[w0 * st] - f0);
#pragma unroll
  for (int m = 1; m < 6; ++m) s = s + a.sbp1[row][m] * (p[(w0 + m) * st] - f0);
  return s;
}

// The four channels of point (i, j) = (i0 + tz, j0 + tr) from the staged box.
__device__ __forceinline__ void features_point(const FeatArgs& a, float (*sb)[FB_R * FB_Z], int i, int j, int tz,
                                               int tr) {
  const Grid g = a.g;
  const long long o = (long long)j * g.P + i;
  const uint32_t dsc = __ldg(a.desc + o);
  const int zr = desc_blank(dsc) ? (int)ROW_NONE : desc_zrow(dsc);
  const int rw = desc_blank(dsc) ? (int)ROW_NONE : desc_rrow(dsc);
  const int bz = tz + FT_H, br = tr + FT_H;
  const float xz = (float)__ldg(a.dxidz + i), er = (float)__ldg(a.detadr + j);
  const float drdz = fd1s(a, sb[0], zr, bz, br, 1) * xz;
  const float dVrdz = fd1s(a, sb[1], zr, bz, br, 1) * xz;
  const float dVzdz = fd1s(a, sb[2], zr, bz, br, 1) * xz;
  const float drdr = fd1s(a, sb[0], rw, bz, br, 2) * er;
  const float dVrdr = fd1s(a, sb[1], rw, bz, br, 2) * er;
  const float dVzdr = fd1s(a, sb[2], rw, bz, br, 2) * er;
  const float vr = sb[1][br * FB_Z + bz];
  const float r = (float)__ldg(a.rc + j);
  const float dil = (j == 0) ? 2.0f * dVrdr + dVzdz : dVrdr + vr / r + dVzdz;
  const float grad = sqrtf(drdz * drdz + drdr * drdr);
  const float vort = fabsf(dVrdz - dVzdr);
  const float h = sqrtf((float)(__ldg(a.dz + i) * __ldg(a.dr + j)));
  a.feat[o] = make_float4(dil, grad, vort, h);
}

template <typename SIN>
__device__ __forceinline__ void features_body(const FeatArgs& a, int i0, int j0, float (*sb)[FB_R * FB_Z]) {
  const Grid g = a.g;
  const SIN* Urho = static_cast<const SIN*>(a.U);  // planes 0 (rho), 1 (V_r), 3 (V_z)
  const SIN* Uvr = Urho + g.plane;
  const SIN* Uvz = Urho + 3 * g.plane;
  const int tz = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int br = w; br < FB_R; br += 8) {
    const int j = j0 - FT_H + br;
    const bool jin = j >= 0 && j < g.Nr;
    const long long ro = (long long)j * g.P;
    for (int bz = tz; bz < FB_Z; bz += 32) {
      const int i = i0 - FT_H + bz;
      float v0 = 0.0f, v1 = 0.0f, v2 = 0.0f;
      if (jin && i >= 0 && i < g.Nz) {
        v0 = float(Urho[ro + i]);
        v1 = float(Uvr[ro + i]);
        v2 = float(Uvz[ro + i]);
      }
      const int q = br * FB_Z + bz;
      sb[0][q] = v0;
      sb[1][q] = v1;
      sb[2][q] = v2;
    }
  }
  __syncthreads();
#pragma unroll 1
  for (int tr = w; tr < FT_R; tr += 8) {
    const int i = i0 + tz, j = j0 + tr;
    if (i >= g.Nz || j >= g.Nr) continue;
    features_point(a, sb, i, j, tz, tr);
  }
}

template <typename SIN>
__global__ void __launch_bounds__(256) features_kernel(const FeatArgs a) {
  __shared__ float sb[3][FB_R * FB_Z];
  features_body<SIN>(a, blockIdx.x * FT_Z, blockIdx.y * FT_R, sb);
}

// Batched: persistent loop over (i0, j0, instance) tiles of 32 x 16 points.
__global__ void __launch_bounds__(256) features_kernel_batch(const FeatArgs* __restrict__ argv,
                                                             const int4* __restrict__ tiles, int ntiles) {
  __shared__ float sb[3][FB_R * FB_Z];
  __shared__ __align__(16) FeatArgs sa;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int4 tt = tiles[t];
    __syncthreads();
    for (int k = threadIdx.x; k < (int)(sizeof(FeatArgs) / 4); k += blockDim.x)
      reinterpret_cast<unsigned int*>(&sa)[k] = reinterpret_cast<const unsigned int*>(argv + tt.z)[k];
    __syncthreads();
    if (sa.f32) features_body<float>(sa, tt.x, tt.y, sb);
    else features_body<double>(sa, tt.x, tt.y, sb);
  }
}

cudaError_t launch_features(const FeatArgs& a, cudaStream_t s) {
  const dim3 grid((a.g.Nz + FT_Z - 1) / FT_Z, (a.g.Nr + FT_R - 1) / FT_R);
  if (a.f32) features_kernel<float><<<grid, 256, 0, s>>>(a);
  else features_kernel<double><<<grid, 256, 0, s>>>(a);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Inference on the tensor cores. A tile is 32 (z) x 4 (r) points, one point per
// thread, thread t = row t of the MMA (TMEM lane t). One CTA of 128 threads owns 64
// TMEM columns: layer 1 accumulates there, and once every thread has read its row,
// layer 2 accumulates in the same columns. Shared memory (from a 128-aligned base):
// W1 64x112 and W2 64x64 in BF16; one A operand region of 128x112 BF16 that holds the
// layer-1 inputs and then (after the layer-1 MMAs completed) the layer-2 inputs, all
// in the no-swizzle K-major layout with the K chunks outermost (chunk c of 8 K values
// at c * rows * 16, row group g at g * 128, row r of the group at r * 16); the
// normalised channel box 4 x 8 x 36 in BF16; biases and layer 3 in FP32. The next
// tile's channel box is loaded into registers while this tile's MMAs run. About 54 KB
// per CTA: 4 CTAs (16 warps, 256 TMEM columns) per SM.
// ---------------------------------------------------------------------------
constexpr int MT_Z = 32, MT_R = 4, MT_THREADS = 128;
constexpr int MBOX_Z = MT_Z + 4, MBOX_R = MT_R + 4, MBOX_N = MBOX_Z * MBOX_R;  // 288 points
constexpr int MBOX_PER = (MBOX_N + MT_THREADS - 1) / MT_THREADS;              // 3
constexpr uint32_t M_OW1 = 0;
constexpr uint32_t M_OW2 = M_OW1 + MLP_HID * MLP_K1 * 2;      // 14336
constexpr uint32_t M_OA = M_OW2 + MLP_HID * MLP_HID * 2;      // 22528
constexpr uint32_t M_OBOX = M_OA + MT_THREADS * MLP_K1 * 2;   // 51200
constexpr uint32_t M_OP = M_OBOX + MLP_CH * MBOX_N * 2;       // 53504
constexpr uint32_t M_NP = MLP_HID + MLP_HID + MLP_OUT * MLP_HID + MLP_OUT;
constexpr size_t M_SMEM = M_OP + M_NP * 4 + 128;  // + alignment slack
constexpr int M_CTAS_PER_SM = 4;

// byte offset of (row, k) in a K-major operand of `rows` rows
__device__ __forceinline__ uint32_t kmaj(int row, int k, int rows) {
  return (uint32_t)((k >> 3) * rows * 16 + (row >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// BATCH: tiles (i0, j0, instance) from a table over many instances, each with its own
// arguments in argv (the model, its normalisation and the error flag are a0's, shared by
// the batch); otherwise the tiles of a0's grid in raster order.
template <bool BATCH>
__global__ void __launch_bounds__(MT_THREADS)
    mlp_infer_kernel(const InferArgs a0, const InferArgs* __restrict__ argv, const int4* __restrict__ tiles, int ntiles) {
  const InferArgs& a = a0;
  extern __shared__ unsigned char m_raw[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_slot;
  unsigned char* base = m_raw + ((128u - (smem_addr(m_raw) & 127u)) & 127u);  // 128-aligned start
  const uint32_t sb = smem_addr(base);
  __nv_bfloat16* sBox = reinterpret_cast<__nv_bfloat16*>(base + M_OBOX);  // [4][8][36]
  float* sB1 = reinterpret_cast<float*>(base + M_OP);
  float* sB2 = sB1 + MLP_HID;
  float* sW3 = sB2 + MLP_HID;  // [2][64]
  float* sB3 = sW3 + MLP_OUT * MLP_HID;
  const int tid = threadIdx.x, warp = tid >> 5;
  // weights in BF16, core-matrix layout
  for (int e = tid; e < MLP_HID * MLP_K1; e += MT_THREADS) {
    const int n = e / MLP_K1, k = e - n * MLP_K1;
    *reinterpret_cast<__nv_bfloat16*>(base + M_OW1 + kmaj(n, k, MLP_HID)) = __float2bfloat16_rn(a.params[MLP_OFF_W1 + e]);
  }
  for (int e = tid; e < MLP_HID * MLP_HID; e += MT_THREADS) {
    const int n = e / MLP_HID, k = e - n * MLP_HID;
    *reinterpret_cast<__nv_bfloat16*>(base + M_OW2 + kmaj(n, k, MLP_HID)) = __float2bfloat16_rn(a.params[MLP_OFF_W2 + e]);
  }
  for (int e = tid; e < MLP_HID; e += MT_THREADS) {
    sB1[e] = a.params[MLP_OFF_B1 + e];
    sB2[e] = a.params[MLP_OFF_B2 + e];
  }
  for (int e = tid; e < MLP_OUT * MLP_HID; e += MT_THREADS) sW3[e] = a.params[MLP_OFF_W3 + e];
  if (tid < MLP_OUT) sB3[tid] = a.params[MLP_OFF_B3 + tid];
  if (tid == 0) bar_init(&bar);
  if (warp == 0) tmem_alloc(&tmem_slot, 64);

  // channel box of a tile: raw loads (zero outside the grid) into registers ...
  // tile t: origin and instance
  auto tile_of = [&](int t, int& ti0, int& tj0, int& inst) {
    if (BATCH) {
      const int4 tt = tiles[t];
      ti0 = tt.x;
      tj0 = tt.y;
      inst = tt.z;
    } else {
      ti0 = (t % a0.ntiles_z) * MT_Z;
      tj0 = (t / a0.ntiles_z) * MT_R;
      inst = 0;
    }
  };
  auto load_box = [&](int t, float4* v) {
    int ti0, tj0, inst;
    tile_of(t, ti0, tj0, inst);
    const InferArgs& at = BATCH ? argv[inst] : a0;
    const Grid g = at.g;
    const int i0 = ti0 - 2, j0 = tj0 - 2;
#pragma unroll
    for (int q = 0; q < MBOX_PER; ++q) {
      const int e = tid + q * MT_THREADS;
      v[q] = make_float4(0.f, 0.f, 0.f, 0.f);
      if (e < MBOX_N) {
        const int br = e / MBOX_Z, bz = e - br * MBOX_Z;
        const int i = i0 + bz, j = j0 + br;
        if (i >= 0 && i < g.Nz && j >= 0 && j < g.Nr) v[q] = __ldg(at.feat + (long long)j * g.P + i);
      }
    }
  };
  // ... then normalised into the BF16 box
  auto store_box = [&](const float4* v) {
#pragma unroll
    for (int q = 0; q < MBOX_PER; ++q) {
      const int e = tid + q * MT_THREADS;
      if (e < MBOX_N) {
        sBox[0 * MBOX_N + e] = __float2bfloat16_rn((v[q].x - a.norm.feat_mean[0]) * a.norm.feat_inv_scale[0]);
        sBox[1 * MBOX_N + e] = __float2bfloat16_rn((v[q].y - a.norm.feat_mean[1]) * a.norm.feat_inv_scale[1]);
        sBox[2 * MBOX_N + e] = __float2bfloat16_rn((v[q].z - a.norm.feat_mean[2]) * a.norm.feat_inv_scale[2]);
        sBox[3 * MBOX_N + e] = __float2bfloat16_rn((v[q].w - a.norm.feat_mean[3]) * a.norm.feat_inv_scale[3]);
      }
    }
  };
  float4 nxt[MBOX_PER];
  if ((int)blockIdx.x < ntiles) {
    load_box(blockIdx.x, nxt);
    store_box(nxt);
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);

  const int c = tid & 31, rr = tid >> 5;  // this thread's point in the tile
  uint32_t phase = 0;
  bool ok = true;
  for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
    int i0, j0, inst;
    tile_of(t, i0, j0, inst);
    const InferArgs& at = BATCH ? argv[inst] : a0;
    const Grid g = at.g;
    // A row `tid` of layer 1: feature k = ch*25 + (dr+2)*5 + (dz+2), zero for k >= 100
    const unsigned short* bx = reinterpret_cast<const unsigned short*>(sBox);
#pragma unroll
    for (int kc = 0; kc < MLP_K1 / 8; ++kc) {
      uint32_t pk[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        uint32_t hv[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int k = kc * 8 + 2 * q + h;
          hv[h] = 0u;
          if (k < MLP_IN) {
            const int ch = k / 25, w = k - ch * 25, dr = w / 5, dz = w - dr * 5;
            hv[h] = bx[ch * MBOX_N + (rr + dr) * MBOX_Z + c + dz];
          }
        }
        pk[q] = hv[0] | (hv[1] << 16);
      }
      *reinterpret_cast<uint4*>(base + M_OA + kmaj(tid, kc * 8, MT_THREADS)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int s = 0; s < MLP_K1 / 16; ++s)
        mma_bf16(tmem, mdesc(sb + M_OA + s * 2 * MT_THREADS * 16, MT_THREADS * 16, 128),
                 mdesc(sb + M_OW1 + s * 2 * MLP_HID * 16, MLP_HID * 16, 128), IDESC_BF16_M128_N64, s > 0);
      mma_commit(&bar);
    }
    __syncwarp();
    // the next tile's channel values travel while the MMAs run
    const int tn = t + gridDim.x;
    if (tn < ntiles) load_box(tn, nxt);
    ok = __syncthreads_and(bar_wait(&bar, phase));
    phase ^= 1u;
    if (!ok) break;
    tc_fence_after();
    // layer 1 epilogue: z1 + b1 -> GELU -> BF16 row of the layer-2 A operand, written
    // over the layer-1 operand (its MMAs completed)
    float z[MLP_HID];
#pragma unroll
    for (int q = 0; q < MLP_HID / 16; ++q) tmem_ld16(lane_base + q * 16, z + q * 16);
    tmem_wait_ld();
#pragma unroll
    for (int q = 0; q < MLP_HID / 8; ++q) {
      uint32_t pk[4];
#pragma unroll
      for (int h = 0; h < 4; ++h)
        pk[h] = pack_bf16(gelu_fast(z[q * 8 + 2 * h] + sB1[q * 8 + 2 * h]),
                          gelu_fast(z[q * 8 + 2 * h + 1] + sB1[q * 8 + 2 * h + 1]));
      *reinterpret_cast<uint4*>(base + M_OA + kmaj(tid, q * 8, MT_THREADS)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int s = 0; s < MLP_HID / 16; ++s)
        mma_bf16(tmem, mdesc(sb + M_OA + s * 2 * MT_THREADS * 16, MT_THREADS * 16, 128),
                 mdesc(sb + M_OW2 + s * 2 * MLP_HID * 16, MLP_HID * 16, 128), IDESC_BF16_M128_N64, s > 0);
      mma_commit(&bar);
    }
    __syncwarp();
    // the box of this tile is no longer read: the next tile's goes in while the MMAs run
    if (tn < ntiles) store_box(nxt);
    ok = __syncthreads_and(bar_wait(&bar, phase));
    phase ^= 1u;
    if (!ok) break;
    tc_fence_after();
    // layer 2 epilogue and layer 3 (64 -> 2) in FP32
#pragma unroll
    for (int q = 0; q < MLP_HID / 16; ++q) tmem_ld16(lane_base + q * 16, z + q * 16);
    tmem_wait_ld();
    float y0 = sB3[0], y1 = sB3[1];
#pragma unroll
    for (int h = 0; h < MLP_HID; ++h) {
      const float hv = gelu_fast(z[h] + sB2[h]);
      y0 = fmaf(sW3[h], hv, y0);
      y1 = fmaf(sW3[MLP_HID + h], hv, y1);
    }
    tc_fence_before();
    const int i = i0 + c, j = j0 + rr;
    if (i < g.Nz && j < g.Nr) {
      const long long o = (long long)j * g.P + i;
      const double ramp = __ldg(at.ramp + i);
      const double p0 = (double)(y0 * a.norm.out_scale[0]) * ramp;
      const double p1 = (double)(y1 * a.norm.out_scale[1]) * ramp;
      if (at.mode == 0) {
        at.out[o] = p0;
        at.out[g.plane + o] = p1;
      } else {
        const unsigned char m = __ldg(at.mask + o);
        at.out[g.plane + o] = (m & 1) ? __ldg(at.held + o) : p0;
        at.out[2 * g.plane + o] = (m & 2) ? __ldg(at.held + g.plane + o) : p1;
      }
    }
    fence_async_smem();  // the next tile's box (generic writes) before its A operand is built
    __syncthreads();
  }
  if (!ok) {
    if (tid == 0) atomicOr(a.flags, 4);
    // let the MMA whose completion timed out finish (bounded) before the columns are
    // released (phase was already advanced past it)
    bar_wait(&bar, phase ^ 1u);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem, 64);
}

cudaError_t mlp_init_attributes() {
  cudaError_t e = cudaFuncSetAttribute(mlp_infer_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)M_SMEM);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(mlp_infer_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)M_SMEM);
}

cudaError_t launch_mlp_infer(const InferArgs& a, cudaStream_t s) {
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  // at most 4 CTAs per SM (shared memory): 4 x 64 of the 512 TMEM columns
  const int grid = a.ntiles < M_CTAS_PER_SM * nsm ? a.ntiles : M_CTAS_PER_SM * nsm;
  if (grid <= 0) return cudaSuccess;
  mlp_infer_kernel<false><<<grid, MT_THREADS, M_SMEM, s>>>(a, nullptr, nullptr, a.ntiles);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Judge
// ---------------------------------------------------------------------------
__device__ __forceinline__ void judge_body(const JudgeArgs& a, long long p) {
  const Grid g = a.g;
  const long long n = (long long)g.Nz * g.Nr;
  unsigned long long fb = 0, judged = 0;
  if (p < n) {
    const int j = (int)(p / g.Nz), i = (int)(p - (long long)j * g.Nz);
    const long long o = (long long)j * g.P + i;
    unsigned char m = 0;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const double* pl = a.plain + k * g.plane;
      double lm = 0.0;
      for (int dr = -2; dr <= 2; ++dr)
        for (int dz = -2; dz <= 2; ++dz) {
          const int ii = i + dz, jj = j + dr;
          if (ii >= 0 && ii < g.Nz && jj >= 0 && jj < g.Nr) lm = fmax(lm, fabs(__ldg(pl + (long long)jj * g.P + ii)));
        }
      const double plain = __ldg(pl + o);
      const double pred = __ldg(a.pred + k * g.plane + o);
      if (fabs(pred - plain) > a.thr * lm) m |= (unsigned char)(1 << k);
      a.held[k * g.plane + o] = plain;
    }
    a.mask[o] = m;
    judged = 2;
    fb = (m & 1) + ((m >> 1) & 1);
  }
  // warp totals, one atomic per warp
  for (int off = 16; off > 0; off >>= 1) {
    fb += __shfl_down_sync(0xffffffffu, fb, off);
    judged += __shfl_down_sync(0xffffffffu, judged, off);
  }
  if ((threadIdx.x & 31) == 0 && judged) {
    atomicAdd(a.counts + 0, judged);
    atomicAdd(a.counts + 1, fb);
  }
}

__global__ void judge_kernel(const JudgeArgs a) { judge_body(a, (long long)blockIdx.x * blockDim.x + threadIdx.x); }

// Batched: blockIdx.y = instance.
__global__ void judge_kernel_batch(const JudgeArgs* __restrict__ argv) {
  judge_body(argv[blockIdx.y], (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

cudaError_t launch_judge_batch(const JudgeArgs* argv, int ninst, long long max_pts, cudaStream_t s) {
  const int bs = 256;
  judge_kernel_batch<<<dim3((unsigned)((max_pts + bs - 1) / bs), ninst), bs, 0, s>>>(argv);
  return cudaGetLastError();
}

cudaError_t launch_features_batch(const FeatArgs* argv, const int4* tiles, int ntiles, int grid, cudaStream_t s) {
  if (ntiles <= 0) return cudaSuccess;
  features_kernel_batch<<<grid, 256, 0, s>>>(argv, tiles, ntiles);
  return cudaGetLastError();
}

cudaError_t launch_mlp_infer_batch(const InferArgs& a0, const InferArgs* argv, const int4* tiles, int ntiles,
                                   cudaStream_t s) {
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int grid = ntiles < M_CTAS_PER_SM * nsm ? ntiles : M_CTAS_PER_SM * nsm;
  if (grid <= 0) return cudaSuccess;
  mlp_infer_kernel<true><<<grid, MT_THREADS, M_SMEM, s>>>(a0, argv, tiles, ntiles);
  return cudaGetLastError();
}

cudaError_t launch_judge(const JudgeArgs& a, cudaStream_t s) {
  const long long n = (long long)a.g.Nz * a.g.Nr;
  const int bs = 256;
  judge_kernel<<<(int)((n + bs - 1) / bs), bs, 0, s>>>(a);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Training (FP32)
// ---------------------------------------------------------------------------
__host__ __device__ inline uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Sample b of training step `step`: snapshot u % S, point (u >> 32) % (Nz*Nr).
__global__ void sample_kernel(const Dataset d, const MlpNorm norm, unsigned long long seed, const int* step, int B,
                              float* X, float* T) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)B * MLP_K1) return;
  const int b = (int)(e / MLP_K1), k = (int)(e - (long long)b * MLP_K1);
  const uint64_t u = mix64(mix64(seed + (uint64_t)(*step) * 0x9E3779B97F4A7C15ull) + (uint64_t)b);
  const int s = (int)(u % (uint64_t)d.S);
  const long long npts = (long long)d.g.Nz * d.g.Nr;
  const long long p = (long long)((u >> 32) % (uint64_t)npts);
  const int j = (int)(p / d.g.Nz), i = (int)(p - (long long)j * d.g.Nz);
  float v = 0.0f;
  if (k < MLP_IN) {
    const int ch = k / 25, w = k - ch * 25, dr = w / 5 - 2, dz = w % 5 - 2;
    const int ii = i + dz, jj = j + dr;
    float raw = 0.0f;
    if (ii >= 0 && ii < d.g.Nz && jj >= 0 && jj < d.g.Nr) {
      const float4 f = __ldg(d.feat + (long long)s * d.g.plane + (long long)jj * d.g.P + ii);
      raw = ch == 0 ? f.x : (ch == 1 ? f.y : (ch == 2 ? f.z : f.w));
    }
    v = (raw - norm.feat_mean[ch]) * norm.feat_inv_scale[ch];
  }
  X[e] = v;
  if (k < MLP_OUT) {
    const float2 t = __ldg(d.targ + (long long)s * d.g.plane + (long long)j * d.g.P + i);
    T[(long long)b * MLP_OUT + k] = (k == 0 ? t.x : t.y) / norm.out_scale[k];
  }
}

cudaError_t launch_sample(const Dataset& d, MlpNorm norm, unsigned long long seed, const int* step, int B, float* X,
                          float* T, cudaStream_t s) {
  const long long n = (long long)B * MLP_K1;
  const int bs = 256;
  sample_kernel<<<(int)((n + bs - 1) / bs), bs, 0, s>>>(d, norm, seed, step, B, X, T);
  return cudaGetLastError();
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(256) gemm_kernel(int M, int N, int K, const float* __restrict__ A, int lda,
                                                   const float* __restrict__ B, int ldb, float* __restrict__ C,
                                                   int ldc, int kchunk, int atomic) {
  __shared__ float As[16][64 + 4];  // [k][m]
  __shared__ float Bs[16][64 + 4];  // [k][n]
  const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
  const int kbeg = blockIdx.z * kchunk;
  const int kend = min(K, kbeg + kchunk);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  float acc[4][4];
#pragma unroll
  for (int x = 0; x < 4; ++x)
#pragma unroll
    for (int y = 0; y < 4; ++y) acc[x][y] = 0.0f;
  for (int k0 = kbeg; k0 < kend; k0 += 16) {
    for (int e = threadIdx.x; e < 1024; e += 256) {
      int mm, kk;
      if (TA) { kk = e >> 6; mm = e & 63; } else { mm = e >> 4; kk = e & 15; }
      const int m = m0 + mm, k = k0 + kk;
      float v = 0.0f;
      if (m < M && k < kend) v = TA ? A[(long long)k * lda + m] : A[(long long)m * lda + k];
      As[kk][mm] = v;
    }
    for (int e = threadIdx.x; e < 1024; e += 256) {
      int nn, kk;
      if (TB) { nn = e >> 4; kk = e & 15; } else { kk = e >> 6; nn = e & 63; }
      const int n = n0 + nn, k = k0 + kk;
      float v = 0.0f;
      if (n < N && k < kend) v = TB ? B[(long long)n * ldb + k] : B[(long long)k * ldb + n];
      Bs[kk][nn] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) {
      float av[4], bv[4];
#pragma unroll
      for (int x = 0; x < 4; ++x) av[x] = As[kk][ty * 4 + x];
#pragma unroll
      for (int y = 0; y < 4; ++y) bv[y] = Bs[kk][tx * 4 + y];
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y) acc[x][y] = fmaf(av[x], bv[y], acc[x][y]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int x = 0; x < 4; ++x)
#pragma unroll
    for (int y = 0; y < 4; ++y) {
      const int m = m0 + ty * 4 + x, n = n0 + tx * 4 + y;
      if (m < M && n < N) {
        float* dst = C + (long long)m * ldc + n;
        if (atomic) atomicAdd(dst, acc[x][y]);
        else *dst = acc[x][y];
      }
    }
}

cudaError_t launch_gemm(bool TA, bool TB, int M, int N, int K, const float* A, int lda, const float* B, int ldb,
                        float* C, int ldc, int ksplit, cudaStream_t s) {
  if (ksplit < 1) ksplit = 1;
  int kchunk = (K + ksplit - 1) / ksplit;
  kchunk = (kchunk + 15) / 16 * 16;
  const int nz = (K + kchunk - 1) / kchunk;
  const dim3 grid((N + 63) / 64, (M + 63) / 64, nz);
  const int atomic = ksplit > 1 ? 1 : 0;
  if (!TA && TB) gemm_kernel<false, true><<<grid, 256, 0, s>>>(M, N, K, A, lda, B, ldb, C, ldc, kchunk, atomic);
  else if (!TA && !TB) gemm_kernel<false, false><<<grid, 256, 0, s>>>(M, N, K, A, lda, B, ldb, C, ldc, kchunk, atomic);
  else if (TA && !TB) gemm_kernel<true, false><<<grid, 256, 0, s>>>(M, N, K, A, lda, B, ldb, C, ldc, kchunk, atomic);
  else gemm_kernel<true, true><<<grid, 256, 0, s>>>(M, N, K, A, lda, B, ldb, C, ldc, kchunk, atomic);
  return cudaGetLastError();
}

__global__ void bias_gelu_kernel(float* Z, const float* b, float* H, long long n, int N) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const float z = Z[e] + b[e % N];
  Z[e] = z;
  if (H) H[e] = gelu_f(z);
}

cudaError_t launch_bias_gelu(float* Z, const float* b, float* H, int B, int N, cudaStream_t s) {
  const long long n = (long long)B * N;
  bias_gelu_kernel<<<(int)((n + 255) / 256), 256, 0, s>>>(Z, b, H, n, N);
  return cudaGetLastError();
}
cudaError_t launch_bias(float* Z, const float* b, int B, int N, cudaStream_t s) {
  return launch_bias_gelu(Z, b, nullptr, B, N, s);
}

__global__ void loss_kernel(const float* Y, const float* T, float* dY, float* loss, const int* step, int B) {
  __shared__ float red[8];
  const long long n = (long long)B * MLP_OUT;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  float sq = 0.0f;
  if (e < n) {
    const float d = Y[e] - T[e];
    dY[e] = 2.0f * d / (float)B;
    sq = d * d;
  }
  for (int off = 16; off > 0; off >>= 1) sq += __shfl_down_sync(0xffffffffu, sq, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sq;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.0f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    atomicAdd(loss + *step, t / (float)B);
  }
}

cudaError_t launch_loss(const float* Y, const float* T, float* dY, float* loss, const int* step, int B,
                        cudaStream_t s) {
  const long long n = (long long)B * MLP_OUT;
  loss_kernel<<<(int)((n + 255) / 256), 256, 0, s>>>(Y, T, dY, loss, step, B);
  return cudaGetLastError();
}

__global__ void gelu_bwd_kernel(float* dH, const float* Z, long long n) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) dH[e] = dH[e] * gelu_grad_f(Z[e]);
}

cudaError_t launch_gelu_bwd(float* dH, const float* Z, int n, cudaStream_t s) {
  gelu_bwd_kernel<<<(n + 255) / 256, 256, 0, s>>>(dH, Z, n);
  return cudaGetLastError();
}

// Column sums over rows: block of 256 threads = 4 row lanes x 64 columns, 512 rows per block.
__global__ void colsum_kernel(const float* dZ, float* db, int B, int N) {
  __shared__ float red[4][64];
  const int col = threadIdx.x & 63, lane = threadIdx.x >> 6;
  const int r0 = blockIdx.x * 512;
  float s = 0.0f;
  if (col < N)
    for (int r = r0 + lane; r < min(B, r0 + 512); r += 4) s += dZ[(long long)r * N + col];
  red[lane][col] = s;
  __syncthreads();
  if (lane == 0 && col < N) atomicAdd(db + col, red[0][col] + red[1][col] + red[2][col] + red[3][col]);
}

cudaError_t launch_colsum(const float* dZ, float* db, int B, int N, cudaStream_t s) {
  colsum_kernel<<<(B + 511) / 512, 256, 0, s>>>(dZ, db, B, N);
  return cudaGetLastError();
}

__global__ void adam_kernel(float* p, const float* g, float* m, float* v, int n, const int* step, float lr, float b1,
                            float b2, float eps) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const float t = (float)(*step + 1);
  const float gg = g[e];
  const float mm = b1 * m[e] + (1.0f - b1) * gg;
  const float vv = b2 * v[e] + (1.0f - b2) * gg * gg;
  m[e] = mm;
  v[e] = vv;
  const float mhat = mm / (1.0f - powf(b1, t));
  const float vhat = vv / (1.0f - powf(b2, t));
  p[e] = p[e] - lr * mhat / (sqrtf(vhat) + eps);
}

cudaError_t launch_adam(float* p, const float* g, float* m, float* v, int n, const int* step, float lr, float b1,
                        float b2, float eps, cudaStream_t s) {
  adam_kernel<<<(n + 255) / 256, 256, 0, s>>>(p, g, m, v, n, step, lr, b1, b2, eps);
  return cudaGetLastError();
}

__global__ void step_inc_kernel(int* step) { *step += 1; }
cudaError_t launch_step_inc(int* step, cudaStream_t s) {
  step_inc_kernel<<<1, 1, 0, s>>>(step);
  return cudaGetLastError();
}

// acc: [0..3] channel sums, [4..7] channel sums of squares, [8..9] target sums of
// squares, [10] point count.
__global__ void dataset_stats_kernel(const Dataset d, double* acc) {
  __shared__ double red[11][8];
  double loc[11];
#pragma unroll
  for (int k = 0; k < 11; ++k) loc[k] = 0.0;
  const long long npts = (long long)d.g.Nz * d.g.Nr;
  const long long n = npts * d.S;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(e / npts);
    const long long p = e - (long long)s * npts;
    const int j = (int)(p / d.g.Nz), i = (int)(p - (long long)j * d.g.Nz);
    const long long o = (long long)s * d.g.plane + (long long)j * d.g.P + i;
    const float4 f = __ldg(d.feat + o);
    const float2 t = __ldg(d.targ + o);
    loc[0] += f.x; loc[1] += f.y; loc[2] += f.z; loc[3] += f.w;
    loc[4] += (double)f.x * f.x; loc[5] += (double)f.y * f.y; loc[6] += (double)f.z * f.z; loc[7] += (double)f.w * f.w;
    loc[8] += (double)t.x * t.x; loc[9] += (double)t.y * t.y;
    loc[10] += 1.0;
  }
#pragma unroll
  for (int k = 0; k < 11; ++k) {
    double v = loc[k];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < 11) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[threadIdx.x][w];
    atomicAdd(acc + threadIdx.x, t);
  }
}

cudaError_t launch_dataset_stats(const Dataset& d, double* acc, cudaStream_t s) {
  dataset_stats_kernel<<<148 * 4, 256, 0, s>>>(d, acc);
  return cudaGetLastError();
}

__global__ void pack_targets_kernel(const Grid g, const double* star, float2* targ) {
  const long long n = (long long)g.Nz * g.Nr;
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int j = (int)(p / g.Nz), i = (int)(p - (long long)j * g.Nz);
  const long long o = (long long)j * g.P + i;
  targ[o] = make_float2((float)star[g.plane + o], (float)star[2 * g.plane + o]);
}

cudaError_t launch_pack_targets(const Grid& g, const double* star, float2* targ, cudaStream_t s) {
  const long long n = (long long)g.Nz * g.Nr;
  pack_targets_kernel<<<(int)((n + 255) / 256), 256, 0, s>>>(g, star, targ);
  return cudaGetLastError();
}

}  // namespace axj
