// axj_noalloc.cu -- ComputeTimeStep for callers that cannot allocate device memory.
//
// The handle-based entry points allocate their buffers with cudaMalloc in axj_create.
// Some hosts cannot do that: code running where the allocator is owned by someone else
// (a framework's caching allocator, a Fortran host that hands in its own device arrays,
// a process that must not grow its device footprint after start-up). For them,
// axj_compute_dt_noalloc evaluates the time step from device arrays the caller owns.
// The only scratch it needs is the per-block minima and a completion counter of its
// reduction, and that lives in the file-scope array g_dt_scratch below: every GPU that
// loads this library holds it (about 512 KB) until the process exits.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>

#include "../../include/axj.h"
#include "axj_common.cuh"
#include "axj_kernels.cuh"
#include "axj_point.cuh"
#include "axj_pow.cuh"

namespace {

constexpr int NA_THREADS = 256;                       // one grid point per thread
constexpr int NA_MAX_BLOCKS = 65536;                  // at most 16,777,216 points
constexpr long long NA_MAX_POINTS = (long long)NA_MAX_BLOCKS * NA_THREADS;
constexpr int NA_COUNTER = NA_MAX_BLOCKS;             // slot of the completion counter
constexpr int NA_BAD = NA_MAX_BLOCKS + 1;             // slot of the non-finite flag

// The scratch: one partial minimum per block, then two 32-bit words (counter, flag)
// kept in the slots after them. Every call shares it and it keeps the last call's
// contents; each call clears the two words before its kernel runs.
static __device__ __align__(256) double g_dt_scratch[NA_MAX_BLOCKS + 2];
// the tables of the FP64 power mu = T**0.666 (axj_pow.cuh), written by the first call on
// each device
static __device__ double g_na_pow[axj::POW_TAB];

__device__ __forceinline__ double na_warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Per-point dt of ComputeTimeStep (ModInputOutput.f90:395-416), block minimum, and the
// last block to finish reduces the per-block minima.
__global__ void __launch_bounds__(NA_THREADS)
    dt_noalloc_kernel(const double* __restrict__ U, long long P, long long plane, int Nz, int Nr,
                      const double* __restrict__ dxidz, const double* __restrict__ detadr,
                      const double* __restrict__ ibval, double staleT, axj::Consts c, double* scratch,
                      double* __restrict__ dt) {
  unsigned int* counter = reinterpret_cast<unsigned int*>(scratch + NA_COUNTER);
  unsigned int* bad = reinterpret_cast<unsigned int*>(scratch + NA_BAD);
  const long long n = (long long)Nz * Nr;
  const long long p = (long long)blockIdx.x * NA_THREADS + threadIdx.x;
  double v = 1.0e300;
  if (p < n) {
    const int j = (int)(p / Nz), i = (int)(p - (long long)j * Nz);
    const long long o = (long long)j * P + i;
    if (ibval && __ldg(ibval + o) == 0.0) {
      v = 100.0;
    } else {
      const double Vr = __ldg(U + 1 * plane + o), Vz = __ldg(U + 3 * plane + o), T = __ldg(U + 4 * plane + o);
      // mu = T**0.666 (AssignValues) from the table-driven power of the handle-based kernels
      const double mu = axj::pow0666(T, g_na_pow);
      const double beta = (3.0 / 5.0) * mu;
      const double lambda = beta - (2.0 / 3.0) * mu;
      const bool phys = c.dt_mode == axj::DT_PHYSICAL;
      v = axj::dt_point(Vz, Vr, phys ? T : staleT, mu, lambda, mu, __ldg(dxidz + i), __ldg(detadr + j), c);
      // an infinite input gives dt = 0, a finite-looking minimum: flag it with the NaNs
      if (!isfinite(Vr) || !isfinite(Vz) || !isfinite(T)) atomicOr(bad, 1u);
    }
    if (!(v == v)) atomicOr(bad, 1u);
  }
  __shared__ double sred[NA_THREADS / 32];
  __shared__ bool last;
  v = na_warp_min(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sred[w] = v;
  __syncthreads();
  if (w == 0) {
    v = lane < NA_THREADS / 32 ? sred[lane] : 1.0e300;
    v = na_warp_min(v);
    if (lane == 0) {
      scratch[blockIdx.x] = v;
      __threadfence();
      last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    }
  }
  __syncthreads();
  if (last) {
    __threadfence();
    double m = 1.0e300;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += NA_THREADS) m = fmin(m, ((volatile double*)scratch)[b]);
    m = na_warp_min(m);
    if (lane == 0) sred[w] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
      double r = sred[0];
      for (int k = 1; k < NA_THREADS / 32; ++k) r = fmin(r, sred[k]);
      *dt = (*(volatile unsigned int*)bad) ? __longlong_as_double(0x7ff8000000000000LL) : r;
    }
  }
}

// Device address of g_dt_scratch per device ordinal, fetched once with that device
// current (the host-side name of a __device__ array is only a stand-in).
std::mutex g_na_lock;
double* g_na_ptr[128] = {nullptr};

}  // namespace

extern "C" int axj_compute_dt_noalloc(const double* d_pv, int64_t pitch, int64_t Nz, int64_t Nr,
                                      const double* d_dxidz, const double* d_detadr, const double* d_ibval,
                                      const axj_params* params, double stale_T, double* d_dt, void* stream) {
  char msg[256];
  if (!d_pv || !d_dxidz || !d_detadr || !params || !d_dt || Nz < 1 || Nr < 1 || pitch < Nz) {
    axj::set_global_error("axj_compute_dt_noalloc: null pointer or bad size");
    return AXJ_ERR_ARG;
  }
  // each factor is bounded before the product is formed (no overflow on any input)
  if (Nz > NA_MAX_POINTS || Nr > NA_MAX_POINTS / Nz) {
    std::snprintf(msg, sizeof(msg),
                  "axj_compute_dt_noalloc: %lld x %lld points exceed the built-in scratch limit of %lld points",
                  (long long)Nz, (long long)Nr, NA_MAX_POINTS);
    axj::set_global_error(msg);
    return AXJ_ERR_ARG;
  }
  // 5 planes of pitch x Nr doubles must be addressable
  if (pitch > (INT64_MAX / 8 / 5) / Nr) {
    axj::set_global_error("axj_compute_dt_noalloc: row pitch too large");
    return AXJ_ERR_ARG;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128) {
    axj::set_global_error("axj_compute_dt_noalloc: no current CUDA device");
    return AXJ_ERR_NODEVICE;
  }
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> g(g_na_lock);
    if (!g_na_ptr[dev]) {
      static double tab[axj::POW_TAB];
      axj::pow0666_fill(tab);
      cudaError_t e = cudaMemcpyToSymbol(g_na_pow, tab, sizeof tab);
      if (e == cudaSuccess) e = cudaGetSymbolAddress(reinterpret_cast<void**>(&g_na_ptr[dev]), g_dt_scratch);
      if (e != cudaSuccess) {
        g_na_ptr[dev] = nullptr;
        std::snprintf(msg, sizeof(msg), "axj_compute_dt_noalloc: device set-up failed: %s",
                      cudaGetErrorString(e));
        axj::set_global_error(msg);
        return AXJ_ERR_CUDA;
      }
    }
    scratch = g_na_ptr[dev];
  }
  axj::Consts c{};
  c.Re = params->Re;
  c.Pr = params->Pr;
  c.CFL = params->CFL;
  c.dt_mode = (int)params->dt_mode;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the counter and the flag must start at zero; the per-block minima are written
  // before they are read
  cudaError_t e = cudaMemsetAsync(scratch + NA_COUNTER, 0, 2 * sizeof(double), s);
  if (e == cudaSuccess) {
    const long long n = Nz * Nr;
    const int blocks = (int)((n + NA_THREADS - 1) / NA_THREADS);
    dt_noalloc_kernel<<<blocks, NA_THREADS, 0, s>>>(d_pv, (long long)pitch, (long long)pitch * Nr, (int)Nz, (int)Nr,
                                                    d_dxidz, d_detadr, d_ibval, stale_T, c, scratch, d_dt);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    std::snprintf(msg, sizeof(msg), "axj_compute_dt_noalloc: %s", cudaGetErrorString(e));
    axj::set_global_error(msg);
    return AXJ_ERR_CUDA;
  }
  return AXJ_OK;
}
