// axj_prep.cu -- the patch preprocessing of axj_prep.cuh on the device: one thread per
// row for the face-list sizes, one thread per row for the descriptors, codes and face
// entries (after a host scan of the row sizes), one thread per tile for the tile classes.
#include <cuda_runtime.h>

#include <cstdio>
#include <vector>

#include "axj_prep.cuh"

namespace axj {

__global__ void prep_row_size_kernel(const PrepArgs a, int64_t* size) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (j <= a.Nr) size[j - 1] = prep_row_size(a, j);
}

__global__ void prep_row_kernel(const PrepArgs a, const int64_t* off, uint32_t* desc, unsigned char* zcode,
                                unsigned char* rcode, int* faces) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (j <= a.Nr) prep_row(a, j, off[j - 1], desc, zcode, rcode, faces);
}

__global__ void prep_tile_kernel(const uint32_t* desc, int64_t P, int64_t Nz, int64_t Nr, const int64_t* cands,
                                 int64_t ncand, unsigned char* flags) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < ncand)
    flags[t] = (unsigned char)prep_tile_flags(desc, P, Nz, Nr, cands[3 * t], cands[3 * t + 1], cands[3 * t + 2]);
}

namespace {
// device buffers of one preprocessing call, released on every exit
struct PrepBuffers {
  std::vector<void*> ptrs;
  ~PrepBuffers() {
    for (void* p : ptrs) cudaFree(p);
  }
  template <typename T>
  T* alloc(size_t n, cudaError_t* e) {
    void* p = nullptr;
    if (*e == cudaSuccess) *e = cudaMalloc(&p, (n ? n : 1) * sizeof(T));
    if (*e == cudaSuccess) ptrs.push_back(p);
    return static_cast<T*>(p);
  }
};
}  // namespace

int prep_on_device(const PrepArgs& host_args, const int64_t* cands, int64_t ncand, uint32_t* desc,
                   unsigned char* zcode, unsigned char* rcode, std::vector<int>& faces, unsigned char* flags,
                   char* msg, int msglen) {
  const PrepArgs& h = host_args;
  const size_t plane = (size_t)h.P * (size_t)h.Nr;
  PrepBuffers b;
  cudaError_t e = cudaSuccess;
  axj_patch* d_patch = b.alloc<axj_patch>((size_t)h.npatch, &e);
  double* d_ib = b.alloc<double>((size_t)h.Nz * h.Nr, &e);
  int64_t* d_size = b.alloc<int64_t>((size_t)h.Nr, &e);
  uint32_t* d_desc = b.alloc<uint32_t>(plane, &e);
  unsigned char* d_z = b.alloc<unsigned char>(plane, &e);
  unsigned char* d_r = b.alloc<unsigned char>(plane, &e);
  int64_t* d_cand = b.alloc<int64_t>((size_t)(3 * ncand), &e);
  unsigned char* d_flags = b.alloc<unsigned char>((size_t)ncand, &e);
  if (e == cudaSuccess && h.npatch)
    e = cudaMemcpy(d_patch, h.patches, sizeof(axj_patch) * h.npatch, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_ib, h.ibval, sizeof(double) * h.Nz * h.Nr, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && ncand)
    e = cudaMemcpy(d_cand, cands, sizeof(int64_t) * 3 * ncand, cudaMemcpyHostToDevice);
  PrepArgs a = h;
  a.patches = d_patch;
  a.ibval = d_ib;
  const int bs = 128;
  const unsigned rows_grid = (unsigned)((h.Nr + bs - 1) / bs);
  if (e == cudaSuccess) {
    prep_row_size_kernel<<<rows_grid, bs>>>(a, d_size);
    e = cudaGetLastError();
  }
  std::vector<int64_t> size((size_t)h.Nr), off((size_t)h.Nr);
  if (e == cudaSuccess) e = cudaMemcpy(size.data(), d_size, sizeof(int64_t) * h.Nr, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    std::snprintf(msg, msglen, "patch preprocessing: %s", cudaGetErrorString(e));
    return AXJ_ERR_CUDA;
  }
  int64_t total = 1;  // faces[0] = 0: descriptors without face operations point there
  for (int64_t j = 0; j < h.Nr; ++j) {
    if (size[j] < 0) {
      std::snprintf(msg, msglen, "more than %d face operations at a point of row %lld", MAX_FACE_OPS,
                    (long long)j + 1);
      return AXJ_ERR_BADPATCH;
    }
    off[j] = total;
    total += size[j];
  }
  if (total >= (1 << 20)) {
    std::snprintf(msg, msglen, "too many face points");
    return AXJ_ERR_BADPATCH;
  }
  int* d_faces = b.alloc<int>((size_t)total, &e);
  int64_t* d_off = b.alloc<int64_t>((size_t)h.Nr, &e);
  if (e == cudaSuccess) e = cudaMemset(d_faces, 0, sizeof(int) * total);
  if (e == cudaSuccess) e = cudaMemcpy(d_off, off.data(), sizeof(int64_t) * h.Nr, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    prep_row_kernel<<<rows_grid, bs>>>(a, d_off, d_desc, d_z, d_r, d_faces);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && ncand) {
    prep_tile_kernel<<<(unsigned)((ncand + bs - 1) / bs), bs>>>(d_desc, h.P, h.Nz, h.Nr, d_cand, ncand, d_flags);
    e = cudaGetLastError();
  }
  faces.assign((size_t)total, 0);
  if (e == cudaSuccess) e = cudaMemcpy(desc, d_desc, sizeof(uint32_t) * plane, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(zcode, d_z, plane, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(rcode, d_r, plane, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(faces.data(), d_faces, sizeof(int) * total, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && ncand) e = cudaMemcpy(flags, d_flags, (size_t)ncand, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    std::snprintf(msg, msglen, "patch preprocessing: %s", cudaGetErrorString(e));
    return AXJ_ERR_CUDA;
  }
  return AXJ_OK;
}

}  // namespace axj
