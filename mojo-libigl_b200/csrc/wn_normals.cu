// Per-vertex normals on sm_100a: a gather over each vertex's (face, corner)
// incidences in face order, the faces' terms recomputed per incidence with the
// reference's separately rounded arithmetic (wn_normals.cuh). Nothing is
// scattered, so no atomics and no order dependence: uniform and area normals
// are bit-identical to the reference's serial loop (src/capi.mojo:146-202).
// The work is a few hundred bytes of L1/L2 reads per vertex: the kernel is
// bound by memory latency and, for a mesh that fits in L2, by launch time.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>

#include "wn_internal.h"
#include "wn_normals.cuh"
#include "wn_normals.h"

namespace wn {
namespace {

constexpr int kNormalThreads = 128;

__global__ void iota_kernel(uint32_t* v, int64_t n) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) v[i] = static_cast<uint32_t>(i);
}

// indptr[v] = first sorted position whose key is >= v, for v in [0, nv].
__global__ void csr_bounds_kernel(const uint32_t* keys, int64_t n, int64_t nv, int32_t* indptr) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t k = keys[i];
  const int64_t prev = i == 0 ? -1 : static_cast<int64_t>(keys[i - 1]);
  for (int64_t v = prev + 1; v <= k; ++v) indptr[v] = static_cast<int32_t>(i);
  if (i == n - 1)
    for (int64_t v = k + 1; v <= nv; ++v) indptr[v] = static_cast<int32_t>(n);
}

__global__ void __launch_bounds__(kNormalThreads)
    vertex_normals_kernel(const double* __restrict__ V, const int32_t* __restrict__ F,
                          const int32_t* __restrict__ indptr, const int32_t* __restrict__ entries,
                          int64_t nv, int mode, double* __restrict__ N) {
  const int64_t v = static_cast<int64_t>(blockIdx.x) * kNormalThreads + threadIdx.x;
  if (v >= nv) return;
  double acc[3] = {0.0, 0.0, 0.0};
  const int32_t e1 = indptr[v + 1];
  for (int32_t e = indptr[v]; e < e1; ++e) {
    const int32_t inc = entries[e];
    const int32_t f = inc / 3, corner = inc - 3 * f;
    double P[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double* src = V + 3 * static_cast<int64_t>(__ldg(F + 3 * f + c));
      P[c][0] = __ldg(src);
      P[c][1] = __ldg(src + 1);
      P[c][2] = __ldg(src + 2);
    }
    normal_corner_add(P[0], P[1], P[2], corner, mode, acc);
  }
  normal_finish(acc);
  N[3 * v] = acc[0];
  N[3 * v + 1] = acc[1];
  N[3 * v + 2] = acc[2];
}

int key_bits(int64_t nv) {
  int b = 1;
  while (b < 32 && (int64_t(1) << b) < nv) ++b;
  return b;
}

}  // namespace

size_t normals_scratch_bytes(int64_t nf) {
  const int64_t n = 3 * nf;
  size_t temp = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, temp, static_cast<const uint32_t*>(nullptr),
                                  static_cast<uint32_t*>(nullptr),
                                  static_cast<const uint32_t*>(nullptr),
                                  static_cast<uint32_t*>(nullptr), static_cast<int>(n));
  const size_t arr = ((static_cast<size_t>(n) * 4 + 255) / 256) * 256;
  return 3 * arr + temp + 256;
}

cudaError_t normals_build(NormalsTopology& t, void* scratch, size_t scratch_bytes,
                          cudaStream_t stream) {
  const int64_t n = 3 * t.nf;
  if (n == 0) return cudaMemsetAsync(t.indptr, 0, sizeof(int32_t) * (t.nv + 1), stream);
  if (scratch_bytes < normals_scratch_bytes(t.nf)) return cudaErrorInvalidValue;
  const size_t arr = ((static_cast<size_t>(n) * 4 + 255) / 256) * 256;
  unsigned char* s = static_cast<unsigned char*>(scratch);
  uint32_t* keys_out = reinterpret_cast<uint32_t*>(s);
  uint32_t* vals_in = reinterpret_cast<uint32_t*>(s + arr);
  uint32_t* keys_in = reinterpret_cast<uint32_t*>(s + 2 * arr);
  void* temp = s + 3 * arr;
  size_t temp_bytes = scratch_bytes - 3 * arr;
  const unsigned blocks = static_cast<unsigned>((n + 255) / 256);
  cudaError_t e = cudaMemcpyAsync(keys_in, t.F, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice,
                                  stream);
  if (e != cudaSuccess) return e;
  iota_kernel<<<blocks, 256, 0, stream>>>(vals_in, n);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  // Stable: equal vertex ids keep incidence order (face, then corner).
  e = cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys_in, keys_out, vals_in,
                                      reinterpret_cast<uint32_t*>(t.entries), static_cast<int>(n),
                                      0, key_bits(t.nv), stream);
  if (e != cudaSuccess) return e;
  csr_bounds_kernel<<<blocks, 256, 0, stream>>>(keys_out, n, t.nv, t.indptr);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError();
}

cudaError_t normals_eval(const NormalsTopology& t, const double* V, int mode, double* N,
                         cudaStream_t stream) {
  if (t.nv <= 0) return cudaSuccess;
  const int64_t blocks = (t.nv + kNormalThreads - 1) / kNormalThreads;
  if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  vertex_normals_kernel<<<static_cast<unsigned>(blocks), kNormalThreads, 0, stream>>>(
      V, t.F, t.indptr, t.entries, t.nv, mode, N);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError();
}

}  // namespace wn
