// Per-vertex normals on sm_100a in two coalesced passes (wn_normals.h):
// face_contrib_kernel (one thread per face: the face normal and its corners'
// contributions, written once) and vertex_gather_kernel (one thread per vertex,
// vertices taken by first incident face: its incidences' contributions added in
// face order, then the division by the length). Nothing is scattered, so there are no atomics and no order
// dependence: uniform and area normals are bit-identical to the reference's
// serial loop (src/capi.mojo:146-202). Both passes stream their own arrays and
// gather the other side's, so the work is bound by memory traffic.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>

#include "wn_internal.h"
#include "wn_normals.cuh"
#include "wn_normals.h"

namespace wn {
namespace {

constexpr int kNormalThreads = 256;

// int64 faces -> int32 faces and sort keys (vertex ids); an index outside
// [0, nv) is counted in *bad, its face entry set to 0 and its key to nv (a
// bucket past every vertex), so nothing downstream reads out of bounds.
__global__ void faces_prepare_kernel(const int64_t* __restrict__ F64, int64_t n, int64_t nv,
                                     int32_t* __restrict__ F32, uint32_t* __restrict__ keys,
                                     uint32_t* __restrict__ vals, int* bad) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t v = F64[i];
  const bool ok = v >= 0 && v < nv;
  if (!ok) atomicAdd(bad, 1);
  F32[i] = ok ? static_cast<int32_t>(v) : 0;
  keys[i] = ok ? static_cast<uint32_t>(v) : static_cast<uint32_t>(nv);
  vals[i] = static_cast<uint32_t>(i);
}

// indptr[v] = first sorted position whose key is >= v, for v in [0, nv].
__global__ void csr_bounds_kernel(const uint32_t* keys, int64_t n, int64_t nv, int32_t* indptr) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t k = keys[i] < nv ? keys[i] : nv;
  const int64_t prev = i == 0 ? -1 : (keys[i - 1] < nv ? keys[i - 1] : nv);
  for (int64_t v = prev + 1; v <= k; ++v) indptr[v] = static_cast<int32_t>(i);
  if (i == n - 1)
    for (int64_t v = k + 1; v <= nv; ++v) indptr[v] = static_cast<int32_t>(n);
}

__global__ void __launch_bounds__(kNormalThreads)
    face_contrib_kernel(const double* __restrict__ V, const int32_t* __restrict__ F, int64_t nf,
                        int mode, double* __restrict__ contrib) {
  const int64_t f = static_cast<int64_t>(blockIdx.x) * kNormalThreads + threadIdx.x;
  if (f >= nf) return;
  double P[3][3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double* src = V + 3 * static_cast<int64_t>(F[3 * f + c]);
    P[c][0] = __ldg(src);
    P[c][1] = __ldg(src + 1);
    P[c][2] = __ldg(src + 2);
  }
  const double* Pp[3] = {P[0], P[1], P[2]};
  double u[3], norm;
  const bool keep = face_unit_normal(P[0], P[1], P[2], u, &norm);
  if (mode == kNormalsAngle) {
    double* out = contrib + 9 * f;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (!keep) {
        out[3 * c] = __longlong_as_double(0x7ff8000000000000LL);  // skipped face
        continue;
      }
      const double w = corner_angle(Pp, c);
      out[3 * c] = dmul(u[0], w);
      out[3 * c + 1] = dmul(u[1], w);
      out[3 * c + 2] = dmul(u[2], w);
    }
  } else {
    double* out = contrib + 3 * f;
    if (!keep) {
      out[0] = __longlong_as_double(0x7ff8000000000000LL);
      return;
    }
    const double w = mode == kNormalsArea ? norm : 1.0;
    out[0] = dmul(u[0], w);
    out[1] = dmul(u[1], w);
    out[2] = dmul(u[2], w);
  }
}

// Sort keys of the visit order: a vertex's first incident face (nf for a
// vertex on no face, so those come last).
__global__ void vertex_keys_kernel(const int32_t* __restrict__ indptr,
                                   const int32_t* __restrict__ entries, int64_t nv, int64_t nf,
                                   uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  const int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  const int32_t e0 = indptr[v];
  keys[v] = e0 < indptr[v + 1] ? static_cast<uint32_t>(entries[e0] / 3)
                               : static_cast<uint32_t>(nf);
  vals[v] = static_cast<uint32_t>(v);
}

// Thread t finishes vertex order[t]. Visiting the vertices by first incident
// face keeps the three readers of a face's contribution close together in time,
// so the repeat reads hit L2 (in vertex-index order they can be a whole mesh
// level apart). Each vertex's sum is unchanged: its incidences in face order.
__global__ void __launch_bounds__(kNormalThreads)
    vertex_gather_kernel(const int32_t* __restrict__ indptr, const int32_t* __restrict__ entries,
                         const int32_t* __restrict__ order, const double* __restrict__ contrib,
                         int64_t nv, int mode, double* __restrict__ N) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * kNormalThreads + threadIdx.x;
  if (t >= nv) return;
  const int64_t v = __ldg(order + t);
  double acc[3] = {0.0, 0.0, 0.0};
  const int32_t e1 = indptr[v + 1];
  for (int32_t e = indptr[v]; e < e1; ++e) {
    const int32_t inc = __ldg(entries + e);
    const double* c = contrib + 3 * static_cast<int64_t>(mode == kNormalsAngle ? inc : inc / 3);
    const double x = __ldg(c);
    if (isnan(x)) continue;  // a face the reference skips
    acc[0] = dadd(acc[0], x);
    acc[1] = dadd(acc[1], __ldg(c + 1));
    acc[2] = dadd(acc[2], __ldg(c + 2));
  }
  normal_finish(acc);
  N[3 * v] = acc[0];
  N[3 * v + 1] = acc[1];
  N[3 * v + 2] = acc[2];
}

int key_bits(int64_t max_key) {
  int b = 1;
  while (b < 32 && (int64_t(1) << b) <= max_key) ++b;
  return b;
}

size_t round256(size_t n) { return ((n + 255) / 256) * 256; }

}  // namespace

size_t normals_scratch_bytes(int64_t nf, int64_t nv) {
  const int64_t n = 3 * nf > nv ? 3 * nf : nv;  // the incidence sort, then the vertex sort
  size_t temp = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, temp, static_cast<const uint32_t*>(nullptr),
                                  static_cast<uint32_t*>(nullptr),
                                  static_cast<const uint32_t*>(nullptr),
                                  static_cast<uint32_t*>(nullptr), static_cast<int>(n));
  return 3 * round256(static_cast<size_t>(n) * 4) + temp + 256;
}

cudaError_t normals_build(NormalsTopology& t, const int64_t* F64, int* bad, void* scratch,
                          size_t scratch_bytes, cudaStream_t stream) {
  const int64_t n = 3 * t.nf;
  cudaError_t e = cudaMemsetAsync(bad, 0, sizeof(int), stream);
  if (e != cudaSuccess) return e;
  if (scratch_bytes < normals_scratch_bytes(t.nf, t.nv)) return cudaErrorInvalidValue;
  const size_t arr = round256(static_cast<size_t>(n > t.nv ? n : t.nv) * 4);
  unsigned char* s = static_cast<unsigned char*>(scratch);
  uint32_t* keys_in = reinterpret_cast<uint32_t*>(s);
  uint32_t* keys_out = reinterpret_cast<uint32_t*>(s + arr);
  uint32_t* vals_in = reinterpret_cast<uint32_t*>(s + 2 * arr);
  void* temp = s + 3 * arr;
  size_t temp_bytes = scratch_bytes - 3 * arr;
  if (n == 0) {
    e = cudaMemsetAsync(t.indptr, 0, sizeof(int32_t) * (t.nv + 1), stream);
  } else {
    const unsigned blocks = static_cast<unsigned>((n + 255) / 256);
    faces_prepare_kernel<<<blocks, 256, 0, stream>>>(F64, n, t.nv, t.F, keys_in, vals_in, bad);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    // Stable: equal vertex ids keep incidence order (face, then corner).
    e = cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys_in, keys_out, vals_in,
                                        reinterpret_cast<uint32_t*>(t.entries),
                                        static_cast<int>(n), 0, key_bits(t.nv), stream);
    if (e != cudaSuccess) return e;
    csr_bounds_kernel<<<blocks, 256, 0, stream>>>(keys_out, n, t.nv, t.indptr);
    g_launches.fetch_add(1, std::memory_order_relaxed);
  }
  if (e != cudaSuccess || t.nv == 0) return e;
  // Visit order of the gather: vertices by first incident face (stable, so
  // ties keep index order).
  const unsigned vblocks = static_cast<unsigned>((t.nv + 255) / 256);
  vertex_keys_kernel<<<vblocks, 256, 0, stream>>>(t.indptr, t.entries, t.nv, t.nf, keys_in,
                                                  vals_in);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  e = cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys_in, keys_out, vals_in,
                                      reinterpret_cast<uint32_t*>(t.order),
                                      static_cast<int>(t.nv), 0, key_bits(t.nf), stream);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

cudaError_t normals_eval(const NormalsTopology& t, const double* V, int mode, double* N,
                         cudaStream_t stream) {
  if (t.nv <= 0) return cudaSuccess;
  if (t.contrib_doubles < (mode == kNormalsAngle ? 9 : 3) * t.nf) return cudaErrorInvalidValue;
  if (t.nf > 0) {
    const int64_t fb = (t.nf + kNormalThreads - 1) / kNormalThreads;
    face_contrib_kernel<<<static_cast<unsigned>(fb), kNormalThreads, 0, stream>>>(
        V, t.F, t.nf, mode, t.contrib);
    g_launches.fetch_add(1, std::memory_order_relaxed);
  }
  const int64_t vb = (t.nv + kNormalThreads - 1) / kNormalThreads;
  vertex_gather_kernel<<<static_cast<unsigned>(vb), kNormalThreads, 0, stream>>>(
      t.indptr, t.entries, t.order, t.contrib, t.nv, mode, N);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError();
}

}  // namespace wn
