// Per-vertex normals on sm_100a in two coalesced passes (wn_normals.h):
// face_contrib_kernel (one thread per face: the face normal and its corners'
// contributions, written once) and vertex_gather_kernel (thread t finishes the
// t-th vertex of the visit order, vertices by first incident face: its
// incidences' contributions added in face order, then the division by the
// length). The incidence lists are stored in visit order, so the gather's index
// reads are contiguous across a warp and only the contributions and the output
// row are addressed through the mesh. Nothing is scattered, so there are no
// atomics in the sums and no order dependence: uniform and area normals are
// bit-identical to the reference's serial loop (src/capi.mojo:146-202). Both
// passes stream their own arrays and gather the other side's, so the work is
// bound by memory traffic.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>

#include "wn_internal.h"
#include "wn_normals.cuh"
#include "wn_normals.h"

namespace wn {
namespace {

constexpr int kNormalThreads = 256;

// first[v] = nf and id[v] = v: the keys and values of the visit-order sort
// before the faces lower them.
__global__ void first_init_kernel(int64_t nv, int64_t nf, uint32_t* __restrict__ first,
                                  uint32_t* __restrict__ ids) {
  const int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  first[v] = static_cast<uint32_t>(nf);
  ids[v] = static_cast<uint32_t>(v);
}

// int64 faces -> int32 faces, and first[v] = the lowest face index on vertex v
// (an atomic minimum: the same result in any order). An index outside [0, nv)
// is counted in *bad and its face entry set to 0, so nothing downstream reads
// out of bounds.
__global__ void faces_prepare_kernel(const int64_t* __restrict__ F64, int64_t n, int64_t nv,
                                     int32_t* __restrict__ F32, uint32_t* __restrict__ first,
                                     int* bad) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t v = F64[i];
  const bool ok = v >= 0 && v < nv;
  if (!ok) atomicAdd(bad, 1);
  F32[i] = ok ? static_cast<int32_t>(v) : 0;
  if (ok) atomicMin(first + v, static_cast<uint32_t>(i / 3));
}

// rank[order[t]] = t.
__global__ void rank_kernel(const int32_t* __restrict__ order, int64_t nv,
                            uint32_t* __restrict__ rank) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= nv) return;
  rank[order[t]] = static_cast<uint32_t>(t);
}

// Incidence i = 3 * face + corner keyed by its vertex's visit rank (nv for an
// index outside [0, nv): a bucket past every vertex).
__global__ void incidence_keys_kernel(const int64_t* __restrict__ F64, int64_t n, int64_t nv,
                                      const uint32_t* __restrict__ rank,
                                      uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t v = F64[i];
  keys[i] = v >= 0 && v < nv ? rank[v] : static_cast<uint32_t>(nv);
  vals[i] = static_cast<uint32_t>(i);
}

// indptr[t] = first sorted position whose key is >= t, for t in [0, nv].
__global__ void csr_bounds_kernel(const uint32_t* keys, int64_t n, int64_t nv, int32_t* indptr) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t k = keys[i] < nv ? keys[i] : nv;
  const int64_t prev = i == 0 ? -1 : (keys[i - 1] < nv ? keys[i - 1] : nv);
  for (int64_t v = prev + 1; v <= k; ++v) indptr[v] = static_cast<int32_t>(i);
  if (i == n - 1)
    for (int64_t v = k + 1; v <= nv; ++v) indptr[v] = static_cast<int32_t>(n);
}

// One contribution record; x = NaN alone marks a face the reference skips.
__device__ __forceinline__ void store_record(double* r, double x, double y, double z) {
  r[0] = x;
  r[1] = y;
  r[2] = z;
}

// Position of vertex v (V rows of 3 doubles, 8-byte aligned) in two 16-byte
// loads: the 16-byte-aligned window [lo, lo + 32) that holds the row (the row
// starts at lo or at lo + 8). The window reaches 8 bytes past the row, into the
// neighbouring vertex, so the first and last vertices take three 8-byte loads.
__device__ __forceinline__ void load_vertex(const double* __restrict__ V, int32_t v, int64_t nv,
                                            double* p) {
  const double* src = V + 3 * static_cast<int64_t>(v);
  if (v == 0 || v == nv - 1) {
    p[0] = __ldg(src);
    p[1] = __ldg(src + 1);
    p[2] = __ldg(src + 2);
    return;
  }
  const uintptr_t a = reinterpret_cast<uintptr_t>(src);
  const double2* lo = reinterpret_cast<const double2*>(a & ~uintptr_t(15));
  const double2 w0 = __ldg(lo), w1 = __ldg(lo + 1);
  const bool at_lo = (a & 15) == 0;
  p[0] = at_lo ? w0.x : w0.y;
  p[1] = at_lo ? w0.y : w1.x;
  p[2] = at_lo ? w1.x : w1.y;
}

// One instance per weighting, so the uniform and area passes carry none of the
// angle weight's registers and fit 40 (six CTAs per SM, no spills). The CTA's
// face rows (3 int32 each, contiguous) are read into shared memory with 16-byte
// loads first, and each position with two (load_vertex), so a face issues about
// 7 load instructions instead of 12.
template <int mode>
__global__ void __launch_bounds__(kNormalThreads, mode == kNormalsAngle ? 1 : 6)
    face_contrib_kernel(const double* __restrict__ V, int64_t nv, const int32_t* __restrict__ F,
                        int64_t nf, double* __restrict__ contrib) {
  __shared__ __align__(16) int32_t sF[3 * kNormalThreads];
  const int64_t f0 = static_cast<int64_t>(blockIdx.x) * kNormalThreads;
  const int nb = nf - f0 < kNormalThreads ? static_cast<int>(nf - f0) : kNormalThreads;
  {
    // F + 3 f0 is 16-byte aligned: F is, and 3 * kNormalThreads * 4 bytes is a
    // multiple of 16.
    const int n = 3 * nb;
    const int4* src4 = reinterpret_cast<const int4*>(F + 3 * f0);
    for (int k = threadIdx.x; k < n / 4; k += kNormalThreads)
      reinterpret_cast<int4*>(sF)[k] = __ldg(src4 + k);
    for (int k = (n / 4) * 4 + threadIdx.x; k < n; k += kNormalThreads)
      sF[k] = __ldg(F + 3 * f0 + k);
  }
  __syncthreads();
  if (static_cast<int>(threadIdx.x) >= nb) return;
  const int64_t f = f0 + threadIdx.x;
  double P[3][3];
#pragma unroll
  for (int c = 0; c < 3; ++c) load_vertex(V, sF[3 * threadIdx.x + c], nv, P[c]);
  const double* Pp[3] = {P[0], P[1], P[2]};
  double u[3], norm;
  const bool keep = face_unit_normal(P[0], P[1], P[2], u, &norm);
  if constexpr (mode == kNormalsAngle) {
    double* out = contrib + 3 * kContribRecord * f;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (!keep) {
        out[kContribRecord * c] = __longlong_as_double(0x7ff8000000000000LL);  // skipped face
        continue;
      }
      const double w = corner_angle(Pp, c);
      store_record(out + kContribRecord * c, dmul(u[0], w), dmul(u[1], w), dmul(u[2], w));
    }
  } else {
    double* out = contrib + kContribRecord * f;
    if (!keep) {
      out[0] = __longlong_as_double(0x7ff8000000000000LL);
      return;
    }
    const double w = mode == kNormalsArea ? norm : 1.0;
    store_record(out, dmul(u[0], w), dmul(u[1], w), dmul(u[2], w));
  }
}

// Thread t finishes vertex order[t] from list t. Visiting the vertices by first
// incident face keeps the three readers of a face's contribution close together
// in time, so the repeat reads hit L2 (in vertex-index order they can be a whole
// mesh level apart), and the lists stored in visit order make the reads of
// indptr and entries contiguous across a warp. Each vertex's sum is unchanged:
// its incidences in face order.
__global__ void __launch_bounds__(kNormalThreads)
    vertex_gather_kernel(const int32_t* __restrict__ indptr, const int32_t* __restrict__ entries,
                         const int32_t* __restrict__ order, const double* __restrict__ contrib,
                         int64_t nv, int mode, double* __restrict__ N) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * kNormalThreads + threadIdx.x;
  if (t >= nv) return;
  const int64_t v = __ldg(order + t);
  double acc[3] = {0.0, 0.0, 0.0};
  const int32_t e1 = __ldg(indptr + t + 1);
  for (int32_t e = __ldg(indptr + t); e < e1; ++e) {
    const int32_t inc = __ldg(entries + e);
    const double* c =
        contrib + kContribRecord * static_cast<int64_t>(mode == kNormalsAngle ? inc : inc / 3);
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
  const unsigned vblocks = static_cast<unsigned>((t.nv + 255) / 256);
  const unsigned blocks = static_cast<unsigned>((n + 255) / 256);
  if (t.nv > 0) {
    first_init_kernel<<<vblocks, 256, 0, stream>>>(t.nv, t.nf, keys_in, vals_in);
    g_launches.fetch_add(1, std::memory_order_relaxed);
  }
  if (n > 0) {
    faces_prepare_kernel<<<blocks, 256, 0, stream>>>(F64, n, t.nv, t.F, keys_in, bad);
    g_launches.fetch_add(1, std::memory_order_relaxed);
  }
  if (t.nv == 0) return cudaMemsetAsync(t.indptr, 0, sizeof(int32_t), stream);
  // Visit order of the gather: vertices by first incident face (stable, so
  // ties keep index order; a vertex on no face has key nf and comes last).
  e = cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys_in, keys_out, vals_in,
                                      reinterpret_cast<uint32_t*>(t.order),
                                      static_cast<int>(t.nv), 0, key_bits(t.nf), stream);
  if (e != cudaSuccess) return e;
  if (n == 0) return cudaMemsetAsync(t.indptr, 0, sizeof(int32_t) * (t.nv + 1), stream);
  // The incidence lists in visit order: incidences sorted by their vertex's rank,
  // stably, so each list keeps incidence order (face, then corner).
  rank_kernel<<<vblocks, 256, 0, stream>>>(t.order, t.nv, keys_in);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  incidence_keys_kernel<<<blocks, 256, 0, stream>>>(F64, n, t.nv, keys_in, keys_out, vals_in);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  e = cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys_out, keys_in, vals_in,
                                      reinterpret_cast<uint32_t*>(t.entries),
                                      static_cast<int>(n), 0, key_bits(t.nv), stream);
  if (e != cudaSuccess) return e;
  csr_bounds_kernel<<<blocks, 256, 0, stream>>>(keys_in, n, t.nv, t.indptr);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError();
}

cudaError_t normals_eval(const NormalsTopology& t, const double* V, int mode, double* N,
                         cudaStream_t stream) {
  if (t.nv <= 0) return cudaSuccess;
  if (t.contrib_doubles < normals_contrib_doubles(t.nf, mode)) return cudaErrorInvalidValue;
  if (t.nf > 0) {
    const int64_t fb = (t.nf + kNormalThreads - 1) / kNormalThreads;
    const unsigned grid = static_cast<unsigned>(fb);
    if (mode == kNormalsAngle)
      face_contrib_kernel<kNormalsAngle><<<grid, kNormalThreads, 0, stream>>>(V, t.nv, t.F, t.nf,
                                                                              t.contrib);
    else if (mode == kNormalsArea)
      face_contrib_kernel<kNormalsArea><<<grid, kNormalThreads, 0, stream>>>(V, t.nv, t.F, t.nf,
                                                                             t.contrib);
    else
      face_contrib_kernel<kNormalsUniform><<<grid, kNormalThreads, 0, stream>>>(
          V, t.nv, t.F, t.nf, t.contrib);
    g_launches.fetch_add(1, std::memory_order_relaxed);
  }
  const int64_t vb = (t.nv + kNormalThreads - 1) / kNormalThreads;
  vertex_gather_kernel<<<static_cast<unsigned>(vb), kNormalThreads, 0, stream>>>(
      t.indptr, t.entries, t.order, t.contrib, t.nv, mode, N);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError();
}

}  // namespace wn
