// Closest-point traversal of the median-split hierarchy on sm_100a: one thread
// per query, the reference's ordered depth-first walk (src/capi.mojo:522-586)
// with its exact FP64 arithmetic (wn_aabb.cuh), so distances, face indices and
// closest points are bit-identical to the reference's CPU path, ties included.
//
// The walk is a chain of dependent reads (node record -> child boxes -> next
// node) over a tree that sits in L2 (a 327,680-face mesh: 21.0 MB of node
// records + 26 MB of face records), so the kernel is bound by load latency and
// FP64 issue, not by HBM bandwidth. What helps is keeping a warp's 32 walks
// alike: above kAabbSortMin queries the threads take their queries in Morton
// order (perm), and every record is read with 16-byte non-coherent loads.
//
// Each stack entry keeps the box distance computed when it was pushed. The
// reference recomputes that distance from the same box when it pops the node;
// the value is the same double, so the pop-time test `d > best` is unchanged.
// The stored key is max(box distance, slab bound) (wn_aabb.h): a child is
// pushed, and later expanded, only when both are <= best. The push order is
// decided by the box distances alone, as in the reference.
#include <cuda_runtime.h>

#include "wn_aabb.cuh"
#include "wn_aabb.h"
#include "wn_common.cuh"
#include "wn_internal.h"

namespace wn {
namespace {

constexpr int kAabbThreads = 128;

struct AabbArgs {
  const AabbNodeRec* __restrict__ nodes;
  const AabbTriRec* __restrict__ tris;
  const double* __restrict__ P;
  const uint32_t* __restrict__ perm;
  double* __restrict__ sqrd;
  int64_t* __restrict__ index;
  double* __restrict__ closest;
  int* err;
  int64_t np, nnodes;
  double root[6];
  double scale;
};

__device__ __forceinline__ double2 ldg2(const double* p) {
  return __ldg(reinterpret_cast<const double2*>(p));
}

// Squared lower bound on the distance from p to the faces inside a slab, less
// the rounding margin `e` (0 when the slab cannot separate them).
__device__ __forceinline__ double slab_bound2(double px, double py, double pz, float nx, float ny,
                                              float nz, float lo, float hi, double e) {
  const double t = fma(static_cast<double>(nz), pz,
                       fma(static_cast<double>(ny), py, static_cast<double>(nx) * px));
  const double g = fmax(static_cast<double>(lo) - t, t - static_cast<double>(hi)) - e;
  return g > 0.0 ? g * g * (1.0 - kSlabMargin) : 0.0;
}

__global__ void __launch_bounds__(kAabbThreads) aabb_query_kernel(const AabbArgs a) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * kAabbThreads + threadIdx.x;
  if (t >= a.np) return;
  const int64_t qi = a.perm ? static_cast<int64_t>(a.perm[t]) : t;
  const double px = a.P[3 * qi], py = a.P[3 * qi + 1], pz = a.P[3 * qi + 2];
  double best = 1.0e300;
  int64_t best_face = -1;
  double bx = 0.0, by = 0.0, bz = 0.0;
  // Slab margin for this point; no slab skips at all for huge or non-finite input.
  double margin = kSlabMargin * (a.scale + fabs(px) + fabs(py) + fabs(pz));
  if (!(margin < 1e100)) margin = INFINITY;
  int stack_node[kAabbStack];
  double stack_d2[kAabbStack];
  int sp = 0;
  if (a.nnodes > 0) {
    stack_node[0] = 0;
    stack_d2[0] = box_distance2(px, py, pz, a.root[0], a.root[1], a.root[2], a.root[3],
                                a.root[4], a.root[5]);
    sp = 1;
  }
  while (sp > 0) {
    --sp;
    if (stack_d2[sp] > best) continue;
    const AabbNodeRec* nd = a.nodes + stack_node[sp];
    const int4 meta = __ldg(reinterpret_cast<const int4*>(nd));
    if (meta.w > 0) {
      const AabbTriRec* tr = a.tris + meta.z;
      for (int k = 0; k < meta.w; ++k, ++tr) {
        const double2 w0 = ldg2(tr->a), w1 = ldg2(tr->a + 2), w2 = ldg2(tr->b + 1);
        const double2 w3 = ldg2(tr->c), w4 = ldg2(tr->c + 2);
        const ClosestHit h = closest_on_triangle(px, py, pz, w0.x, w0.y, w1.x, w1.y, w2.x, w2.y,
                                                 w3.x, w3.y, w4.x);
        if (h.d2 < best) {
          best = h.d2;
          best_face = __double_as_longlong(w4.y);
          bx = h.x;
          by = h.y;
          bz = h.z;
        }
      }
    } else {
      const double2 l0 = ldg2(nd->lbox), l1 = ldg2(nd->lbox + 2), l2 = ldg2(nd->lbox + 4);
      const double2 r0 = ldg2(nd->rbox), r1 = ldg2(nd->rbox + 2), r2 = ldg2(nd->rbox + 4);
      const float4 s0 = __ldg(reinterpret_cast<const float4*>(&nd->lslab));
      const float4 s1 = __ldg(reinterpret_cast<const float4*>(&nd->lslab) + 1);
      const float2 s2 = __ldg(reinterpret_cast<const float2*>(&nd->rslab.lo));
      const double dl = box_distance2(px, py, pz, l0.x, l0.y, l1.x, l1.y, l2.x, l2.y);
      const double dr = box_distance2(px, py, pz, r0.x, r0.y, r1.x, r1.y, r2.x, r2.y);
      const double kl = fmax(dl, slab_bound2(px, py, pz, s0.x, s0.y, s0.z, s0.w, s1.x, margin));
      const double kr = fmax(dr, slab_bound2(px, py, pz, s1.y, s1.z, s1.w, s2.x, s2.y, margin));
      // Farther child first, so the nearer one is popped next (capi.mojo:571-586).
      const bool left_near = dl < dr;
      const int first = left_near ? meta.y : meta.x, second = left_near ? meta.x : meta.y;
      const double dfirst = left_near ? kr : kl, dsecond = left_near ? kl : kr;
      if (sp + 2 > kAabbStack) {  // cannot happen for a validated tree
        atomicOr(a.err, kErrBadLaunch);
        best_face = -2;
        break;
      }
      if (dfirst <= best) {
        stack_node[sp] = first;
        stack_d2[sp] = dfirst;
        ++sp;
      }
      if (dsecond <= best) {
        stack_node[sp] = second;
        stack_d2[sp] = dsecond;
        ++sp;
      }
    }
  }
  a.sqrd[qi] = best;
  a.index[qi] = best_face;
  a.closest[3 * qi] = bx;
  a.closest[3 * qi + 1] = by;
  a.closest[3 * qi + 2] = bz;
}

__global__ void signed_from_winding_kernel(const double* __restrict__ w, double* __restrict__ s,
                                           int64_t n) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double d = __dsqrt_rn(s[i]);
  s[i] = fabs(w[i]) > 0.5 ? -d : d;
}

}  // namespace

cudaError_t aabb_query(const AabbDeviceTree& t, const double* P, int64_t np, const uint32_t* perm,
                       double* sqrd, int64_t* index, double* closest, int* err,
                       cudaStream_t stream) {
  if (np <= 0) return cudaSuccess;
  if (t.depth + 1 > kAabbStack) return cudaErrorInvalidValue;
  AabbArgs a{t.nodes, t.tris, P, perm, sqrd, index, closest, err, np, t.nnodes, {}, t.scale};
  for (int k = 0; k < 6; ++k) a.root[k] = t.root[k];
  const int64_t blocks = (np + kAabbThreads - 1) / kAabbThreads;
  if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  aabb_query_kernel<<<static_cast<unsigned>(blocks), kAabbThreads, 0, stream>>>(a);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError();
}

cudaError_t signed_from_winding(const double* w, double* s, int64_t n, cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  const int64_t blocks = (n + 255) / 256;
  if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  signed_from_winding_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(w, s, n);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError();
}

}  // namespace wn
