// Fast winding number on sm_100a: one thread per query walks the moment tree
// (wn_fwn.h) depth first; a node far enough away (|q - p| > beta r) adds its
// second-order expansion, a nearer leaf adds its faces' exact solid angles.
// The work per query is O(log nf) nodes plus the faces of the few leaves
// around it, instead of all nf faces; the tree (64-byte nodes, 192-byte
// moments, 80-byte faces: 58 MB at 327,680 faces) stays in L2. Like the
// closest-point traversal the walk is a chain of dependent reads, so queries
// are taken in Morton order to keep a warp's walks alike.
#include <cuda_runtime.h>

#include "wn_common.cuh"
#include "wn_fwn.cuh"
#include "wn_fwn.h"
#include "wn_internal.h"

namespace wn {
namespace {

constexpr int kFwnThreads = 128;
constexpr double kPiD = 3.14159265358979323846264338327950288;

struct FwnArgs {
  const FwnNode* __restrict__ nodes;
  const FwnMoments* __restrict__ moments;
  const AabbTriRec* __restrict__ tris;
  const double* __restrict__ q;
  const uint32_t* __restrict__ perm;
  double* __restrict__ w;
  int* err;
  int64_t nq, nnodes;
  double beta;
};

__device__ __forceinline__ double2 ld2(const double* p) {
  return __ldg(reinterpret_cast<const double2*>(p));
}

__global__ void __launch_bounds__(kFwnThreads) fwn_kernel(const FwnArgs a) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * kFwnThreads + threadIdx.x;
  if (t >= a.nq) return;
  const int64_t qi = a.perm ? static_cast<int64_t>(a.perm[t]) : t;
  const double qx = a.q[3 * qi], qy = a.q[3 * qi + 1], qz = a.q[3 * qi + 2];
  double far = 0.0, angle = 0.0;
  int32_t stack[kAabbStack];
  int sp = 0;
  if (a.nnodes > 0) stack[sp++] = 0;
  while (sp > 0) {
    const int32_t i = stack[--sp];
    const FwnNode* n = a.nodes + i;
    const double2 p01 = ld2(n->p), p2r = ld2(n->p + 2);
    const double y0 = p01.x - qx, y1 = p01.y - qy, y2 = p2r.x - qz;
    if (fwn_is_far(y0 * y0 + y1 * y1 + y2 * y2, a.beta, p2r.y)) {
      FwnMoments m;
      const double* src = reinterpret_cast<const double*>(a.moments + i);
      double* dst = reinterpret_cast<double*>(&m);
#pragma unroll
      for (int k = 0; k < 12; ++k) {
        const double2 v = ld2(src + 2 * k);
        dst[2 * k] = v.x;
        dst[2 * k + 1] = v.y;
      }
      far += fwn_far_eval(m, y0, y1, y2);
      continue;
    }
    const int4 meta = __ldg(reinterpret_cast<const int4*>(&n->left));
    if (meta.w > 0) {
      for (int32_t k = meta.z; k < meta.z + meta.w; ++k) {
        const AabbTriRec* tr = a.tris + k;
        AabbTriRec rec;
        const double2 w0 = ld2(tr->a), w1 = ld2(tr->a + 2), w2 = ld2(tr->b + 1);
        const double2 w3 = ld2(tr->c), w4 = ld2(tr->c + 2);
        rec.a[0] = w0.x; rec.a[1] = w0.y; rec.a[2] = w1.x;
        rec.b[0] = w1.y; rec.b[1] = w2.x; rec.b[2] = w2.y;
        rec.c[0] = w3.x; rec.c[1] = w3.y; rec.c[2] = w4.x;
        angle += fwn_face_angle(qx, qy, qz, rec);
      }
    } else {
      if (sp + 2 > kAabbStack) {  // cannot happen for a tree of depth < kAabbStack
        atomicOr(a.err, kErrBadLaunch);
        break;
      }
      stack[sp++] = meta.y;  // right, then left: the left child is walked first
      stack[sp++] = meta.x;
    }
  }
  a.w[qi] = far / (4.0 * kPiD) + angle / (2.0 * kPiD);
}

}  // namespace

cudaError_t fwn_eval_device(const FwnDeviceTree& t, const double* q, int64_t nq,
                            const uint32_t* perm, double beta, double* w, int* err,
                            cudaStream_t stream) {
  if (nq <= 0) return cudaSuccess;
  if (t.depth + 1 > kAabbStack) return cudaErrorInvalidValue;
  const int64_t blocks = (nq + kFwnThreads - 1) / kFwnThreads;
  if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  const FwnArgs a{t.nodes, t.moments, t.tris, q, perm, w, err, nq, t.nnodes, beta};
  fwn_kernel<<<static_cast<unsigned>(blocks), kFwnThreads, 0, stream>>>(a);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError();
}

}  // namespace wn
