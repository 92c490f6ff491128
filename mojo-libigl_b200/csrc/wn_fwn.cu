// Fast winding number on sm_100a: one thread per query walks the moment tree
// (wn_fwn.h) depth first; a node far enough away (|q - p| > beta r) adds its
// second-order expansion, a nearer leaf adds its faces' exact solid angles.
// The work per query is O(log nf) nodes plus the faces of the few leaves
// around it, instead of all nf faces; the tree (64-byte nodes, 192-byte
// moments, 80-byte faces: 58 MB at 327,680 faces) stays in L2. Queries are
// taken in Morton order to keep a warp's walks alike.
//
// The walk has three kinds of step: opening an internal node (cheap), a far
// node (~70 FP64 operations on 23 coefficients) and a leaf (up to 8 faces,
// each the exact pair terms and an atan2). Evaluated where they are met, a
// warp's lanes take different kinds at nearly every step and each expensive
// step runs with a few lanes on. So the walk only classifies: far nodes and
// leaf faces go to per-thread lists in shared memory (a column per thread,
// conflict free), and when any lane's list is full the whole warp evaluates
// its lists together. The far terms are added in the walk's order; the faces
// of one flush are multiplied into a running complex product (as in the exact
// kernels) whose argument is taken once, so a flush costs one atan2 instead of
// one per face. The results are deterministic and agree with the host
// evaluator's per-face sums to rounding (~1e-15).
#include <cuda_runtime.h>

#include "wn_common.cuh"
#include "wn_fwn.cuh"
#include "wn_fwn.h"
#include "wn_internal.h"

namespace wn {
namespace {

constexpr int kFwnThreads = 128;
constexpr int kFarSlots = 16;   // deferred far nodes per thread
constexpr int kFaceSlots = 48;  // deferred leaf faces per thread (>= kFwnLeafFaces)
constexpr double kPiD = 3.14159265358979323846264338327950288;
static_assert(kFaceSlots >= kFwnLeafFaces, "a leaf must fit an empty face list");

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

// Per-thread lists, one column per thread: entry k of thread t at [k][t].
struct FwnLists {
  int32_t far[kFarSlots][kFwnThreads];
  int32_t face[kFaceSlots][kFwnThreads];
};

__device__ __forceinline__ double2 ld2(const double* p) {
  return __ldg(reinterpret_cast<const double2*>(p));
}

// 4 pi x the far-field term of node i at q.
__device__ __forceinline__ double far_term(const FwnArgs& a, int32_t i, double qx, double qy,
                                           double qz) {
  const FwnNode* n = a.nodes + i;
  const double2 p01 = ld2(n->p), p2r = ld2(n->p + 2);
  FwnMoments m;
  const double* src = reinterpret_cast<const double*>(a.moments + i);
  double* dst = reinterpret_cast<double*>(&m);
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    const double2 v = ld2(src + 2 * k);
    dst[2 * k] = v.x;
    dst[2 * k + 1] = v.y;
  }
  return fwn_far_eval(m, p01.x - qx, p01.y - qy, p2r.x - qz);
}

// Face record k, read as five 16-byte words.
__device__ __forceinline__ AabbTriRec face_rec(const FwnArgs& a, int32_t k) {
  const AabbTriRec* tr = a.tris + k;
  AabbTriRec rec;
  const double2 w0 = ld2(tr->a), w1 = ld2(tr->a + 2), w2 = ld2(tr->b + 1);
  const double2 w3 = ld2(tr->c), w4 = ld2(tr->c + 2);
  rec.a[0] = w0.x; rec.a[1] = w0.y; rec.a[2] = w1.x;
  rec.b[0] = w1.y; rec.b[1] = w2.x; rec.b[2] = w2.y;
  rec.c[0] = w3.x; rec.c[1] = w3.y; rec.c[2] = w4.x;
  return rec;
}

// Sum of the half solid angles of the thread's n listed faces at q: the
// faces' (denom, det) pairs are multiplied into one running complex product
// (the exact kernels' argument-of-product sum, wn_pair.cuh) and its argument
// taken once, instead of one atan2 per face; if the product degenerates, the
// per-face atan2 sum of the same faces.
__device__ __forceinline__ double face_list_angle(const FwnArgs& a, const FwnLists& lists,
                                                  int tid, int n, double qx, double qy,
                                                  double qz) {
  ArgAcc acc;
  argacc_init(acc);
  for (int k = 0; k < n; ++k) {
    const AabbTriRec rec = face_rec(a, lists.face[k][tid]);
    double det, denom;
    pair_terms_exact(qx, qy, qz, rec.a[0], rec.a[1], rec.a[2], rec.b[0], rec.b[1], rec.b[2],
                     rec.c[0], rec.c[1], rec.c[2], det, denom);
    argacc_push(acc, denom, det);
  }
  if (!acc.bad) return atan2(acc.zi, acc.zr) + static_cast<double>(acc.k) * kTwoPi;
  double sum = 0.0;
  for (int k = 0; k < n; ++k) sum += fwn_face_angle(qx, qy, qz, face_rec(a, lists.face[k][tid]));
  return sum;
}

__global__ void __launch_bounds__(kFwnThreads) fwn_kernel(const FwnArgs a) {
  __shared__ FwnLists lists;
  const int tid = threadIdx.x;
  const int64_t t = static_cast<int64_t>(blockIdx.x) * kFwnThreads + tid;
  // Threads past nq walk nothing but stay for the warp votes.
  const bool live = t < a.nq;
  int64_t qi = 0;
  double qx = 0.0, qy = 0.0, qz = 0.0;
  if (live) {
    qi = a.perm ? static_cast<int64_t>(a.perm[t]) : t;
    qx = a.q[3 * qi];
    qy = a.q[3 * qi + 1];
    qz = a.q[3 * qi + 2];
  }
  double far = 0.0, angle = 0.0;
  // `node` is the next node to classify (-1: pop one); opening a node goes on
  // with its left child in a register and stacks only the right one.
  int32_t stack[kAabbStack];
  int sp = 0;
  int32_t node = live && a.nnodes > 0 ? 0 : -1;
  int nfar = 0, nface = 0;
  bool bad = false;
  for (;;) {
    if (node < 0 && sp > 0) node = stack[--sp];
    if (node >= 0) {
      const FwnNode* n = a.nodes + node;
      const double2 p01 = ld2(n->p), p2r = ld2(n->p + 2);
      const int4 meta = __ldg(reinterpret_cast<const int4*>(&n->left));
      const double y0 = p01.x - qx, y1 = p01.y - qy, y2 = p2r.x - qz;
      if (fwn_is_far(fwn_dist2(y0, y1, y2), a.beta, p2r.y)) {
        lists.far[nfar++][tid] = node;
        node = -1;
      } else if (meta.w > 0) {
        if (meta.w > kFwnLeafFaces) {  // not a tree of fwn_build
          bad = true;
          sp = 0;
        } else {
          for (int k = 0; k < meta.w; ++k) lists.face[nface++][tid] = meta.z + k;
        }
        node = -1;
      } else if (sp + 1 > kAabbStack) {  // cannot happen for a tree of depth < kAabbStack
        bad = true;
        sp = 0;
        node = -1;
      } else {
        stack[sp++] = meta.y;  // the right child waits; the left one is walked first
        node = meta.x;
      }
    }
    const unsigned flags = (nfar == kFarSlots ? 1u : 0u) |
                           (nface > kFaceSlots - kFwnLeafFaces ? 2u : 0u) |
                           (sp > 0 || node >= 0 ? 4u : 0u);
    const unsigned any = __reduce_or_sync(0xffffffffu, flags);
    if (any & 1u) {
      for (int k = 0; k < nfar; ++k) far += far_term(a, lists.far[k][tid], qx, qy, qz);
      nfar = 0;
    }
    if (any & 2u) {
      angle += face_list_angle(a, lists, tid, nface, qx, qy, qz);
      nface = 0;
    }
    if (!(any & 4u)) break;
  }
  for (int k = 0; k < nfar; ++k) far += far_term(a, lists.far[k][tid], qx, qy, qz);
  angle += face_list_angle(a, lists, tid, nface, qx, qy, qz);
  if (bad) atomicOr(a.err, kErrBadLaunch);
  if (live) a.w[qi] = far / (4.0 * kPiD) + angle / (2.0 * kPiD);
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
