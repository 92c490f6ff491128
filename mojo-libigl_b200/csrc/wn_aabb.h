// Closest-point queries over the reference's median-split hierarchy: the
// device layout of the tree and the host-side builder (internal interface
// between wn_aabb.cu, wn_aabb_host.cpp and the C ABI in wn_capi.cu).
//
// The tree is the one the reference builds in python/igl/__init__.py:286-319
// (boxes lo/hi, nodes left/right/start/count, faces in leaf order, nodes in
// preorder); the traversal is src/capi.mojo:522-586. On the device each node
// becomes one 160-byte record holding the boxes of BOTH children next to the
// child indices, so an internal node costs one record read for its two box
// tests; the faces of every leaf sit contiguously in leaf order, 80 bytes each
// (corners A, B, C and the face index).
//
// Each child also carries a slab: a unit normal n (the normalised area-weighted
// sum of its faces' normals) and the range [lo, hi] of n.x over every vertex of
// its faces, rounded outward. Every point of those faces lies in the slab, so
// max(lo - n.p, n.p - hi) bounds the distance from p to any of them from below.
// The traversal skips a child when that bound, less a rounding margin, already
// exceeds the best squared distance: none of its faces could be taken (a face
// is taken only when strictly closer than the best so far, and the best only
// decreases), so skipping changes no later decision and the result stays the
// reference's. For curved surfaces it removes most of the leaves whose boxes
// reach toward a point that is far from the surface.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace wn {

struct AabbSlab {
  float n[3];   // unit normal
  float lo, hi;  // range of n.x over the child's vertices, rounded outward (+-inf: no slab)
};

struct __align__(32) AabbNodeRec {
  int32_t left, right, start, count;  // count > 0: a leaf of faces [start, start+count)
  double lbox[6];  // left child's box (lo xyz, hi xyz); unused for a leaf
  double rbox[6];  // right child's box
  AabbSlab lslab, rslab;
  int32_t pad[2];
};
static_assert(sizeof(AabbNodeRec) == 160, "node record is five 32-byte sectors");

struct __align__(16) AabbTriRec {
  double a[3], b[3], c[3];
  int64_t face;
};
static_assert(sizeof(AabbTriRec) == 80, "face record is five 16-byte words");

// A device-resident tree (immutable once built).
struct AabbDeviceTree {
  AabbNodeRec* nodes = nullptr;
  AabbTriRec* tris = nullptr;
  int64_t nnodes = 0, nleaf_faces = 0;
  int depth = 0;       // levels, root = 1
  double root[6] = {};  // root box (the traversal tests it when the root is popped)
  double scale = 0.0;   // largest |coordinate| of the mesh (sets the slab margin)
};

// Deepest tree the kernels accept (traversal stack of kAabbStack entries,
// which a tree of depth D never exceeds when D + 1 <= kAabbStack).
constexpr int kAabbStack = 64;

// Queries below this count are traversed in input order; above it they are
// Morton-ordered first so that a warp's threads walk nearby paths.
constexpr int64_t kAabbSortMin = 1 << 14;

// Closest point of each query (P: np x 3) over the tree. perm (optional):
// thread t handles query perm[t]. Writes sqrd[i], index[i], closest[3i..3i+2]
// for every query i, in input order. Sets kErrBadLaunch in *err if a
// traversal stack would overflow (never for a validated tree).
cudaError_t aabb_query(const AabbDeviceTree& t, const double* P, int64_t np, const uint32_t* perm,
                       double* sqrd, int64_t* index, double* closest, int* err,
                       cudaStream_t stream);

// s[i] <- sqrt(s[i]), negated where |w[i]| > 1/2 (inside a closed, consistently
// oriented surface).
cudaError_t signed_from_winding(const double* w, double* s, int64_t n, cudaStream_t stream);

// ---- host side (wn_aabb_host.cpp) -------------------------------------------
// Nodes of the hierarchy over nf faces with at most `leaf` faces per leaf.
int64_t aabb_node_count(int64_t nf, int64_t leaf);

// Builds the tree of python/igl/__init__.py:286-319 into boxes (nnodes x 6),
// nodes (nnodes x 4) and order (nf); returns the stack size (depth + 1), or a
// negative value for invalid input (message in *why). threads <= 0: all cores.
int64_t aabb_build(const double* V, int64_t nv, const int64_t* F, int64_t nf, int64_t leaf,
                   double* boxes, int64_t* nodes, int64_t* order, int threads, const char** why);

// Validates caller-supplied tree arrays and converts them to the device
// records (host memory, caller-sized: nnodes node records, nf face records),
// slabs included; *scale receives the largest |coordinate| of the mesh.
// Returns the depth (root = 1), or a negative value with the reason in *why.
int64_t aabb_pack(const double* V, int64_t nv, const int64_t* F, int64_t nf, const double* boxes,
                  const int64_t* nodes, const int64_t* order, int64_t nnodes,
                  AabbNodeRec* node_out, AabbTriRec* tri_out, double* scale, const char** why);

// Relative size of the slab margin: a child is skipped only when
// (bound - kSlabMargin * (scale + |px| + |py| + |pz|))^2 * (1 - kSlabMargin)
// exceeds the best squared distance. The margin covers the rounding of n.p,
// of the slab ends and of the reference's own closest-point arithmetic (each
// a few units of 2^-53 of the coordinates), with a factor above 1000 to spare.
constexpr double kSlabMargin = 4e-12;

}  // namespace wn
