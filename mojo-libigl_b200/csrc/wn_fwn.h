// Fast approximate winding numbers (Barill, Dickson, Schmidt, Levin, Jacobson,
// "Fast Winding Numbers for Soups and Clouds", ACM TOG 37(4), 2018): internal
// interface between wn_fwn_host.cpp (moments, host evaluation), wn_fwn.cu (the
// CUDA kernel) and the C ABI.
//
// The faces are organised by the same median-split tree as the closest-point
// path (wn_aabb_build, leaves of at most 8 faces). Every node stores the
// area-weighted centre p of its faces, the radius r of the ball around p that
// holds all their vertices, and the Taylor coefficients of their dipole field
// about p up to second order:
//   T0 = sum_t a_t n_t,  T1[j][i] = sum_t a_t d_j n_i,
//   T2[j][k][i] = 1/2 sum_t a_t n_i (d_j d_k + C_t[j][k]),
// with a_t n_t = (B - A) x (C - A) / 2, d = centroid - p and C_t the second
// moment of the triangle about its centroid, (1/12) sum_v (v - c)(v - c)^T.
// For a point q with y = p - q and s = |y| > beta * r, the node contributes
//   4 pi w = (T0.y + tr T1) / s^3 - 3 (y^T T1 y + (2u + v).y) / s^5
//            + 15 sum T2[j][k][i] y_i y_j y_k / s^7,
// u_k = sum_i T2[i][k][i], v_i = sum_j T2[j][j][i] (the first three terms of
// the expansion of (x - q) / |x - q|^3 about x = p, integrated over the faces).
// Nearer nodes are opened; leaves add their faces' exact solid angles (the
// bit-exact pair terms of the exact path, their angles summed through a running
// complex product as there, the per-face atan2 sum when it degenerates). Each
// query walks the tree depth first, left child first, so its sum has a fixed
// order.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "wn_aabb.h"

namespace wn {

// Most faces in one leaf (the kernel's deferred face lists rely on it).
constexpr int kFwnLeafFaces = 8;

struct __align__(64) FwnNode {
  double p[3];  // area-weighted centre of the node's faces
  double r;     // radius about p holding every vertex of those faces
  int32_t left, right, start, count;  // count > 0: a leaf of face records [start, start+count)
  double pad[2];
};
static_assert(sizeof(FwnNode) == 64, "FwnNode is one 64-byte record");

// Folded expansion of one node (see the file comment):
//   4 pi w = s^-3 (t0.y + tr) + s^-5 (q . [y0^2, y1^2, y2^2, y0 y1, y0 y2, y1 y2] + l.y)
//            + s^-7 (c . [y0^3, y1^3, y2^3, y0^2 y1, y0^2 y2, y0 y1^2, y0 y2^2, y1^2 y2,
//                         y1 y2^2, y0 y1 y2])
struct __align__(64) FwnMoments {
  double t0[3];
  double tr;
  double q[6];   // -3 x the quadratic form of T1 (off-diagonal pairs summed)
  double l[3];   // -3 (2u + v)
  double c[10];  // 15 x the cubic form of T2 (all index orders summed)
  double pad;
};
static_assert(sizeof(FwnMoments) == 192, "FwnMoments is three 64-byte lines");

// Host-side tree with moments (built once, evaluated on the host directly and
// uploaded per device on first use).
struct FwnHostTree {
  int64_t nnodes = 0, nf = 0;
  int depth = 0;
  FwnNode* nodes = nullptr;        // nnodes
  FwnMoments* moments = nullptr;   // nnodes
  AabbTriRec* tris = nullptr;      // nf, leaf order
};

// Builds the tree of (V, F) (median split, leaves of at most 8) with moments.
// Returns 0, or a negative value with *why set. threads <= 0: all cores.
int fwn_build(const double* V, int64_t nv, const int64_t* F, int64_t nf, int threads,
              FwnHostTree* out, const char** why);
void fwn_free(FwnHostTree* t);

// Host evaluation of queries [q0, q1) (q: nq x 3) into w (same indexing).
void fwn_eval_host(const FwnHostTree& t, const double* q, int64_t q0, int64_t q1, double beta,
                   double* w);

// Device copy of a tree.
struct FwnDeviceTree {
  FwnNode* nodes = nullptr;
  FwnMoments* moments = nullptr;
  AabbTriRec* tris = nullptr;
  int64_t nnodes = 0;
  int depth = 0;
};

// One thread per query (perm: optional Morton order, thread t takes query
// perm[t]); writes w for every query. Sets kErrBadLaunch in *err if a
// traversal stack would overflow (never for a tree of depth <= kAabbStack - 1).
cudaError_t fwn_eval_device(const FwnDeviceTree& t, const double* q, int64_t nq,
                            const uint32_t* perm, double beta, double* w, int* err,
                            cudaStream_t stream);

}  // namespace wn
