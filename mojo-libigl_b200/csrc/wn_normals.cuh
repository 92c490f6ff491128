// Per-vertex normals (the reference's src/capi.mojo:146-202), shared by the
// host path (`mli_vertex_normals`) and the CUDA gather kernel.
//
// Arithmetic of the reference, each operation rounded on its own (the __d*_rn
// intrinsics on the device; -ffp-contract=off on the host): n = (B - A) x
// (C - A) with its component formulas, |n| = sqrt((nx*nx + ny*ny) + nz*nz),
// faces with |n| <= 1e-30 contribute nothing, u = n / |n|; the weight of a
// corner is 1 (uniform), |n| (area) or acos(clamp(e1.e2 / (|e1| |e2|))) (angle);
// a vertex's sum takes u * weight in face order, corners in order; then the sum
// is divided by its length when that exceeds 1e-30. Uniform and area weights
// are therefore bit-identical to the reference's loop; the angle weight goes
// through the platform's acos (CUDA's or the C library's).
#pragma once

#include <cmath>
#include <cstdint>

#include "wn_aabb.cuh"

namespace wn {

enum NormalWeighting : int { kNormalsUniform = 0, kNormalsArea = 1, kNormalsAngle = 2 };

#if defined(__CUDA_ARCH__)
WN_HD double dacos(double x) { return acos(x); }
#else
WN_HD double dacos(double x) { return std::acos(x); }
#endif

// Unit normal u and |n| of face (A, B, C); false when the reference skips the
// face (|n| <= 1e-30).
WN_HD bool face_unit_normal(const double* A, const double* B, const double* C, double* u,
                            double* norm_out) {
  const double abx = dsub(B[0], A[0]), aby = dsub(B[1], A[1]), abz = dsub(B[2], A[2]);
  const double acx = dsub(C[0], A[0]), acy = dsub(C[1], A[1]), acz = dsub(C[2], A[2]);
  const double nx = dsub(dmul(aby, acz), dmul(abz, acy));
  const double ny = dsub(dmul(abz, acx), dmul(abx, acz));
  const double nz = dsub(dmul(abx, acy), dmul(aby, acx));
  const double norm = dsqrt(dot3(nx, ny, nz, nx, ny, nz));
  if (norm <= 1.0e-30) return false;
  u[0] = ddiv(nx, norm);
  u[1] = ddiv(ny, norm);
  u[2] = ddiv(nz, norm);
  *norm_out = norm;
  return true;
}

// Interior angle at corner `corner` of the face whose corners are P[0..2].
WN_HD double corner_angle(const double* const* P, int corner) {
  const double* vi = P[corner];
  const double* vj = P[(corner + 1) % 3];
  const double* vk = P[(corner + 2) % 3];
  const double e1x = dsub(vj[0], vi[0]), e1y = dsub(vj[1], vi[1]), e1z = dsub(vj[2], vi[2]);
  const double e2x = dsub(vk[0], vi[0]), e2y = dsub(vk[1], vi[1]), e2z = dsub(vk[2], vi[2]);
  const double l1 = dsqrt(dot3(e1x, e1y, e1z, e1x, e1y, e1z));
  const double l2 = dsqrt(dot3(e2x, e2y, e2z, e2x, e2y, e2z));
  double cosine = ddiv(dot3(e1x, e1y, e1z, e2x, e2y, e2z), dmul(l1, l2));
  cosine = dmax(-1.0, dmin(1.0, cosine));
  return dacos(cosine);
}

// Weight of a corner: 1 (uniform), |n| (area) or its angle.
WN_HD double corner_weight(const double* const* P, int corner, int mode, double norm) {
  if (mode == kNormalsAngle) return corner_angle(P, corner);
  return mode == kNormalsArea ? norm : 1.0;
}

// Final division of a vertex sum by its length (when > 1e-30).
WN_HD void normal_finish(double* acc) {
  const double norm = dsqrt(dot3(acc[0], acc[1], acc[2], acc[0], acc[1], acc[2]));
  if (norm > 1.0e-30) {
    acc[0] = ddiv(acc[0], norm);
    acc[1] = ddiv(acc[1], norm);
    acc[2] = ddiv(acc[2], norm);
  }
}

}  // namespace wn
