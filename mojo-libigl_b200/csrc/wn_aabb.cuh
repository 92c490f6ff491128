// Closest point on a triangle and point-to-box distance, shared by the CUDA
// traversal kernel and the host (device="cpu") path of libwn_b200.
//
// Same arithmetic as the reference's closest-point query (lee101/mojo-libigl,
// src/capi.mojo:401-502): the Voronoi-region walk of Ericson, "Real-Time
// Collision Detection" (2005) sec. 5.1.5 (vertex A, vertex B, edge AB, vertex C,
// edge AC, edge BC, interior), plus the reference's branch for a degenerate
// triangle (|va + vb + vc| <= 1e-30: the longest edge, clamped to [0, 1]; all
// edges of zero length answer vertex A). Every product, sum, quotient and the
// final squared distance are rounded on their own and in the reference's
// order (the __d*_rn intrinsics on the device; the host file is built with
// -ffp-contract=off), so the squared distance, the closest point and hence
// every comparison of the traversal are bit-identical on both sides.
#pragma once

#include <cmath>
#include <cstdint>

#include "wn_pair.cuh"

namespace wn {

#if defined(__CUDA_ARCH__)
WN_HD double ddiv(double a, double b) { return __ddiv_rn(a, b); }
#else
WN_HD double ddiv(double a, double b) { return a / b; }
#endif

WN_HD double dmax(double a, double b) { return fmax(a, b); }
WN_HD double dmin(double a, double b) { return fmin(a, b); }

// a.b, summed left to right.
WN_HD double dot3(double ax, double ay, double az, double bx, double by, double bz) {
  return dadd(dadd(dmul(ax, bx), dmul(ay, by)), dmul(az, bz));
}

struct ClosestHit {
  double d2, x, y, z;
};

// capi.mojo:401-495.
WN_HD ClosestHit closest_on_triangle(double px, double py, double pz, double ax, double ay,
                                     double az, double bx, double by, double bz, double cx,
                                     double cy, double cz) {
  const double abx = dsub(bx, ax), aby = dsub(by, ay), abz = dsub(bz, az);
  const double acx = dsub(cx, ax), acy = dsub(cy, ay), acz = dsub(cz, az);
  const double apx = dsub(px, ax), apy = dsub(py, ay), apz = dsub(pz, az);
  const double d1 = dot3(abx, aby, abz, apx, apy, apz);
  const double d2 = dot3(acx, acy, acz, apx, apy, apz);
  double qx = ax, qy = ay, qz = az;
  if (!(d1 <= 0.0 && d2 <= 0.0)) {
    const double bpx = dsub(px, bx), bpy = dsub(py, by), bpz = dsub(pz, bz);
    const double d3 = dot3(abx, aby, abz, bpx, bpy, bpz);
    const double d4 = dot3(acx, acy, acz, bpx, bpy, bpz);
    const double vc = dsub(dmul(d1, d4), dmul(d3, d2));
    if (d3 >= 0.0 && d4 <= d3) {
      qx = bx; qy = by; qz = bz;
    } else if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
      const double t = ddiv(d1, dsub(d1, d3));
      qx = dadd(ax, dmul(t, abx)); qy = dadd(ay, dmul(t, aby)); qz = dadd(az, dmul(t, abz));
    } else {
      const double cpx = dsub(px, cx), cpy = dsub(py, cy), cpz = dsub(pz, cz);
      const double d5 = dot3(abx, aby, abz, cpx, cpy, cpz);
      const double d6 = dot3(acx, acy, acz, cpx, cpy, cpz);
      const double vb = dsub(dmul(d5, d2), dmul(d1, d6));
      if (d6 >= 0.0 && d5 <= d6) {
        qx = cx; qy = cy; qz = cz;
      } else if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
        const double t = ddiv(d2, dsub(d2, d6));
        qx = dadd(ax, dmul(t, acx)); qy = dadd(ay, dmul(t, acy)); qz = dadd(az, dmul(t, acz));
      } else {
        const double va = dsub(dmul(d3, d6), dmul(d5, d4));
        const double u43 = dsub(d4, d3), u56 = dsub(d5, d6);
        if (va <= 0.0 && u43 >= 0.0 && u56 >= 0.0) {
          const double t = ddiv(u43, dadd(u43, u56));
          qx = dadd(bx, dmul(t, dsub(cx, bx)));
          qy = dadd(by, dmul(t, dsub(cy, by)));
          qz = dadd(bz, dmul(t, dsub(cz, bz)));
        } else {
          const double denom = dadd(dadd(va, vb), vc);
          if (fabs(denom) <= 1.0e-30) {
            const double bcx = dsub(cx, bx), bcy = dsub(cy, by), bcz = dsub(cz, bz);
            const double lab = dot3(abx, aby, abz, abx, aby, abz);
            const double lbc = dot3(bcx, bcy, bcz, bcx, bcy, bcz);
            const double lca = dot3(acx, acy, acz, acx, acy, acz);
            if (lab >= lbc && lab >= lca && lab > 0.0) {
              const double t = dmax(0.0, dmin(1.0, ddiv(d1, lab)));
              qx = dadd(ax, dmul(t, abx)); qy = dadd(ay, dmul(t, aby)); qz = dadd(az, dmul(t, abz));
            } else if (lbc >= lca && lbc > 0.0) {
              const double t = dmax(0.0, dmin(1.0, ddiv(dot3(bpx, bpy, bpz, bcx, bcy, bcz), lbc)));
              qx = dadd(bx, dmul(t, bcx)); qy = dadd(by, dmul(t, bcy)); qz = dadd(bz, dmul(t, bcz));
            } else if (lca > 0.0) {
              const double t = dmax(0.0, dmin(1.0, ddiv(d2, lca)));
              qx = dadd(ax, dmul(t, acx)); qy = dadd(ay, dmul(t, acy)); qz = dadd(az, dmul(t, acz));
            }
          } else {
            const double inv = ddiv(1.0, denom);
            const double v = dmul(vb, inv), w = dmul(vc, inv);
            qx = dadd(dadd(ax, dmul(abx, v)), dmul(acx, w));
            qy = dadd(dadd(ay, dmul(aby, v)), dmul(acy, w));
            qz = dadd(dadd(az, dmul(abz, v)), dmul(acz, w));
          }
        }
      }
    }
  }
  const double dx = dsub(px, qx), dy = dsub(py, qy), dz = dsub(pz, qz);
  return ClosestHit{dot3(dx, dy, dz, dx, dy, dz), qx, qy, qz};
}

// capi.mojo:498-502 for a box stored as lo xyz, hi xyz.
WN_HD double box_distance2(double px, double py, double pz, double lx, double ly, double lz,
                           double hx, double hy, double hz) {
  const double dx = dmax(dsub(lx, px), dmax(0.0, dsub(px, hx)));
  const double dy = dmax(dsub(ly, py), dmax(0.0, dsub(py, hy)));
  const double dz = dmax(dsub(lz, pz), dmax(0.0, dsub(pz, hz)));
  return dot3(dx, dy, dz, dx, dy, dz);
}

}  // namespace wn
