// Per-node and per-face terms of the fast winding number, shared by the CUDA
// kernel and the host evaluator (wn_fwn.h has the expansion).
#pragma once

#include <cmath>

#include "wn_fwn.h"
#include "wn_pair.cuh"

namespace wn {

// 4 pi x the far-field contribution of a node, y = p - q.
WN_HD double fwn_far_eval(const FwnMoments& m, double y0, double y1, double y2) {
  const double s2 = y0 * y0 + y1 * y1 + y2 * y2;
  const double i1 = 1.0 / sqrt(s2);
  const double i2 = i1 * i1;
  const double i3 = i1 * i2, i5 = i3 * i2, i7 = i5 * i2;
  const double y00 = y0 * y0, y11 = y1 * y1, y22 = y2 * y2;
  const double y01 = y0 * y1, y02 = y0 * y2, y12 = y1 * y2;
  const double a = m.t0[0] * y0 + m.t0[1] * y1 + m.t0[2] * y2 + m.tr;
  const double b = m.q[0] * y00 + m.q[1] * y11 + m.q[2] * y22 + m.q[3] * y01 + m.q[4] * y02 +
                   m.q[5] * y12 + m.l[0] * y0 + m.l[1] * y1 + m.l[2] * y2;
  const double c = m.c[0] * y00 * y0 + m.c[1] * y11 * y1 + m.c[2] * y22 * y2 +
                   m.c[3] * y00 * y1 + m.c[4] * y00 * y2 + m.c[5] * y0 * y11 +
                   m.c[6] * y0 * y22 + m.c[7] * y11 * y2 + m.c[8] * y1 * y22 + m.c[9] * y01 * y2;
  return a * i3 + b * i5 + c * i7;
}

// |y|^2 with every product and sum rounded separately (no contraction into
// FMAs), so the GPU and the host classify every node the same way, also for a
// query exactly on a node's sphere (a vertex at its radius).
WN_HD double fwn_dist2(double y0, double y1, double y2) {
  return dadd(dadd(dmul(y0, y0), dmul(y1, y1)), dmul(y2, y2));
}

// A node is replaced by its expansion when |q - p|^2 > (beta r)^2.
WN_HD bool fwn_is_far(double d2, double beta, double r) {
  const double br = beta * r;
  return d2 > br * br;
}

// atan2 of one face's exact pair terms (the face's solid angle / 2).
WN_HD double fwn_face_angle(double qx, double qy, double qz, const AabbTriRec& t) {
  double det, denom;
  pair_terms_exact(qx, qy, qz, t.a[0], t.a[1], t.a[2], t.b[0], t.b[1], t.b[2], t.c[0], t.c[1],
                   t.c[2], det, denom);
  return atan2(det, denom);
}

}  // namespace wn
