// Host side of the fast winding number: the tree with per-node moments
// (wn_fwn.h) and the host evaluator (device="cpu"). Built with
// -ffp-contract=off like the other host files.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <new>
#include <thread>
#include <vector>

#include "wn_aabb.h"
#include "wn_fwn.cuh"
#include "wn_fwn.h"

namespace wn {
namespace {

// Moments of the faces in records [lo, hi) about their area-weighted centre.
void node_moments(const AabbTriRec* tris, int64_t lo, int64_t hi, FwnNode& node,
                  FwnMoments& out) {
  double area = 0.0, pa[3] = {0.0, 0.0, 0.0}, pc[3] = {0.0, 0.0, 0.0};
  for (int64_t k = lo; k < hi; ++k) {
    const AabbTriRec& t = tris[k];
    const double u[3] = {t.b[0] - t.a[0], t.b[1] - t.a[1], t.b[2] - t.a[2]};
    const double v[3] = {t.c[0] - t.a[0], t.c[1] - t.a[1], t.c[2] - t.a[2]};
    const double n[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2],
                         u[0] * v[1] - u[1] * v[0]};
    const double a = 0.5 * std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    for (int j = 0; j < 3; ++j) {
      const double c = (t.a[j] + t.b[j] + t.c[j]) / 3.0;
      pa[j] += a * c;
      pc[j] += c;
    }
    area += a;
  }
  double p[3];
  for (int j = 0; j < 3; ++j)
    p[j] = area > 0.0 ? pa[j] / area : pc[j] / static_cast<double>(hi - lo);
  double r2 = 0.0, T0[3] = {0, 0, 0}, T1[3][3] = {}, T2[3][3][3] = {};
  for (int64_t k = lo; k < hi; ++k) {
    const AabbTriRec& t = tris[k];
    const double* vtx[3] = {t.a, t.b, t.c};
    const double u[3] = {t.b[0] - t.a[0], t.b[1] - t.a[1], t.b[2] - t.a[2]};
    const double v[3] = {t.c[0] - t.a[0], t.c[1] - t.a[1], t.c[2] - t.a[2]};
    const double an[3] = {0.5 * (u[1] * v[2] - u[2] * v[1]), 0.5 * (u[2] * v[0] - u[0] * v[2]),
                          0.5 * (u[0] * v[1] - u[1] * v[0])};
    double c[3], d[3];
    for (int j = 0; j < 3; ++j) {
      c[j] = (t.a[j] + t.b[j] + t.c[j]) / 3.0;
      d[j] = c[j] - p[j];
    }
    double cov[3][3] = {};
    for (int s = 0; s < 3; ++s) {
      double e[3];
      for (int j = 0; j < 3; ++j) e[j] = vtx[s][j] - c[j];
      for (int j = 0; j < 3; ++j)
        for (int kk = 0; kk < 3; ++kk) cov[j][kk] += e[j] * e[kk] / 12.0;
      double g2 = 0.0;
      for (int j = 0; j < 3; ++j) g2 += (vtx[s][j] - p[j]) * (vtx[s][j] - p[j]);
      r2 = std::max(r2, g2);
    }
    for (int i = 0; i < 3; ++i) {
      T0[i] += an[i];
      for (int j = 0; j < 3; ++j) {
        T1[j][i] += d[j] * an[i];
        for (int kk = 0; kk < 3; ++kk) T2[j][kk][i] += 0.5 * an[i] * (d[j] * d[kk] + cov[j][kk]);
      }
    }
  }
  for (int j = 0; j < 3; ++j) node.p[j] = p[j];
  node.r = std::sqrt(r2);
  for (int i = 0; i < 3; ++i) out.t0[i] = T0[i];
  out.tr = T1[0][0] + T1[1][1] + T1[2][2];
  out.q[0] = -3.0 * T1[0][0];
  out.q[1] = -3.0 * T1[1][1];
  out.q[2] = -3.0 * T1[2][2];
  out.q[3] = -3.0 * (T1[0][1] + T1[1][0]);
  out.q[4] = -3.0 * (T1[0][2] + T1[2][0]);
  out.q[5] = -3.0 * (T1[1][2] + T1[2][1]);
  for (int i = 0; i < 3; ++i) {
    double u = 0.0, v = 0.0;
    for (int j = 0; j < 3; ++j) {
      u += T2[j][i][j];  // u_i = sum_j T2[j][i][j]
      v += T2[j][j][i];  // v_i = sum_j T2[j][j][i]
    }
    out.l[i] = -3.0 * (2.0 * u + v);
  }
  // Cubic form sum T2[j][k][i] y_i y_j y_k, one coefficient per monomial.
  double cub[10] = {};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int kk = 0; kk < 3; ++kk) {
        const int n0 = (i == 0) + (j == 0) + (kk == 0), n1 = (i == 1) + (j == 1) + (kk == 1);
        const int n2 = 3 - n0 - n1;
        int slot;
        if (n0 == 3) slot = 0;
        else if (n1 == 3) slot = 1;
        else if (n2 == 3) slot = 2;
        else if (n0 == 2) slot = n1 == 1 ? 3 : 4;
        else if (n1 == 2) slot = n0 == 1 ? 5 : 7;
        else if (n2 == 2) slot = n0 == 1 ? 6 : 8;
        else slot = 9;
        cub[slot] += T2[j][kk][i];
      }
  for (int s = 0; s < 10; ++s) out.c[s] = 15.0 * cub[s];
  out.pad = 0.0;
}

}  // namespace

int fwn_build(const double* V, int64_t nv, const int64_t* F, int64_t nf, int threads,
              FwnHostTree* out, const char** why) {
  *out = FwnHostTree{};
  if (nv < 0 || nf < 0) {
    *why = "negative size";
    return -1;
  }
  if (nf == 0) return 0;
  if (nf > 0x7fffffffLL) {
    *why = "more than 2^31-1 faces";
    return -1;
  }
  const int64_t nn = aabb_node_count(nf, kFwnLeafFaces);
  std::vector<double> boxes(6 * nn);
  std::vector<int64_t> nodes(4 * nn), order(nf);
  const int64_t stack = aabb_build(V, nv, F, nf, kFwnLeafFaces, boxes.data(), nodes.data(),
                                   order.data(), threads, why);
  if (stack < 0) return -1;
  if (stack > kAabbStack) {
    *why = "tree deeper than the traversal stack";
    return -1;
  }
  out->nodes = new (std::nothrow) FwnNode[nn];
  out->moments = new (std::nothrow) FwnMoments[nn];
  out->tris = new (std::nothrow) AabbTriRec[nf];
  if (!out->nodes || !out->moments || !out->tris) {
    fwn_free(out);
    *why = "host allocation failed";
    return -1;
  }
  out->nnodes = nn;
  out->nf = nf;
  out->depth = static_cast<int>(stack - 1);
  for (int64_t k = 0; k < nf; ++k) {
    AabbTriRec& r = out->tris[k];
    const int64_t f = order[k];
    for (int j = 0; j < 3; ++j) {
      r.a[j] = V[3 * F[3 * f] + j];
      r.b[j] = V[3 * F[3 * f + 1] + j];
      r.c[j] = V[3 * F[3 * f + 2] + j];
    }
    r.face = f;
  }
  // Face-record range of every node (contiguous: preorder, leaves in order).
  std::vector<int64_t> first(nn), last(nn);
  for (int64_t i = nn - 1; i >= 0; --i) {
    const int64_t* nd = &nodes[4 * i];
    FwnNode& n = out->nodes[i];
    if (nd[3] > 0) {
      first[i] = nd[2];
      last[i] = nd[2] + nd[3];
      n.left = n.right = -1;
      n.start = static_cast<int32_t>(nd[2]);
      n.count = static_cast<int32_t>(nd[3]);
    } else {
      first[i] = first[nd[0]];
      last[i] = last[nd[1]];
      n.left = static_cast<int32_t>(nd[0]);
      n.right = static_cast<int32_t>(nd[1]);
      n.start = 0;
      n.count = 0;
    }
    n.pad[0] = n.pad[1] = 0.0;
  }
  if (threads <= 0) threads = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
  auto work = [&](int64_t begin, int64_t step) {
    for (int64_t i = begin; i < nn; i += step)
      node_moments(out->tris, first[i], last[i], out->nodes[i], out->moments[i]);
  };
  if (threads <= 1 || nn < 4096) {
    work(0, 1);
  } else {
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(work, t, threads);
    for (auto& th : pool) th.join();
  }
  return 0;
}

void fwn_free(FwnHostTree* t) {
  delete[] t->nodes;
  delete[] t->moments;
  delete[] t->tris;
  *t = FwnHostTree{};
}

namespace {

// One depth-first walk of query q (left child first): the far terms summed in
// walk order into *far, and the leaf faces either multiplied into *acc (the
// argument-of-product sum of wn_pair.cuh) or, when acc is null, their half
// solid angles summed into *angle.
void fwn_walk(const FwnHostTree& t, double qx, double qy, double qz, double beta, double* far,
              ArgAcc* acc, double* angle) {
  int32_t stack[kAabbStack];
  int sp = 0;
  if (t.nnodes > 0) stack[sp++] = 0;
  while (sp > 0) {
    const FwnNode& n = t.nodes[stack[--sp]];
    const double y0 = n.p[0] - qx, y1 = n.p[1] - qy, y2 = n.p[2] - qz;
    if (fwn_is_far(fwn_dist2(y0, y1, y2), beta, n.r)) {
      if (far) *far += fwn_far_eval(t.moments[&n - t.nodes], y0, y1, y2);
    } else if (n.count > 0) {
      for (int32_t k = n.start; k < n.start + n.count; ++k) {
        const AabbTriRec& r = t.tris[k];
        if (acc) {
          double det, denom;
          pair_terms_exact(qx, qy, qz, r.a[0], r.a[1], r.a[2], r.b[0], r.b[1], r.b[2], r.c[0],
                           r.c[1], r.c[2], det, denom);
          argacc_push(*acc, denom, det);
        } else {
          *angle += fwn_face_angle(qx, qy, qz, r);
        }
      }
    } else {
      stack[sp++] = n.right;  // left child first
      stack[sp++] = n.left;
    }
  }
}

}  // namespace

void fwn_eval_host(const FwnHostTree& t, const double* q, int64_t q0, int64_t q1, double beta,
                   double* w) {
  for (int64_t qi = q0; qi < q1; ++qi) {
    const double qx = q[3 * qi], qy = q[3 * qi + 1], qz = q[3 * qi + 2];
    double far = 0.0, angle = 0.0;
    ArgAcc acc;
    argacc_init(acc);
    fwn_walk(t, qx, qy, qz, beta, &far, &acc, nullptr);
    if (!acc.bad)
      angle = std::atan2(acc.zi, acc.zr) + static_cast<double>(acc.k) * kTwoPi;
    else  // the product degenerated: the per-face sum of the same faces
      fwn_walk(t, qx, qy, qz, beta, nullptr, nullptr, &angle);
    w[qi] = far / (4.0 * kPi) + angle / (2.0 * kPi);
  }
}

}  // namespace wn
