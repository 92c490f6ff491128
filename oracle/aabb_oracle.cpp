// ORACLE — test infrastructure only. Not part of the product library.
//
// CPU restatement of the reference's closest-point query over its median-split
// bounding-volume hierarchy (lee101/mojo-libigl, src/capi.mojo:401-586,
// exported as `mli_aabb_squared_distance` at capi.mojo:950-959). Linked into
// liboracle_wn.so beside the winding-number oracle; only tests, the smoke check
// and bench.py's CPU-baseline / reference legs may load it.
//
// What is restated, branch for branch:
//   * closest point on a triangle (capi.mojo:401-495): the Voronoi-region walk
//     of Ericson, "Real-Time Collision Detection" (2005), sec. 5.1.5 — vertex A,
//     vertex B, edge AB, vertex C, edge AC, edge BC, interior — with the
//     reference's extra branch for a degenerate triangle (|va+vb+vc| <= 1e-30:
//     project onto the longest edge, clamped; a triangle with all edges of zero
//     length answers vertex A), then the squared distance dx*dx+dy*dy+dz*dz.
//   * the squared distance from a point to a node's box (capi.mojo:498-502):
//     per axis max(lo - p, max(0, p - hi)).
//   * the traversal (capi.mojo:522-586): a stack seeded with the root; a popped
//     node is skipped when out of range or when its box is farther than the best
//     distance so far (strictly); a leaf tests its faces in `order` sequence and
//     takes a face only when strictly closer; an internal node pushes the farther
//     child first so the nearer one is popped next, each child only when its box
//     distance is <= best. Initial best 1e300, face -1, point (0, 0, 0).
//   * Tree arrays as the reference's python/igl/__init__.py:286-319 builds them:
//     boxes (nnodes, 6) = lo xyz, hi xyz; nodes (nnodes, 4) = left, right,
//     start, count (count > 0 marks a leaf); order = faces in leaf order.
//   * Every product and sum is rounded on its own (-ffp-contract=off), the
//     division is IEEE division, and dot products add left to right.
#include <cmath>
#include <cstdint>

namespace {

struct Hit {
  double d2, x, y, z;
};

inline double dot3(double ax, double ay, double az, double bx, double by, double bz) {
  return ax * bx + ay * by + az * bz;
}

inline double clamp01(double t) { return std::fmax(0.0, std::fmin(1.0, t)); }

// capi.mojo:401-495.
Hit closest_point(double px, double py, double pz, double ax, double ay, double az, double bx,
                  double by, double bz, double cx, double cy, double cz) {
  const double abx = bx - ax, aby = by - ay, abz = bz - az;
  const double acx = cx - ax, acy = cy - ay, acz = cz - az;
  const double apx = px - ax, apy = py - ay, apz = pz - az;
  const double d1 = dot3(abx, aby, abz, apx, apy, apz);
  const double d2 = dot3(acx, acy, acz, apx, apy, apz);
  double qx = ax, qy = ay, qz = az;
  bool done = d1 <= 0.0 && d2 <= 0.0;  // region of vertex A
  const double bpx = px - bx, bpy = py - by, bpz = pz - bz;
  double d3 = 0, d4 = 0, d5 = 0, d6 = 0, vc = 0, vb = 0;
  if (!done) {
    d3 = dot3(abx, aby, abz, bpx, bpy, bpz);
    d4 = dot3(acx, acy, acz, bpx, bpy, bpz);
    if (d3 >= 0.0 && d4 <= d3) {  // vertex B
      qx = bx; qy = by; qz = bz;
      done = true;
    }
  }
  if (!done) {
    vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {  // edge AB
      const double t = d1 / (d1 - d3);
      qx = ax + t * abx; qy = ay + t * aby; qz = az + t * abz;
      done = true;
    }
  }
  if (!done) {
    const double cpx = px - cx, cpy = py - cy, cpz = pz - cz;
    d5 = dot3(abx, aby, abz, cpx, cpy, cpz);
    d6 = dot3(acx, acy, acz, cpx, cpy, cpz);
    if (d6 >= 0.0 && d5 <= d6) {  // vertex C
      qx = cx; qy = cy; qz = cz;
      done = true;
    }
  }
  if (!done) {
    vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {  // edge AC
      const double t = d2 / (d2 - d6);
      qx = ax + t * acx; qy = ay + t * acy; qz = az + t * acz;
      done = true;
    }
  }
  if (!done) {
    const double va = d3 * d6 - d5 * d4;
    if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {  // edge BC
      const double t = (d4 - d3) / ((d4 - d3) + (d5 - d6));
      qx = bx + t * (cx - bx); qy = by + t * (cy - by); qz = bz + t * (cz - bz);
    } else {
      const double denom = va + vb + vc;
      if (std::fabs(denom) <= 1.0e-30) {  // degenerate: longest edge, clamped
        const double lab = dot3(abx, aby, abz, abx, aby, abz);
        const double bcx = cx - bx, bcy = cy - by, bcz = cz - bz;
        const double lbc = dot3(bcx, bcy, bcz, bcx, bcy, bcz);
        const double lca = dot3(acx, acy, acz, acx, acy, acz);
        if (lab >= lbc && lab >= lca && lab > 0.0) {
          const double t = clamp01(d1 / lab);
          qx = ax + t * abx; qy = ay + t * aby; qz = az + t * abz;
        } else if (lbc >= lca && lbc > 0.0) {
          const double t = clamp01(dot3(bpx, bpy, bpz, bcx, bcy, bcz) / lbc);
          qx = bx + t * bcx; qy = by + t * bcy; qz = bz + t * bcz;
        } else if (lca > 0.0) {
          const double t = clamp01(d2 / lca);
          qx = ax + t * acx; qy = ay + t * acy; qz = az + t * acz;
        }
      } else {  // interior
        const double inv = 1.0 / denom;
        const double v = vb * inv, w = vc * inv;
        qx = ax + abx * v + acx * w;
        qy = ay + aby * v + acy * w;
        qz = az + abz * v + acz * w;
      }
    }
  }
  const double dx = px - qx, dy = py - qy, dz = pz - qz;
  return Hit{dx * dx + dy * dy + dz * dz, qx, qy, qz};
}

// capi.mojo:498-502.
inline double box_d2(double px, double py, double pz, const double* b) {
  const double dx = std::fmax(b[0] - px, std::fmax(0.0, px - b[3]));
  const double dy = std::fmax(b[1] - py, std::fmax(0.0, py - b[4]));
  const double dz = std::fmax(b[2] - pz, std::fmax(0.0, pz - b[5]));
  return dx * dx + dy * dy + dz * dz;
}

// capi.mojo:522-586, one query.
void query_one(const double* p, const double* v, const int64_t* f, const double* boxes,
               const int64_t* nodes, const int64_t* order, double* sqrd, int64_t* index,
               double* closest, int64_t* stack, int64_t nnodes, int64_t qi) {
  const double px = p[3 * qi], py = p[3 * qi + 1], pz = p[3 * qi + 2];
  double best = 1.0e300;
  int64_t best_face = -1;
  double bx = 0.0, by = 0.0, bz = 0.0;
  int64_t top = 0;
  stack[top++] = 0;
  while (top > 0) {
    const int64_t node = stack[--top];
    if (node < 0 || node >= nnodes || box_d2(px, py, pz, boxes + 6 * node) > best) continue;
    const int64_t* nd = nodes + 4 * node;
    if (nd[3] > 0) {
      for (int64_t k = 0; k < nd[3]; ++k) {
        const int64_t fi = order[nd[2] + k];
        const double* A = v + 3 * f[3 * fi];
        const double* B = v + 3 * f[3 * fi + 1];
        const double* C = v + 3 * f[3 * fi + 2];
        const Hit h = closest_point(px, py, pz, A[0], A[1], A[2], B[0], B[1], B[2], C[0], C[1],
                                    C[2]);
        if (h.d2 < best) {
          best = h.d2;
          best_face = fi;
          bx = h.x; by = h.y; bz = h.z;
        }
      }
    } else {
      const int64_t l = nd[0], r = nd[1];
      const double dl = box_d2(px, py, pz, boxes + 6 * l);
      const double dr = box_d2(px, py, pz, boxes + 6 * r);
      const int64_t first = dl < dr ? r : l, second = dl < dr ? l : r;
      const double dfirst = dl < dr ? dr : dl, dsecond = dl < dr ? dl : dr;
      if (dfirst <= best) stack[top++] = first;
      if (dsecond <= best) stack[top++] = second;
    }
  }
  sqrd[qi] = best;
  index[qi] = best_face;
  closest[3 * qi] = bx;
  closest[3 * qi + 1] = by;
  closest[3 * qi + 2] = bz;
}

}  // namespace

extern "C" {

// capi.mojo:505-519 behind the export at capi.mojo:950-959: queries q0..q1-1,
// every argument an int64 (host addresses), `stack` one traversal stack of at
// least the tree's depth + 1 entries.
void mli_aabb_squared_distance(int64_t p, int64_t v, int64_t f, int64_t boxes, int64_t nodes,
                               int64_t order, int64_t sqrd, int64_t indices, int64_t closest,
                               int64_t stack, int64_t np, int64_t nnodes, int64_t q0,
                               int64_t q1) {
  (void)np;
  for (int64_t qi = q0; qi < q1; ++qi)
    query_one(reinterpret_cast<const double*>(p), reinterpret_cast<const double*>(v),
              reinterpret_cast<const int64_t*>(f), reinterpret_cast<const double*>(boxes),
              reinterpret_cast<const int64_t*>(nodes), reinterpret_cast<const int64_t*>(order),
              reinterpret_cast<double*>(sqrd), reinterpret_cast<int64_t*>(indices),
              reinterpret_cast<double*>(closest), reinterpret_cast<int64_t*>(stack), nnodes,
              qi);
}

// Oracle extra (no reference counterpart): the closest point on one triangle,
// (d2, x, y, z), for per-triangle bit comparisons.
void oracle_closest_point(const double* p, const double* tri9, double* out4) {
  const Hit h = closest_point(p[0], p[1], p[2], tri9[0], tri9[1], tri9[2], tri9[3], tri9[4],
                              tri9[5], tri9[6], tri9[7], tri9[8]);
  out4[0] = h.d2;
  out4[1] = h.x;
  out4[2] = h.y;
  out4[3] = h.z;
}

}  // extern "C"
