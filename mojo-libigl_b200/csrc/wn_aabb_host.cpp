// Host side of the closest-point path in libwn_b200:
//   * the tree builder (`wn_aabb_build`): the median-split hierarchy that the
//     reference builds in Python (python/igl/__init__.py:286-319), here in C++
//     with subtrees built on separate threads;
//   * the packer that validates tree arrays and lays them out for the device;
//   * `mli_aabb_squared_distance`, the reference's C-ABI export for the CPU
//     query (src/capi.mojo:950-959, traversal capi.mojo:505-586), on the shared
//     bit-exact arithmetic of wn_aabb.cuh (this file is built with
//     -ffp-contract=off).
//
// Tree definition (what makes two builds identical): face boxes lo/hi are the
// per-axis min/max of the three corners and the centre is 0.5 * (lo + hi).
// A node over a list of faces stores the box of their boxes. A list of at most
// `leaf` faces is a leaf (left = right = -1, start = its position in `order`,
// count = its size). Otherwise the split axis is the first axis of largest
// centre extent (max - min), the list is stably sorted by that centre
// coordinate (equal keys keep their current relative order), and the first
// len / 2 faces go left. Nodes are numbered in preorder, the left subtree
// before the right one, so a node with n faces owns the next count(n) indices,
// count(n) = 1 for n <= leaf and 1 + count(n / 2) + count(n - n / 2) above.
// That fixed numbering lets two subtrees be built at the same time.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <thread>
#include <unordered_map>
#include <utility>
#include <vector>

#include "wn_aabb.cuh"
#include "wn_aabb.h"

namespace wn {
namespace {

struct NodeCounter {
  int64_t leaf;
  std::unordered_map<int64_t, int64_t> memo;
  int64_t operator()(int64_t n) {
    if (n <= leaf) return 1;
    auto it = memo.find(n);
    if (it != memo.end()) return it->second;
    const int64_t c = 1 + (*this)(n / 2) + (*this)(n - n / 2);
    memo.emplace(n, c);
    return c;
  }
};

// Subtrees with more faces than this may be handed to another thread.
constexpr int64_t kParallelFaces = 1 << 14;

struct Builder {
  const double* low;      // nf x 3
  const double* high;     // nf x 3
  const double* centers;  // nf x 3
  int64_t* ids;           // nf, permuted in place; ends as `order`
  double* boxes;
  int64_t* nodes;
  int64_t leaf;
  std::atomic<int> spare{0};
  std::atomic<int64_t> depth{0};

  void build(int64_t lo, int64_t hi, int64_t node, int64_t level,
             std::vector<std::pair<double, int64_t>>& keys) {
    const int64_t n = hi - lo;
    double b[6] = {low[3 * ids[lo]], low[3 * ids[lo] + 1], low[3 * ids[lo] + 2],
                   high[3 * ids[lo]], high[3 * ids[lo] + 1], high[3 * ids[lo] + 2]};
    for (int64_t i = lo + 1; i < hi; ++i) {
      const int64_t f = ids[i];
      for (int k = 0; k < 3; ++k) {
        if (low[3 * f + k] < b[k]) b[k] = low[3 * f + k];
        if (high[3 * f + k] > b[3 + k]) b[3 + k] = high[3 * f + k];
      }
    }
    std::copy(b, b + 6, boxes + 6 * node);
    if (n <= leaf) {
      int64_t* nd = nodes + 4 * node;
      nd[0] = -1;
      nd[1] = -1;
      nd[2] = lo;
      nd[3] = n;
      int64_t seen = depth.load(std::memory_order_relaxed);
      while (level > seen && !depth.compare_exchange_weak(seen, level)) {
      }
      return;
    }
    double cmin[3], cmax[3];
    for (int k = 0; k < 3; ++k) cmin[k] = cmax[k] = centers[3 * ids[lo] + k];
    for (int64_t i = lo + 1; i < hi; ++i) {
      const double* c = centers + 3 * ids[i];
      for (int k = 0; k < 3; ++k) {
        if (c[k] < cmin[k]) cmin[k] = c[k];
        if (c[k] > cmax[k]) cmax[k] = c[k];
      }
    }
    int axis = 0;
    for (int k = 1; k < 3; ++k)
      if (cmax[k] - cmin[k] > cmax[axis] - cmin[axis]) axis = k;
    keys.resize(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) keys[i] = {centers[3 * ids[lo + i] + axis], ids[lo + i]};
    std::stable_sort(keys.begin(), keys.end(),
                     [](const std::pair<double, int64_t>& x, const std::pair<double, int64_t>& y) {
                       return x.first < y.first;
                     });
    for (int64_t i = 0; i < n; ++i) ids[lo + i] = keys[i].second;
    const int64_t half = n / 2;
    NodeCounter count{leaf, {}};
    const int64_t left = node + 1, right = node + 1 + count(half);
    int64_t* nd = nodes + 4 * node;
    nd[0] = left;
    nd[1] = right;
    nd[2] = 0;
    nd[3] = 0;
    bool fork = false;
    if (half > kParallelFaces) {
      int s = spare.load(std::memory_order_relaxed);
      while (s > 0 && !spare.compare_exchange_weak(s, s - 1)) {
      }
      fork = s > 0;
    }
    if (fork) {
      std::thread worker([this, lo, half, left, level] {
        std::vector<std::pair<double, int64_t>> own;
        build(lo, lo + half, left, level + 1, own);
      });
      build(lo + half, hi, right, level + 1, keys);
      worker.join();
      spare.fetch_add(1);
    } else {
      build(lo, lo + half, left, level + 1, keys);
      build(lo + half, hi, right, level + 1, keys);
    }
  }
};

}  // namespace

int64_t aabb_node_count(int64_t nf, int64_t leaf) {
  if (nf <= 0) return 0;
  NodeCounter count{leaf, {}};
  return count(nf);
}

int64_t aabb_build(const double* V, int64_t nv, const int64_t* F, int64_t nf, int64_t leaf,
                   double* boxes, int64_t* nodes, int64_t* order, int threads, const char** why) {
  if (nv < 0 || nf < 0 || leaf < 1) {
    *why = "negative size or leaf size < 1";
    return -1;
  }
  if (nf == 0) return 0;
  if (!V || !F || !boxes || !nodes || !order) {
    *why = "null pointer";
    return -1;
  }
  for (int64_t i = 0; i < 3 * nf; ++i)
    if (F[i] < 0 || F[i] >= nv) {
      *why = "face index outside V";
      return -1;
    }
  std::vector<double> low(3 * nf), high(3 * nf), centers(3 * nf);
  for (int64_t f = 0; f < nf; ++f) {
    for (int k = 0; k < 3; ++k) {
      const double a = V[3 * F[3 * f] + k], b = V[3 * F[3 * f + 1] + k],
                   c = V[3 * F[3 * f + 2] + k];
      if (!std::isfinite(a) || !std::isfinite(b) || !std::isfinite(c)) {
        *why = "non-finite vertex coordinate";
        return -1;
      }
      low[3 * f + k] = std::min(std::min(a, b), c);
      high[3 * f + k] = std::max(std::max(a, b), c);
      centers[3 * f + k] = 0.5 * (low[3 * f + k] + high[3 * f + k]);
    }
  }
  for (int64_t f = 0; f < nf; ++f) order[f] = f;
  Builder b;
  b.low = low.data();
  b.high = high.data();
  b.centers = centers.data();
  b.ids = order;
  b.boxes = boxes;
  b.nodes = nodes;
  b.leaf = leaf;
  if (threads <= 0) threads = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
  b.spare.store(threads - 1);
  std::vector<std::pair<double, int64_t>> keys;
  b.build(0, nf, 0, 1, keys);
  return b.depth.load() + 1;
}

namespace {

float round_down(double x) {
  float f = static_cast<float>(x);
  if (static_cast<double>(f) > x) f = std::nextafter(f, -INFINITY);
  return f;
}

float round_up(double x) {
  float f = static_cast<float>(x);
  if (static_cast<double>(f) < x) f = std::nextafter(f, INFINITY);
  return f;
}

// Slab of every node: the normalised area-weighted normal sum of its faces,
// stored as floats scaled so that |n| <= 1 (then |n.(p - x)| <= |p - x|), and
// the range of n.x over the vertices of its faces, widened by a margin for the
// FP64 rounding of n.x and rounded outward to float. A node whose faces are not
// one contiguous run of `order` (possible only in a caller-made tree) gets the
// empty slab [-inf, +inf], which never skips anything.
void build_slabs(const AabbTriRec* tris, const int64_t* nodes, int64_t nnodes, double scale,
                 std::vector<AabbSlab>& slabs, int threads) {
  std::vector<double> nsum(3 * static_cast<size_t>(nnodes), 0.0);
  std::vector<int64_t> first(nnodes), last(nnodes);
  std::vector<char> whole(nnodes, 1);
  for (int64_t i = nnodes - 1; i >= 0; --i) {  // children come after their parent
    const int64_t* nd = nodes + 4 * i;
    double* n = &nsum[3 * i];
    if (nd[3] > 0) {
      first[i] = nd[2];
      last[i] = nd[2] + nd[3];
      for (int64_t k = first[i]; k < last[i]; ++k) {
        const AabbTriRec& t = tris[k];
        const double u[3] = {t.b[0] - t.a[0], t.b[1] - t.a[1], t.b[2] - t.a[2]};
        const double w[3] = {t.c[0] - t.a[0], t.c[1] - t.a[1], t.c[2] - t.a[2]};
        n[0] += u[1] * w[2] - u[2] * w[1];
        n[1] += u[2] * w[0] - u[0] * w[2];
        n[2] += u[0] * w[1] - u[1] * w[0];
      }
    } else {
      const int64_t l = nd[0], r = nd[1];
      for (int k = 0; k < 3; ++k) n[k] = nsum[3 * l + k] + nsum[3 * r + k];
      first[i] = std::min(first[l], first[r]);
      last[i] = std::max(last[l], last[r]);
      whole[i] = whole[l] && whole[r] && (last[l] == first[r] || last[r] == first[l]);
    }
  }
  slabs.assign(static_cast<size_t>(nnodes), AabbSlab{{0.f, 0.f, 0.f}, -INFINITY, INFINITY});
  const double pad = 1e-13 * 3.0 * scale;  // >> the rounding of a 3-term dot product
  auto work = [&](int64_t begin, int64_t step) {
    for (int64_t i = begin; i < nnodes; i += step) {
      if (!whole[i]) continue;
      const double* s = &nsum[3 * i];
      const double len = std::sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
      double n[3] = {1.0, 0.0, 0.0};
      if (len > 0.0 && std::isfinite(len))
        for (int k = 0; k < 3; ++k) n[k] = s[k] / len;
      float nf[3];
      for (int k = 0; k < 3; ++k) nf[k] = static_cast<float>(n[k]);
      for (int guard = 0; guard < 8; ++guard) {  // shrink until |nf| <= 1
        const double m = std::sqrt(static_cast<double>(nf[0]) * nf[0] +
                                   static_cast<double>(nf[1]) * nf[1] +
                                   static_cast<double>(nf[2]) * nf[2]);
        if (m <= 1.0) break;
        for (int k = 0; k < 3; ++k) nf[k] *= 1.0f - 1.0f / 8388608.0f;
      }
      double lo = INFINITY, hi = -INFINITY;
      for (int64_t k = first[i]; k < last[i]; ++k) {
        const AabbTriRec& t = tris[k];
        for (const double* v : {t.a, t.b, t.c}) {
          const double d = static_cast<double>(nf[0]) * v[0] + static_cast<double>(nf[1]) * v[1] +
                           static_cast<double>(nf[2]) * v[2];
          lo = std::min(lo, d);
          hi = std::max(hi, d);
        }
      }
      AabbSlab& out = slabs[i];
      for (int k = 0; k < 3; ++k) out.n[k] = nf[k];
      out.lo = round_down(lo - pad);
      out.hi = round_up(hi + pad);
    }
  };
  if (threads <= 1 || nnodes < 4096) {
    work(0, 1);
  } else {
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(work, t, threads);
    for (auto& th : pool) th.join();
  }
}

}  // namespace

int64_t aabb_pack(const double* V, int64_t nv, const int64_t* F, int64_t nf, const double* boxes,
                  const int64_t* nodes, const int64_t* order, int64_t nnodes,
                  AabbNodeRec* node_out, AabbTriRec* tri_out, double* scale, const char** why) {
  *scale = 0.0;
  if (nnodes == 0) return 0;
  if (nnodes < 0 || nnodes > 0x7fffffffLL || nf <= 0 || nf > 0x7fffffffLL) {
    *why = "node or face count out of range";
    return -1;
  }
  for (int64_t i = 0; i < nf; ++i) {
    const int64_t f = order[i];
    if (f < 0 || f >= nf) {
      *why = "order entry outside the faces";
      return -1;
    }
    AabbTriRec& r = tri_out[i];
    for (int c = 0; c < 3; ++c) {
      const int64_t v = F[3 * f + c];
      if (v < 0 || v >= nv) {
        *why = "face index outside V";
        return -1;
      }
      double* dst = c == 0 ? r.a : (c == 1 ? r.b : r.c);
      for (int k = 0; k < 3; ++k) {
        dst[k] = V[3 * v + k];
        if (!std::isfinite(dst[k])) {
          *why = "non-finite vertex coordinate";
          return -1;
        }
        *scale = std::max(*scale, std::fabs(dst[k]));
      }
    }
    r.face = f;
  }
  // Depth of every node, walking in index order: children must come after
  // their parent (true of any preorder numbering), which also rules out cycles.
  std::vector<int32_t> level(static_cast<size_t>(nnodes), 0);
  level[0] = 1;
  int64_t depth = 0;
  for (int64_t i = 0; i < nnodes; ++i) {
    const int64_t* nd = nodes + 4 * i;
    AabbNodeRec& r = node_out[i];
    for (int k = 0; k < 6; ++k) r.lbox[k] = r.rbox[k] = 0.0;
    for (int k = 0; k < 2; ++k) r.pad[k] = 0;
    if (level[i] == 0) {
      *why = "node unreachable from the root";
      return -1;
    }
    depth = std::max<int64_t>(depth, level[i]);
    if (nd[3] > 0) {
      if (nd[2] < 0 || nd[3] > nf || nd[2] > nf - nd[3]) {
        *why = "leaf range outside order";
        return -1;
      }
      r.left = r.right = -1;
      r.start = static_cast<int32_t>(nd[2]);
      r.count = static_cast<int32_t>(nd[3]);
      continue;
    }
    const int64_t l = nd[0], rr = nd[1];
    if (l <= i || l >= nnodes || rr <= i || rr >= nnodes) {
      *why = "child index not after its parent or outside the tree";
      return -1;
    }
    level[l] = std::max(level[l], level[i] + 1);
    level[rr] = std::max(level[rr], level[i] + 1);
    r.left = static_cast<int32_t>(l);
    r.right = static_cast<int32_t>(rr);
    r.start = 0;
    r.count = 0;
    for (int k = 0; k < 6; ++k) {
      r.lbox[k] = boxes[6 * l + k];
      r.rbox[k] = boxes[6 * rr + k];
    }
  }
  if (depth + 1 > kAabbStack) {
    *why = "tree deeper than the traversal stack";
    return -1;
  }
  std::vector<AabbSlab> slabs;
  build_slabs(tri_out, nodes, nnodes, *scale, slabs,
              static_cast<int>(std::max(1u, std::thread::hardware_concurrency())));
  for (int64_t i = 0; i < nnodes; ++i) {
    AabbNodeRec& r = node_out[i];
    if (r.count > 0) {
      r.lslab = r.rslab = AabbSlab{{0.f, 0.f, 0.f}, -INFINITY, INFINITY};
    } else {
      r.lslab = slabs[r.left];
      r.rslab = slabs[r.right];
    }
  }
  return depth;
}

}  // namespace wn

namespace {

// capi.mojo:522-586 for one query.
void query_one(const double* p, const double* v, const int64_t* f, const double* boxes,
               const int64_t* nodes, const int64_t* order, double* sqrd, int64_t* index,
               double* closest, int64_t* stack, int64_t nnodes, int64_t qi) {
  const double px = p[3 * qi], py = p[3 * qi + 1], pz = p[3 * qi + 2];
  auto box = [&](int64_t n) {
    const double* b = boxes + 6 * n;
    return wn::box_distance2(px, py, pz, b[0], b[1], b[2], b[3], b[4], b[5]);
  };
  double best = 1.0e300, bx = 0.0, by = 0.0, bz = 0.0;
  int64_t best_face = -1;
  int64_t sp = 1;
  stack[0] = 0;
  while (sp > 0) {
    const int64_t node = stack[--sp];
    if (node < 0 || node >= nnodes || box(node) > best) continue;
    const int64_t* nd = nodes + 4 * node;
    if (nd[3] > 0) {
      for (int64_t k = nd[2]; k < nd[2] + nd[3]; ++k) {
        const int64_t fi = order[k];
        const double* A = v + 3 * f[3 * fi];
        const double* B = v + 3 * f[3 * fi + 1];
        const double* C = v + 3 * f[3 * fi + 2];
        const wn::ClosestHit h =
            wn::closest_on_triangle(px, py, pz, A[0], A[1], A[2], B[0], B[1], B[2], C[0], C[1],
                                    C[2]);
        if (h.d2 < best) {
          best = h.d2;
          best_face = fi;
          bx = h.x;
          by = h.y;
          bz = h.z;
        }
      }
    } else {
      const double dl = box(nd[0]), dr = box(nd[1]);
      const bool left_near = dl < dr;
      const int64_t first = left_near ? nd[1] : nd[0], second = left_near ? nd[0] : nd[1];
      if ((left_near ? dr : dl) <= best) stack[sp++] = first;
      if ((left_near ? dl : dr) <= best) stack[sp++] = second;
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

// Reference: src/capi.mojo:950-959 `mli_aabb_squared_distance(p, v, f, boxes,
// nodes, order, sqrd, indices, closest, stack, np, nnodes, q0, q1)`, every
// argument an int64 (host addresses, python/igl/_lib.py:23); fills queries
// q0..q1-1 using `stack` (at least depth + 1 entries) as the traversal stack.
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

// Diagnostic (no reference counterpart): the closest point on one triangle
// (A, B, C as 9 doubles) from p, out4 = (d2, x, y, z), by the function the
// host traversal and the GPU kernel share (wn_aabb.cuh). Lets tests pin that
// arithmetic against the reference's on arbitrary triangles.
int wn_closest_point(const double* p, const double* tri9, double* out4) {
  if (!p || !tri9 || !out4) return 1;
  const wn::ClosestHit h =
      wn::closest_on_triangle(p[0], p[1], p[2], tri9[0], tri9[1], tri9[2], tri9[3], tri9[4],
                              tri9[5], tri9[6], tri9[7], tri9[8]);
  out4[0] = h.d2;
  out4[1] = h.x;
  out4[2] = h.y;
  out4[3] = h.z;
  return 0;
}

}  // extern "C"
