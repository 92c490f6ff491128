// Host side of the closest-point path in libwn_b200:
//   * the tree builder (`wn_aabb_build`): the median-split hierarchy that the
//     reference builds in Python (python/igl/__init__.py:286-319), here in C++
//     with subtrees built on separate threads;
//   * the packer that validates tree arrays and lays them out for the device;
//   * `mli_aabb_squared_distance`, the reference's C-ABI export for the CPU
//     query (src/capi.mojo:950-959, traversal capi.mojo:505-586), on the shared
//     bit-exact arithmetic of wn_aabb.cuh (this file is built with
//     -ffp-contract=off): the reference's walk, with each pushed node's box
//     distance kept on the stack and a leaf's faces evaluated eight at a time
//     in AVX-512 lanes (closest8), both without changing a bit.
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
#include <immintrin.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <memory>
#include <new>
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

// ---- a leaf's faces eight at a time (AVX-512) -------------------------------
// closest_on_triangle on eight faces at once, one per 64-bit lane: every
// quantity of every region (the Voronoi walk's vertex, edge and interior
// cases) is computed in all lanes with the scalar code's IEEE operations in the
// same order (this file is built without FMA contraction; vector add, multiply
// and divide round like their scalar forms), and each lane keeps the region the
// scalar code would enter, decided by the same comparisons (ordered: false on
// NaN, like C's). A lane whose triangle is degenerate (|denom| <= 1e-30 in the
// interior case) is redone by the scalar function. So every lane's squared
// distance and closest point are the scalar bits, and the caller still takes
// the faces one by one in leaf order with the strict `<` update.

#define WN_AVX512 __attribute__((target("avx512f,avx512dq")))

struct Vec3x8 {
  __m512d x, y, z;
};

WN_AVX512 inline Vec3x8 sub3(const Vec3x8& a, const Vec3x8& b) {
  return {_mm512_sub_pd(a.x, b.x), _mm512_sub_pd(a.y, b.y), _mm512_sub_pd(a.z, b.z)};
}

WN_AVX512 inline __m512d dot3x8(const Vec3x8& a, const Vec3x8& b) {
  return _mm512_add_pd(_mm512_add_pd(_mm512_mul_pd(a.x, b.x), _mm512_mul_pd(a.y, b.y)),
                       _mm512_mul_pd(a.z, b.z));
}

// o + t * e, per component as the scalar dadd(o, dmul(t, e)).
WN_AVX512 inline Vec3x8 along(const Vec3x8& o, __m512d t, const Vec3x8& e) {
  return {_mm512_add_pd(o.x, _mm512_mul_pd(t, e.x)), _mm512_add_pd(o.y, _mm512_mul_pd(t, e.y)),
          _mm512_add_pd(o.z, _mm512_mul_pd(t, e.z))};
}

// a <= b and a >= b per lane, false on NaN (C's relational operators).
WN_AVX512 inline __mmask8 le(__m512d a, __m512d b) { return _mm512_cmp_pd_mask(a, b, _CMP_LE_OQ); }
WN_AVX512 inline __mmask8 ge(__m512d a, __m512d b) { return _mm512_cmp_pd_mask(a, b, _CMP_GE_OQ); }

WN_AVX512 inline Vec3x8 pick(__mmask8 m, const Vec3x8& a, const Vec3x8& b) {  // m ? b : a
  return {_mm512_mask_blend_pd(m, a.x, b.x), _mm512_mask_blend_pd(m, a.y, b.y),
          _mm512_mask_blend_pd(m, a.z, b.z)};
}

// tri: 9 x 8 doubles (A xyz, B xyz, C xyz rows, one face per column).
// out: d2, x, y, z rows of 8. Lanes not in `live` are computed but unused.
WN_AVX512 void closest8(double px, double py, double pz, const double* tri, double* out) {
  const Vec3x8 P{_mm512_set1_pd(px), _mm512_set1_pd(py), _mm512_set1_pd(pz)};
  const Vec3x8 A{_mm512_load_pd(tri), _mm512_load_pd(tri + 8), _mm512_load_pd(tri + 16)};
  const Vec3x8 B{_mm512_load_pd(tri + 24), _mm512_load_pd(tri + 32), _mm512_load_pd(tri + 40)};
  const Vec3x8 C{_mm512_load_pd(tri + 48), _mm512_load_pd(tri + 56), _mm512_load_pd(tri + 64)};
  const __m512d zero = _mm512_setzero_pd();
  const Vec3x8 ab = sub3(B, A), ac = sub3(C, A), ap = sub3(P, A);
  const __m512d d1 = dot3x8(ab, ap), d2 = dot3x8(ac, ap);
  const Vec3x8 bp = sub3(P, B);
  const __m512d d3 = dot3x8(ab, bp), d4 = dot3x8(ac, bp);
  const __m512d vc = _mm512_sub_pd(_mm512_mul_pd(d1, d4), _mm512_mul_pd(d3, d2));
  const Vec3x8 cp = sub3(P, C);
  const __m512d d5 = dot3x8(ab, cp), d6 = dot3x8(ac, cp);
  const __m512d vb = _mm512_sub_pd(_mm512_mul_pd(d5, d2), _mm512_mul_pd(d1, d6));
  const __m512d va = _mm512_sub_pd(_mm512_mul_pd(d3, d6), _mm512_mul_pd(d5, d4));
  const __m512d u43 = _mm512_sub_pd(d4, d3), u56 = _mm512_sub_pd(d5, d6);
  const __m512d denom = _mm512_add_pd(_mm512_add_pd(va, vb), vc);
  // The scalar code's regions, first match wins.
  const __mmask8 r0 = le(d1, zero) & le(d2, zero);                 // vertex A
  const __mmask8 r1 = ge(d3, zero) & le(d4, d3);                   // vertex B
  const __mmask8 r2 = le(vc, zero) & ge(d1, zero) & le(d3, zero);  // edge AB
  const __mmask8 r3 = ge(d6, zero) & le(d5, d6);                   // vertex C
  const __mmask8 r4 = le(vb, zero) & ge(d2, zero) & le(d6, zero);  // edge AC
  const __mmask8 r5 = le(va, zero) & ge(u43, zero) & ge(u56, zero);  // edge BC
  const __mmask8 rd =
      _mm512_cmp_pd_mask(_mm512_abs_pd(denom), _mm512_set1_pd(1.0e-30), _CMP_LE_OQ);
  const __m512d inv = _mm512_div_pd(_mm512_set1_pd(1.0), denom);
  const __m512d v = _mm512_mul_pd(vb, inv), w = _mm512_mul_pd(vc, inv);
  Vec3x8 q{_mm512_add_pd(_mm512_add_pd(A.x, _mm512_mul_pd(ab.x, v)), _mm512_mul_pd(ac.x, w)),
           _mm512_add_pd(_mm512_add_pd(A.y, _mm512_mul_pd(ab.y, v)), _mm512_mul_pd(ac.y, w)),
           _mm512_add_pd(_mm512_add_pd(A.z, _mm512_mul_pd(ab.z, v)), _mm512_mul_pd(ac.z, w))};
  // Apply the regions from the last to the first, so the first match is what stays.
  const Vec3x8 bc = sub3(C, B);
  q = pick(r5, q, along(B, _mm512_div_pd(u43, _mm512_add_pd(u43, u56)), bc));
  q = pick(r4, q, along(A, _mm512_div_pd(d2, _mm512_sub_pd(d2, d6)), ac));
  q = pick(r3, q, C);
  q = pick(r2, q, along(A, _mm512_div_pd(d1, _mm512_sub_pd(d1, d3)), ab));
  q = pick(r1, q, B);
  q = pick(r0, q, A);
  const Vec3x8 dq = sub3(P, q);
  _mm512_store_pd(out, dot3x8(dq, dq));
  _mm512_store_pd(out + 8, q.x);
  _mm512_store_pd(out + 16, q.y);
  _mm512_store_pd(out + 24, q.z);
  // Degenerate triangles (interior case with |denom| <= 1e-30): the scalar walk.
  __mmask8 redo = static_cast<__mmask8>(rd & ~(r0 | r1 | r2 | r3 | r4 | r5));
  while (redo) {
    const int j = __builtin_ctz(redo);
    redo = static_cast<__mmask8>(redo & (redo - 1));
    const wn::ClosestHit h = wn::closest_on_triangle(
        px, py, pz, tri[j], tri[8 + j], tri[16 + j], tri[24 + j], tri[32 + j], tri[40 + j],
        tri[48 + j], tri[56 + j], tri[64 + j]);
    out[j] = h.d2;
    out[8 + j] = h.x;
    out[16 + j] = h.y;
    out[24 + j] = h.z;
  }
}

#undef WN_AVX512

bool has_avx512() {
  static const bool yes = __builtin_cpu_supports("avx512f") && __builtin_cpu_supports("avx512dq");
  return yes;
}

// capi.mojo:522-586 for one query.
void query_one(const double* p, const double* v, const int64_t* f, const double* boxes,
               const int64_t* nodes, const int64_t* order, double* sqrd, int64_t* index,
               double* closest, int64_t* stack, double* stack_d2, int64_t nnodes, int64_t qi,
               bool vector8) {
  const double px = p[3 * qi], py = p[3 * qi + 1], pz = p[3 * qi + 2];
  auto box = [&](int64_t n) {
    const double* b = boxes + 6 * n;
    return wn::box_distance2(px, py, pz, b[0], b[1], b[2], b[3], b[4], b[5]);
  };
  double best = 1.0e300, bx = 0.0, by = 0.0, bz = 0.0;
  int64_t best_face = -1;
  int64_t sp = 1;
  stack[0] = 0;
  // Each entry keeps the box distance computed when it was pushed: the
  // reference recomputes it at the pop from the same box and point, which is
  // the same double, so the pop test is unchanged.
  if (stack_d2) stack_d2[0] = nnodes > 0 ? box(0) : 0.0;
  while (sp > 0) {
    const int64_t node = stack[--sp];
    if (node < 0 || node >= nnodes || (stack_d2 ? stack_d2[sp] : box(node)) > best) continue;
    const int64_t* nd = nodes + 4 * node;
    if (nd[3] > 0 && vector8) {
      // Eight faces at a time through closest8, then taken one by one in order.
      alignas(64) double tri[72], hit[32];
      for (int64_t k0 = nd[2]; k0 < nd[2] + nd[3]; k0 += 8) {
        const int n = static_cast<int>(std::min<int64_t>(8, nd[2] + nd[3] - k0));
        for (int j = 0; j < 8; ++j) {
          const int64_t fi = order[k0 + (j < n ? j : 0)];
          for (int c = 0; c < 3; ++c) {
            const double* X = v + 3 * f[3 * fi + c];
            tri[24 * c + j] = X[0];
            tri[24 * c + 8 + j] = X[1];
            tri[24 * c + 16 + j] = X[2];
          }
        }
        closest8(px, py, pz, tri, hit);
        for (int j = 0; j < n; ++j)
          if (hit[j] < best) {
            best = hit[j];
            best_face = order[k0 + j];
            bx = hit[8 + j];
            by = hit[16 + j];
            bz = hit[24 + j];
          }
      }
    } else if (nd[3] > 0) {
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
      if ((left_near ? dr : dl) <= best) {
        if (stack_d2) stack_d2[sp] = left_near ? dr : dl;
        stack[sp++] = first;
      }
      if ((left_near ? dl : dr) <= best) {
        if (stack_d2) stack_d2[sp] = left_near ? dl : dr;
        stack[sp++] = second;
      }
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
  const bool vector8 = has_avx512();
  // Distances beside the caller's stack: a node is pushed at most once per
  // query, so nnodes + 1 entries always suffice. Without the memory the pop
  // recomputes the distance, as the reference does.
  std::unique_ptr<double[]> stack_d2(
      new (std::nothrow) double[static_cast<size_t>(nnodes > 0 ? nnodes : 0) + 1]);
  for (int64_t qi = q0; qi < q1; ++qi)
    query_one(reinterpret_cast<const double*>(p), reinterpret_cast<const double*>(v),
              reinterpret_cast<const int64_t*>(f), reinterpret_cast<const double*>(boxes),
              reinterpret_cast<const int64_t*>(nodes), reinterpret_cast<const int64_t*>(order),
              reinterpret_cast<double*>(sqrd), reinterpret_cast<int64_t*>(indices),
              reinterpret_cast<double*>(closest), reinterpret_cast<int64_t*>(stack),
              stack_d2.get(), nnodes, qi, vector8);
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

// Diagnostic (no reference counterpart): closest8, the eight-lane form the
// host traversal uses for leaf faces, on eight triangles (tri72: rows Ax, Ay,
// Az, Bx, ..., Cz of eight doubles) from p; out32 = rows d2, x, y, z of eight.
// Lets tests pin every lane against the scalar arithmetic. Returns 0, 1 for a
// null argument, 2 when the CPU has no AVX-512.
int wn_closest_point8(const double* p, const double* tri72, double* out32) {
  if (!p || !tri72 || !out32) return 1;
  if (!has_avx512()) return 2;
  alignas(64) double tri[72], hit[32];
  std::copy(tri72, tri72 + 72, tri);
  closest8(p[0], p[1], p[2], tri, hit);
  std::copy(hit, hit + 32, out32);
  return 0;
}

}  // extern "C"
