// Mixed-precision forward: FP32 pair terms, compensated FP32 accumulation
// across face tiles, FP64 refinement of near-surface pairs.
//
// Same sum as the plain kernel (lee101/mojo-libigl, src/capi.mojo:205-286):
// W(o) = sum_f atan2(det_f, denom_f) / (2*pi). Built in three parts.
//
// 1. Mesh preparation (once per mesh). Faces are ordered along a Morton curve
//    of their centroids and cut into tiles of T = 64 consecutive faces. Per
//    tile: an FP64 centre c, a power-of-two scale s ~ 1/radius, and the squared
//    "far" radius (r + kappa*h_tile)^2, where r bounds |v - c| over the tile's
//    vertices and h_tile is its longest edge. Per face, in FP32 tile-local
//    scaled coordinates: A, B, C, the normal n = (B-A) x (C-A) (formed in FP64,
//    then rounded), and thr = (kappa*h_face*s)^2. An FP64 copy of the sorted
//    soup serves the refinement.
// 2. Query preparation (once per batch). Queries are ordered along a Morton
//    curve so that a warp's 32 queries are spatial neighbours.
// 3. The kernel. A CTA holds THREADS*QPT sorted queries, QPT per thread, and
//    streams tile records through a shared-memory ring filled by 1-D bulk
//    copies. Per (query, tile), in FP64: o - c, the far test, and o_local =
//    float((o - c)*s). Per pair, in FP32, with a = A - o_local etc.:
//       ra = rsqrt(|a|^2) ...,  denom' = 1 + (a.b) ra rb + (b.c) rb rc + (c.a) rc ra
//       det' = (a . n) ra rb rc      [det = a.(b x c) = a.((B-A) x (C-A))]
//    so z' = denom' + i det' = z / (la lb lc) has the pair's angle and a
//    magnitude in [3.8, 4.01] (see below). The tile's angles are added by
//    multiplying the z' (the argument of a product is the sum of arguments),
//    then one atan2f per (query, tile); tile angles are summed in an FP32
//    two-sum (hi, lo) pair.
//
// Why this is safe. A pair is "near" when some vertex is closer than
// kappa*h_face (h_face = the face's longest edge); near pairs are evaluated in
// FP64 with the bit-exact pair terms and atan2, into an FP64 sum. For every
// other pair the triangle lies at distance >= (kappa - 1/sqrt(3)) h_face, so
// its solid angle is <= (sqrt(3)/4)/(kappa - 0.577)^2 and each side subtends
// <= 2 asin(1/(2 kappa)): with kappa >= 3, |atan2| <= 0.037 per pair (sum over
// a 64-face tile < pi, so atan2f of the product needs no turn counting) and
// denom' >= 3.8. The running product starts at 2^-100 and after 64 factors in
// [1, 4.01] stays within [2^-100, 2^28.1]: no rescaling. A tile whose ball
// B(c, r + kappa*h_tile) excludes every query of a warp has no near pair: the
// warp then runs the loop without the near test (the fast path).
#include <cub/cub.cuh>

#include <algorithm>
#include <numeric>
#include <vector>

#include "wn_batch.h"
#include "wn_common.cuh"
#include "wn_internal.h"
#include "wn_mixed.h"
#include "wn_pair.cuh"

namespace wn {
namespace {

constexpr float kZ0 = 7.8886090522101181e-31f;  // 2^-100, start of each tile product

__device__ __forceinline__ float rsqrt_approx(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Order-preserving map double -> uint64 (for atomic min/max of coordinates).
__device__ __forceinline__ unsigned long long ordered_key(double x) {
  const unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(x));
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double from_ordered_key(unsigned long long k) {
  const unsigned long long b = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double(static_cast<long long>(b));
}

__global__ void bbox_init_kernel(unsigned long long* box) {
  if (threadIdx.x < 3) box[threadIdx.x] = ~0ull;      // minima
  else if (threadIdx.x < 6) box[threadIdx.x] = 0ull;  // maxima
}

// Bounding box of face centroids (tri SoA) or of points (AoS xyz).
template <bool CENTROIDS>
__global__ void bbox_kernel(const double* __restrict__ data, int64_t ld, int64_t n,
                            unsigned long long* box) {
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
#pragma unroll
    for (int x = 0; x < 3; ++x) {
      const double v = CENTROIDS ? (data[x * ld + i] + data[(3 + x) * ld + i] +
                                    data[(6 + x) * ld + i]) * (1.0 / 3.0)
                                 : data[3 * i + x];
      lo[x] = fmin(lo[x], v);
      hi[x] = fmax(hi[x], v);
    }
  }
#pragma unroll
  for (int x = 0; x < 3; ++x) {
    for (int off = 16; off; off >>= 1) {
      lo[x] = fmin(lo[x], __shfl_xor_sync(0xffffffffu, lo[x], off));
      hi[x] = fmax(hi[x], __shfl_xor_sync(0xffffffffu, hi[x], off));
    }
  }
  if ((threadIdx.x & 31) == 0 && isfinite(lo[0])) {
#pragma unroll
    for (int x = 0; x < 3; ++x) {
      atomicMin(&box[x], ordered_key(lo[x]));
      atomicMax(&box[3 + x], ordered_key(hi[x]));
    }
  }
}

__device__ __forceinline__ uint32_t spread10(uint32_t v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000ffu;
  v = (v | (v << 8)) & 0x0300f00fu;
  v = (v | (v << 4)) & 0x030c30c3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

__device__ __forceinline__ uint32_t morton30(const double p[3], const unsigned long long* box) {
  uint32_t code = 0;
#pragma unroll
  for (int x = 0; x < 3; ++x) {
    const double lo = from_ordered_key(box[x]), hi = from_ordered_key(box[3 + x]);
    const double ext = hi - lo;
    double u = ext > 0 ? (p[x] - lo) / ext : 0.0;
    u = fmin(fmax(u, 0.0), 1.0);
    const uint32_t c = min(static_cast<uint32_t>(u * 1024.0), 1023u);
    code |= spread10(c) << x;
  }
  return code;
}

template <bool CENTROIDS>
__global__ void morton_kernel(const double* __restrict__ data, int64_t ld, int64_t n,
                              const unsigned long long* __restrict__ box, uint32_t* keys,
                              uint32_t* vals) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double p[3];
#pragma unroll
  for (int x = 0; x < 3; ++x)
    p[x] = CENTROIDS ? (data[x * ld + i] + data[(3 + x) * ld + i] + data[(6 + x) * ld + i]) *
                           (1.0 / 3.0)
                     : data[3 * i + x];
  keys[i] = morton30(p, box);
  vals[i] = static_cast<uint32_t>(i);
}

__device__ __forceinline__ double warp_max(double v) {
  for (int off = 16; off; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
  for (int off = 16; off; off >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, off));
  return v;
}

// One CTA of kTileFaces threads per tile: gathers the tile's faces in Morton
// order, writes the FP64 sorted copy, the tile header and the FP32 records.
// Tile t holds the sorted faces order[first + j], j < count, where first/count
// come from tile_first/tile_count (several meshes, each tiled on its own) or,
// when those are null, first = 64 t and count = min(64, nf - first).
__global__ void __launch_bounds__(kTileFaces) build_tiles_kernel(
    const double* __restrict__ tri, int64_t ld, int64_t nf, const uint32_t* __restrict__ order,
    double kappa, unsigned char* __restrict__ tiles, double* __restrict__ tri64, int64_t ld64,
    uint32_t* __restrict__ face_of, const int64_t* __restrict__ tile_first,
    const int32_t* __restrict__ tile_count, uint8_t* __restrict__ reuse) {
  __shared__ double red[6][kTileFaces / 32];
  __shared__ double sv[kTileFaces][9];  // the tile's faces, input order
  __shared__ int64_t sf[kTileFaces];
  __shared__ int sorder[kTileFaces];
  __shared__ int sbest[kTileFaces / 32];
  const int j = threadIdx.x, warp = j >> 5, lane = j & 31;
  const int64_t tile = blockIdx.x;
  const int64_t first = tile_first ? tile_first[tile] : tile * kTileFaces;
  int cnt = kTileFaces;
  if (tile_count) {
    cnt = tile_count[tile];
  } else {
    const int64_t left = nf - first;
    cnt = static_cast<int>(left < kTileFaces ? (left > 0 ? left : 0) : kTileFaces);
  }
  bool valid = j < cnt;
  double v[9];
  int64_t f = valid ? order[first + j] : 0;
#pragma unroll
  for (int r = 0; r < 9; ++r) v[r] = valid ? tri[r * ld + f] : 0.0;

  // Tile bounding box -> centre.
  double lo[3], hi[3];
#pragma unroll
  for (int x = 0; x < 3; ++x) {
    lo[x] = valid ? fmin(v[x], fmin(v[3 + x], v[6 + x])) : INFINITY;
    hi[x] = valid ? fmax(v[x], fmax(v[3 + x], v[6 + x])) : -INFINITY;
    lo[x] = warp_min(lo[x]);
    hi[x] = warp_max(hi[x]);
  }
  if (lane == 0)
    for (int x = 0; x < 3; ++x) {
      red[x][warp] = lo[x];
      red[3 + x][warp] = hi[x];
    }
  __syncthreads();
  double c[3];
#pragma unroll
  for (int x = 0; x < 3; ++x) {
    double l = red[x][0], h = red[3 + x][0];
    for (int w = 1; w < kTileFaces / 32; ++w) {
      l = fmin(l, red[x][w]);
      h = fmax(h, red[3 + x][w]);
    }
    c[x] = 0.5 * (l + h);
  }
  __syncthreads();
  // Radius (max vertex distance to c) and longest edge, over the tile.
  double r2 = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double dx = v[3 * k] - c[0], dy = v[3 * k + 1] - c[1], dz = v[3 * k + 2] - c[2];
    r2 = fmax(r2, dx * dx + dy * dy + dz * dz);
  }
  double h2 = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int k2 = (k + 1) % 3;
    const double dx = v[3 * k2] - v[3 * k], dy = v[3 * k2 + 1] - v[3 * k + 1],
                 dz = v[3 * k2 + 2] - v[3 * k + 2];
    h2 = fmax(h2, dx * dx + dy * dy + dz * dz);
  }
  if (!valid) r2 = h2 = 0.0;
  double rt = warp_max(sqrt(r2)), ht = warp_max(sqrt(h2));
  if (lane == 0) {
    red[0][warp] = rt;
    red[1][warp] = ht;
  }
  __syncthreads();
  rt = red[0][0];
  ht = red[1][0];
  for (int w = 1; w < kTileFaces / 32; ++w) {
    rt = fmax(rt, red[0][w]);
    ht = fmax(ht, red[1][w]);
  }
  // Power-of-two scale bringing the tile radius near 1 (exact in FP64).
  int e = 0;
  if (rt > 0.0) frexp(rt, &e);
  const double scale = ldexp(1.0, -e);

  unsigned char* rec = tiles + tile * kTileBytes;
  if (j == 0) {
    TileHeader* th = reinterpret_cast<TileHeader*>(rec);
    th->cx = c[0];
    th->cy = c[1];
    th->cz = c[2];
    const double far = rt + kappa * ht;
    th->far_r2 = far * far;
    th->scale = scale;
    th->n = cnt;
    th->first = 0;
    th->r = static_cast<float>(rt);
    th->h = static_cast<float>(ht);
  }
  // Order the tile's faces as strips: each next face is the unvisited one that
  // shares the most corners (bitwise-equal coordinates) with the current one.
  // Consecutive faces then share corners, whose (v - o, |v - o|) the FP64 kernel
  // reuses; reuse[slot] says, per corner, which corner of the previous face it
  // equals (0..2) or 3 for a new one (0xff marks padding).
#pragma unroll
  for (int r = 0; r < 9; ++r) sv[j][r] = v[r];
  sf[j] = f;
  if (j == 0) sorder[0] = 0;
  __syncthreads();
  bool visited = (j == 0) || !valid;
  int cur = 0;
  for (int p = 1; p < cnt; ++p) {
    int key = -1;
    if (!visited) {
      int shared = 0;
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int m = 0; m < 3; ++m)
          shared += (__double_as_longlong(v[3 * k]) == __double_as_longlong(sv[cur][3 * m]) &&
                     __double_as_longlong(v[3 * k + 1]) == __double_as_longlong(sv[cur][3 * m + 1]) &&
                     __double_as_longlong(v[3 * k + 2]) == __double_as_longlong(sv[cur][3 * m + 2]))
                        ? 1 : 0;
      key = (min(shared, 3) << 7) | (127 - j);
    }
    for (int off = 16; off; off >>= 1) key = max(key, __shfl_xor_sync(0xffffffffu, key, off));
    if (lane == 0) sbest[warp] = key;
    __syncthreads();
    int best = sbest[0];
    for (int w = 1; w < kTileFaces / 32; ++w) best = max(best, sbest[w]);
    cur = 127 - (best & 127);
    if (j == cur) visited = true;
    if (j == 0) sorder[p] = cur;
    __syncthreads();
  }
  const int src = j < cnt ? sorder[j] : j;
  const int prev = j >= 1 && j < cnt ? sorder[j - 1] : -1;
  valid = j < cnt;
#pragma unroll
  for (int r = 0; r < 9; ++r) v[r] = sv[src][r];
  f = sf[src];
  const int64_t slot = tile * kTileFaces + j;
#pragma unroll
  for (int r = 0; r < 9; ++r) tri64[r * ld64 + slot] = valid ? v[r] : 0.0;
  face_of[slot] = valid ? static_cast<uint32_t>(f) : 0xffffffffu;
  if (reuse) {
    unsigned code = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      unsigned match = 3;
      if (prev >= 0)
        for (int m = 2; m >= 0; --m)
          if (__double_as_longlong(v[3 * k]) == __double_as_longlong(sv[prev][3 * m]) &&
              __double_as_longlong(v[3 * k + 1]) == __double_as_longlong(sv[prev][3 * m + 1]) &&
              __double_as_longlong(v[3 * k + 2]) == __double_as_longlong(sv[prev][3 * m + 2]))
            match = static_cast<unsigned>(m);
      code |= match << (2 * k);
    }
    reuse[slot] = valid ? static_cast<uint8_t>(code) : static_cast<uint8_t>(0xff);
  }
  double h2f = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int k2 = (k + 1) % 3;
    const double dx = v[3 * k2] - v[3 * k], dy = v[3 * k2 + 1] - v[3 * k + 1],
                 dz = v[3 * k2 + 2] - v[3 * k + 2];
    h2f = fmax(h2f, dx * dx + dy * dy + dz * dz);
  }
  const double h_face = valid ? sqrt(h2f) : 0.0;

  // Half headers: warp w holds faces [32 w, 32 w + 32) of the sorted tile, i.e.
  // half w. Centre of the half's vertex box, radius about it, longest edge.
  static_assert(kHalfFaces == 32, "one warp per half tile");
  {
    double hlo[3], hhi[3], hc[3];
#pragma unroll
    for (int x = 0; x < 3; ++x) {
      hlo[x] = warp_min(valid ? fmin(v[x], fmin(v[3 + x], v[6 + x])) : INFINITY);
      hhi[x] = warp_max(valid ? fmax(v[x], fmax(v[3 + x], v[6 + x])) : -INFINITY);
      hc[x] = isfinite(hlo[x]) ? 0.5 * (hlo[x] + hhi[x]) : c[x];
    }
    double hr2 = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double dx = v[3 * k] - hc[0], dy = v[3 * k + 1] - hc[1], dz = v[3 * k + 2] - hc[2];
      hr2 = fmax(hr2, dx * dx + dy * dy + dz * dz);
    }
    const double hr = warp_max(valid ? sqrt(hr2) : 0.0);
    const double hh = warp_max(h_face);
    if (lane == 0) {
      HalfHeader* half = reinterpret_cast<HalfHeader*>(rec + sizeof(TileHeader));
      const double far = ((hr + kappa * hh) * scale) * (1.0 + 1e-5) + 1e-5;
      half->cx[warp] = static_cast<float>((hc[0] - c[0]) * scale);
      half->cy[warp] = static_cast<float>((hc[1] - c[1]) * scale);
      half->cz[warp] = static_cast<float>((hc[2] - c[2]) * scale);
      half->far_r2[warp] = __double2float_ru(far * far);
      for (int i = 0; i < 4; ++i) half->pad[4 * warp + i] = 0;
    }
  }

  FaceRec fr;
  const double ax = (v[0] - c[0]) * scale, ay = (v[1] - c[1]) * scale, az = (v[2] - c[2]) * scale;
  const double e1x = (v[3] - v[0]) * scale, e1y = (v[4] - v[1]) * scale,
               e1z = (v[5] - v[2]) * scale;
  const double e2x = (v[6] - v[0]) * scale, e2y = (v[7] - v[1]) * scale,
               e2z = (v[8] - v[2]) * scale;
  fr.ax = static_cast<float>(ax);
  fr.ay = static_cast<float>(ay);
  fr.az = static_cast<float>(az);
  fr.e1x = static_cast<float>(e1x);
  fr.e1y = static_cast<float>(e1y);
  fr.e1z = static_cast<float>(e1z);
  fr.e2x = static_cast<float>(e2x);
  fr.e2y = static_cast<float>(e2y);
  fr.e2z = static_cast<float>(e2z);
  fr.nx = static_cast<float>(e1y * e2z - e1z * e2y);
  fr.ny = static_cast<float>(e1z * e2x - e1x * e2z);
  fr.nz = static_cast<float>(e1x * e2y - e1y * e2x);
  fr.e11 = static_cast<float>(e1x * e1x + e1y * e1y + e1z * e1z);
  fr.e22 = static_cast<float>(e2x * e2x + e2y * e2y + e2z * e2z);
  fr.e12 = static_cast<float>(e1x * e2x + e1y * e2y + e1z * e2z);
  // A collapsed face (h = 0) is always refined: in FP64 it contributes
  // atan2(0, denom >= 0) = 0 exactly, and it never reaches rsqrt(0).
  const double thr = kappa * h_face * scale;
  fr.thr = (valid && h_face == 0.0) ? INFINITY : static_cast<float>(thr * thr);
  reinterpret_cast<FaceRec*>(rec + kTileHeaderBytes)[j] = fr;
}

struct MixedArgs {
  const unsigned char* tiles;  // ntiles * kTileBytes
  int64_t ntiles;
  const double* tri64;  // sorted FP64 soup, 9 rows x ld64
  int64_t ld64;
  const double* q;         // nq x 3
  const uint32_t* perm;    // sorted position -> query index
  int64_t nq;
  double* w;                  // output when gridDim.y == 1
  double* partial;            // [gridDim.y][nq] angle sums when gridDim.y > 1
  int64_t tiles_per_split;    // tiles handled by one grid.y slice
  unsigned long long* stats;  // [0] refined pairs, [1] careful (query-warp, tile) visits
  int* err;
};

// Squared lengths and dot products of one pair from a face record (FaceRec
// layout: r0 = A.xyz e1.x, r1 = e1.yz e2.xy, r2 = e2.z n.xyz, r3 = e11 e22 e12 thr).
struct PairSq {
  float aa, bb, cc, ab, bc, ca, det;
};

__device__ __forceinline__ PairSq pair_sq(const float4& r0, const float4& r1, const float4& r2,
                                          const float4& r3, float lx, float ly, float lz) {
  const float ax = r0.x - lx, ay = r0.y - ly, az = r0.z - lz;
  PairSq p;
  p.aa = fmaf(ax, ax, fmaf(ay, ay, az * az));
  const float s1 = fmaf(ax, r0.w, fmaf(ay, r1.x, az * r1.y));  // a.e1
  const float s2 = fmaf(ax, r1.z, fmaf(ay, r1.w, az * r2.x));  // a.e2
  p.det = fmaf(ax, r2.y, fmaf(ay, r2.z, az * r2.w));          // a.(e1 x e2) = a.(b x c)
  p.ab = p.aa + s1;
  p.ca = p.aa + s2;
  p.bb = fmaf(2.f, s1, p.aa + r3.x);
  p.cc = fmaf(2.f, s2, p.aa + r3.y);
  p.bc = p.ab + (s2 + r3.z);
  return p;
}

// z' = (denom + i det) / (|a||b||c|) of a far pair, multiplied into (zr, zi).
__device__ __forceinline__ void pair_mul(const PairSq& p, float& zr, float& zi) {
  const float ra = rsqrt_approx(p.aa), rb = rsqrt_approx(p.bb), rc = rsqrt_approx(p.cc);
  const float rab = ra * rb, rbc = rb * rc, rca = rc * ra;
  const float dn = fmaf(p.ab, rab, fmaf(p.bc, rbc, fmaf(p.ca, rca, 1.f)));
  const float dt = p.det * (rab * rc);
  const float nr = fmaf(zr, dn, -zi * dt);
  const float ni = fmaf(zr, dt, zi * dn);
  zr = nr;
  zi = ni;
}

// Tile angle of one query, added with an FP32 two-sum (Knuth) into (hi, lo).
__device__ __forceinline__ void add_tile_angle(float zr, float zi, float& hi, float& lo) {
  const float ang = atan2f(zi, zr);
  const float s = hi + ang;
  const float bp = s - hi;
  const float err = (hi - (s - bp)) + (ang - bp);
  hi = s;
  lo += err;
}

// Faces [j0, j1) of a tile against the QPT queries of this thread on the careful
// path: FP32 argument-of-product for far pairs, bit-exact FP64 terms + atan2 for
// near pairs, then the range's angle added to the FP32 two-sum (hi, lo). `fr` holds
// the tile's face records, `first` is the tile's first slot in the sorted FP64
// soup, (lx, ly, lz) the queries in the tile's frame, skip[k] marks a query for
// which the tile is dropped (beyond 2^40 tile radii). Warp-collective.
template <int QPT>
__device__ __forceinline__ void careful_range(const float4* fr, int j0, int j1, int64_t first,
                                              const double* __restrict__ tri64, int64_t ld64,
                                              const double (&ox)[QPT], const double (&oy)[QPT],
                                              const double (&oz)[QPT],
                                              const int64_t (&qidx)[QPT],
                                              const float (&lx)[QPT], const float (&ly)[QPT],
                                              const float (&lz)[QPT], const bool (&skip)[QPT],
                                              float (&hi)[QPT], float (&lo)[QPT],
                                              double (&s64)[QPT], unsigned& refined) {
  float zr[QPT], zi[QPT];
#pragma unroll
  for (int k = 0; k < QPT; ++k) {
    zr[k] = kZ0;
    zi[k] = 0.f;
  }
  // Near pairs are only marked here (bit j of near[k]; a tile has at most 64
  // faces) and refined below with the warp's lanes in step, each taking its
  // own next near face in ascending order, instead of the whole warp waiting
  // on every face that any lane finds near.
  static_assert(kTileFaces <= 64, "one bit per face of a tile");
  unsigned long long near[QPT];
#pragma unroll
  for (int k = 0; k < QPT; ++k) near[k] = 0ull;
#pragma unroll 1
  for (int j = j0; j < j1; ++j) {
    const float4 r0 = fr[4 * j], r1 = fr[4 * j + 1], r2 = fr[4 * j + 2], r3 = fr[4 * j + 3];
#pragma unroll
    for (int k = 0; k < QPT; ++k) {
      const PairSq p = pair_sq(r0, r1, r2, r3, lx[k], ly[k], lz[k]);
      if (fminf(p.aa, fminf(p.bb, p.cc)) < r3.w && qidx[k] >= 0)
        near[k] |= 1ull << j;
      else if (!skip[k])
        pair_mul(p, zr[k], zi[k]);
    }
  }
  // A query's refined pairs in this range are multiplied into one FP64 running
  // product (the argument-of-product sum of the FP64 kernels) whose argument
  // is taken once; if it degenerates, the per-pair atan2 sum of the same faces.
#pragma unroll
  for (int k = 0; k < QPT; ++k) {
    const unsigned long long marked = near[k];
    ArgAcc acc;
    argacc_init(acc);
    while (__any_sync(0xffffffffu, near[k] != 0ull)) {
      if (near[k] != 0ull) {
        const int j = __ffsll(static_cast<long long>(near[k])) - 1;
        near[k] &= near[k] - 1ull;
        const double* f64 = tri64 + first + j;
        const int64_t L = ld64;
        double det, denom;
        pair_terms_exact(ox[k], oy[k], oz[k], f64[0], f64[L], f64[2 * L], f64[3 * L],
                         f64[4 * L], f64[5 * L], f64[6 * L], f64[7 * L], f64[8 * L], det,
                         denom);
        argacc_push(acc, denom, det);
        ++refined;
      }
    }
    if (marked != 0ull) {
      if (!acc.bad) {
        s64[k] += atan2(acc.zi, acc.zr) + static_cast<double>(acc.k) * kTwoPi;
      } else {
        for (unsigned long long m = marked; m != 0ull; m &= m - 1ull) {
          const double* f64 = tri64 + first + (__ffsll(static_cast<long long>(m)) - 1);
          const int64_t L = ld64;
          double det, denom;
          pair_terms_exact(ox[k], oy[k], oz[k], f64[0], f64[L], f64[2 * L], f64[3 * L],
                           f64[4 * L], f64[5 * L], f64[6 * L], f64[7 * L], f64[8 * L], det,
                           denom);
          s64[k] += atan2(det, denom);
        }
      }
    }
    add_tile_angle(zr[k], zi[k], hi[k], lo[k]);
  }
}

// ---- face-pair (packed FP32x2) fast path ---------------------------------
// sm_100 issues two FP32 operations per instruction (add/mul/fma .f32x2). The
// fast path packs two FACES of a tile against one query: the query's
// coordinates are the duplicated operand (set once per tile) and a face-pair
// transposed copy of the tile records supplies both faces' fields in adjacent
// registers. The four query-dependent products are expanded about per-face
// constants formed once per tile (in FP64 from the FP32 record, rounded once):
// a.e1 = A.e1 - o.e1, a.e2, a.n likewise and |a|^2 = (|A|^2 + |o|^2) - 2A.o, 13
// packed operations instead of 15 for a = A - o and its four products. On this
// path every query is outside the tile's ball B(c, r + kappa h) while |A| <= r,
// so |A| + |o| <= 3 |a| at worst and the expansion loses at most a few ulps more
// than forming a first. The rest is the scalar path's arithmetic, rounded the
// same way per lane; each lane keeps its own running product (even faces, odd
// faces), both started at 2^-50, and the two are multiplied once per range.
// Each holds at most 32 factors of modulus in [3.8, 4.01], so both stay inside
// [2^-50, 2^14.1] and their product inside [2^-100, 2^28.1], as the scalar
// product does; the sum of the range's angles is the same (< pi in magnitude).
constexpr float kZ0Half = 8.8817841970012523e-16f;  // 2^-50
constexpr int kPairFields = 20;                     // per face: see transpose_tile
constexpr int kPairFloats = 2 * kPairFields;        // one face pair, both lanes
constexpr int kTileTransposedBytes = (kTileFaces / 2) * kPairFloats * 4;

// tbuf[40 p + 2 f + lane] = field f of face 2 p + lane, for the tile at `rec`: 2A
// (0-2), e1 (3-5), e2 (6-8), n (9-11), |e1|^2, |e2|^2, e1.e2 (12-14), |A|^2, A.e1,
// A.e2, A.n (15-18), 0 (19). One thread per face.
__device__ __forceinline__ void transpose_tile(const unsigned char* rec, float* tbuf, int tid,
                                               int threads) {
  const FaceRec* src = reinterpret_cast<const FaceRec*>(rec + kTileHeaderBytes);
  for (int j = tid; j < kTileFaces; j += threads) {
    const FaceRec r = src[j];
    const double ax = r.ax, ay = r.ay, az = r.az;
    const float f[kPairFields] = {
        2.f * r.ax, 2.f * r.ay, 2.f * r.az, r.e1x, r.e1y, r.e1z, r.e2x, r.e2y, r.e2z, r.nx,
        r.ny, r.nz, r.e11, r.e22, r.e12,
        static_cast<float>(ax * ax + ay * ay + az * az),
        static_cast<float>(ax * r.e1x + ay * r.e1y + az * r.e1z),
        static_cast<float>(ax * r.e2x + ay * r.e2y + az * r.e2z),
        static_cast<float>(ax * r.nx + ay * r.ny + az * r.nz), 0.f};
    float* dst = tbuf + kPairFloats * (j >> 1) + (j & 1);
#pragma unroll
    for (int k = 0; k < kPairFields; ++k) dst[2 * k] = f[k];
  }
}

// pair_sq + pair_mul for two faces (lanes) against one query, (nlx, nly, nlz)
// = minus the query's tile-local coordinates and oo = their squared norm, in both
// lanes; v = the face pair's fields as laid out by transpose_tile.
__device__ __forceinline__ void pair2_mul(const float4* v, float2 nlx, float2 nly, float2 nlz,
                                          float2 oo, float2& zr, float2& zi) {
  const float4 v0 = v[0], v1 = v[1], v2 = v[2], v3 = v[3], v4 = v[4];
  const float4 v5 = v[5], v6 = v[6], v7 = v[7], v8 = v[8], v9 = v[9];
  const float2 e12 = make_float2(v7.x, v7.y);
  const float2 one = make_float2(1.f, 1.f), two = make_float2(2.f, 2.f);
  const float2 aa =
      __ffma2_rn(nlx, make_float2(v0.x, v0.y),
                 __ffma2_rn(nly, make_float2(v0.z, v0.w),
                            __ffma2_rn(nlz, make_float2(v1.x, v1.y),
                                       __fadd2_rn(make_float2(v7.z, v7.w), oo))));
  const float2 s1 = __ffma2_rn(nlx, make_float2(v1.z, v1.w),
                               __ffma2_rn(nly, make_float2(v2.x, v2.y),
                                          __ffma2_rn(nlz, make_float2(v2.z, v2.w),
                                                     make_float2(v8.x, v8.y))));
  const float2 s2 = __ffma2_rn(nlx, make_float2(v3.x, v3.y),
                               __ffma2_rn(nly, make_float2(v3.z, v3.w),
                                          __ffma2_rn(nlz, make_float2(v4.x, v4.y),
                                                     make_float2(v8.z, v8.w))));
  const float2 det = __ffma2_rn(nlx, make_float2(v4.z, v4.w),
                                __ffma2_rn(nly, make_float2(v5.x, v5.y),
                                           __ffma2_rn(nlz, make_float2(v5.z, v5.w),
                                                      make_float2(v9.x, v9.y))));
  const float2 ab = __fadd2_rn(aa, s1), ca = __fadd2_rn(aa, s2);
  const float2 bb = __ffma2_rn(two, s1, __fadd2_rn(aa, make_float2(v6.x, v6.y)));
  const float2 cc = __ffma2_rn(two, s2, __fadd2_rn(aa, make_float2(v6.z, v6.w)));
  const float2 bc = __fadd2_rn(ab, __fadd2_rn(s2, e12));
  const float2 ra = make_float2(rsqrt_approx(aa.x), rsqrt_approx(aa.y));
  const float2 rb = make_float2(rsqrt_approx(bb.x), rsqrt_approx(bb.y));
  const float2 rc = make_float2(rsqrt_approx(cc.x), rsqrt_approx(cc.y));
  const float2 rab = __fmul2_rn(ra, rb), rbc = __fmul2_rn(rb, rc), rca = __fmul2_rn(rc, ra);
  const float2 dn = __ffma2_rn(ab, rab, __ffma2_rn(bc, rbc, __ffma2_rn(ca, rca, one)));
  const float2 dt = __fmul2_rn(det, __fmul2_rn(rab, rc));
  const float2 nzi = make_float2(-zi.x, -zi.y);
  const float2 nr = __ffma2_rn(zr, dn, __fmul2_rn(nzi, dt));
  const float2 ni = __ffma2_rn(zr, dt, __fmul2_rn(zi, dn));
  zr = nr;
  zi = ni;
}

// Faces [j0, j1) (j0 even) of a tile on the fast path: face pairs packed, an odd
// last face on the scalar path, then the range's angle into (hi, lo).
template <int QPT>
__device__ __forceinline__ void packed_range(const float4* fr, const float* tbuf, int j0, int j1,
                                             const float (&lx)[QPT], const float (&ly)[QPT],
                                             const float (&lz)[QPT], float (&hi)[QPT],
                                             float (&lo)[QPT]) {
  float2 zr2[QPT], zi2[QPT], nlx[QPT], nly[QPT], nlz[QPT], oo[QPT];
#pragma unroll
  for (int k = 0; k < QPT; ++k) {
    zr2[k] = make_float2(kZ0Half, kZ0Half);
    zi2[k] = make_float2(0.f, 0.f);
    nlx[k] = make_float2(-lx[k], -lx[k]);
    nly[k] = make_float2(-ly[k], -ly[k]);
    nlz[k] = make_float2(-lz[k], -lz[k]);
    const float o2 = fmaf(lx[k], lx[k], fmaf(ly[k], ly[k], lz[k] * lz[k]));
    oo[k] = make_float2(o2, o2);
  }
  const int p1 = j1 >> 1;
  // Eight face pairs per pass: with the shorter products a deeper unroll is what shows
  // in time (four pairs: 440.8 -> 430.1 ms at four CTAs per SM, where either change
  // alone measured no faster; eight pairs at five CTAs: 413.2 -> 410.0 ms).
#pragma unroll 8
  for (int p = j0 >> 1; p < p1; ++p) {
    const float4* v = reinterpret_cast<const float4*>(tbuf + kPairFloats * p);
#pragma unroll
    for (int k = 0; k < QPT; ++k) pair2_mul(v, nlx[k], nly[k], nlz[k], oo[k], zr2[k], zi2[k]);
  }
#pragma unroll
  for (int k = 0; k < QPT; ++k) {
    float zr = zr2[k].x * zr2[k].y - zi2[k].x * zi2[k].y;
    float zi = zr2[k].x * zi2[k].y + zi2[k].x * zr2[k].y;
    if (j1 & 1) {  // the odd last face, on the scalar path
      const int j = j1 - 1;
      pair_mul(pair_sq(fr[4 * j], fr[4 * j + 1], fr[4 * j + 2], fr[4 * j + 3], lx[k], ly[k],
                       lz[k]),
               zr, zi);
    }
    add_tile_angle(zr, zi, hi[k], lo[k]);
  }
}

// One tile against the QPT queries of this thread (tbuf: the face-pair transposed
// records of the tile at `rec`). Warps whose queries all lie outside the tile's
// ball B(c, r + kappa h_tile) take the packed fast path over the whole tile;
// otherwise, with HALF, each 32-face half is tested against its own ball and
// takes the fast or the careful path on its own, and without HALF the whole
// tile takes the careful path. One angle per (query, range) goes into (hi, lo).
// Warp-collective: every lane of the warp must call it.
template <int QPT, bool HALF>
__device__ __forceinline__ void mixed_tile_pairs(const unsigned char* rec, const float* tbuf,
                                                 int64_t first, const double* __restrict__ tri64,
                                                 int64_t ld64, const double (&ox)[QPT],
                                                 const double (&oy)[QPT], const double (&oz)[QPT],
                                                 const int64_t (&qidx)[QPT], float (&hi)[QPT],
                                                 float (&lo)[QPT], double (&s64)[QPT],
                                                 unsigned& refined, unsigned& careful_tiles) {
  const TileHeader& th = *reinterpret_cast<const TileHeader*>(rec);
  const float4* fr = reinterpret_cast<const float4*>(rec + kTileHeaderBytes);
  const int n = th.n;
  bool all_far = true;
  float lx[QPT], ly[QPT], lz[QPT];
  bool skip[QPT];
#pragma unroll
  for (int k = 0; k < QPT; ++k) {
    const double dx = ox[k] - th.cx, dy = oy[k] - th.cy, dz = oz[k] - th.cz;
    const double d2 = dx * dx + dy * dy + dz * dz;
    all_far &= (d2 >= th.far_r2) || qidx[k] < 0;
    lx[k] = static_cast<float>(dx * th.scale);
    ly[k] = static_cast<float>(dy * th.scale);
    lz[k] = static_cast<float>(dz * th.scale);
    // Beyond 2^40 tile radii the tile's solid angle is below 2^-80: it
    // cannot change an FP32 sum, and squared distances could overflow.
    skip[k] = d2 * th.scale * th.scale > 1.2089258196146292e24;
    all_far &= !skip[k];
  }
  if (__all_sync(0xffffffffu, all_far)) {
    packed_range<QPT>(fr, tbuf, 0, n, lx, ly, lz, hi, lo);
    return;
  }
  if constexpr (!HALF) {
    ++careful_tiles;
    careful_range<QPT>(fr, 0, n, first, tri64, ld64, ox, oy, oz, qidx, lx, ly, lz, skip, hi, lo,
                       s64, refined);
  } else {
    const HalfHeader& hh = *reinterpret_cast<const HalfHeader*>(rec + sizeof(TileHeader));
#pragma unroll 1
    for (int h = 0; h < 2; ++h) {
      const int j0 = h * kHalfFaces, j1 = min(n, j0 + kHalfFaces);
      if (j0 >= j1) break;
      // Far test against the half's ball in the tile's FP32 frame; the stored
      // radius is inflated beyond the frame's rounding, so "far" stays exact.
      bool far_h = true;
#pragma unroll
      for (int k = 0; k < QPT; ++k) {
        const float dx = lx[k] - hh.cx[h], dy = ly[k] - hh.cy[h], dz = lz[k] - hh.cz[h];
        far_h &= (fmaf(dx, dx, fmaf(dy, dy, dz * dz)) >= hh.far_r2[h] && !skip[k]) ||
                 qidx[k] < 0;
      }
      if (__all_sync(0xffffffffu, far_h)) {
        packed_range<QPT>(fr, tbuf, j0, j1, lx, ly, lz, hi, lo);
      } else {
        ++careful_tiles;
        careful_range<QPT>(fr, j0, j1, first, tri64, ld64, ox, oy, oz, qidx, lx, ly, lz, skip,
                           hi, lo, s64, refined);
      }
    }
  }
}

// Five CTAs per SM (at most 102 registers; it takes 94-96 without spills): the
// extra warps hide more of the MUFU and packed-FMA latency than the four CTAs at
// 122 registers did (c3 x 2^20: 430.2 -> 413.2 ms, the same results to the bit).
template <int THREADS, int QPT, int STAGES, bool HALF>
__global__ void __launch_bounds__(THREADS, 5) mixed_forward_kernel(const MixedArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* ring = smem_raw;  // [STAGES][kTileBytes]
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + STAGES * kTileBytes);
  // Two face-pair transposed tiles (tile t uses tbuf[t & 1]).
  float* tbuf = reinterpret_cast<float*>(smem_raw + STAGES * kTileBytes + 8 * STAGES);
  const int tid = threadIdx.x;
  const int64_t base = static_cast<int64_t>(blockIdx.x) * (THREADS * QPT);

  double ox[QPT], oy[QPT], oz[QPT];
  int64_t qidx[QPT];
#pragma unroll
  for (int k = 0; k < QPT; ++k) {
    const int64_t s = base + k * THREADS + tid;
    qidx[k] = s < a.nq ? static_cast<int64_t>(a.perm[s]) : -1;
    const int64_t i = qidx[k] >= 0 ? qidx[k] : 0;
    ox[k] = a.nq > 0 ? a.q[3 * i] : 0.0;
    oy[k] = a.nq > 0 ? a.q[3 * i + 1] : 0.0;
    oz[k] = a.nq > 0 ? a.q[3 * i + 2] : 0.0;
  }

  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(&full[s], 1);
    fence_barrier_init();
  }
  __syncthreads();
  const int64_t t_begin = static_cast<int64_t>(blockIdx.y) * a.tiles_per_split;
  const int64_t t_left = a.ntiles - t_begin < a.tiles_per_split ? a.ntiles - t_begin : a.tiles_per_split;
  const int ntiles = static_cast<int>(t_left > 0 ? t_left : 0);
  auto issue = [&](int t) {
    const int slot = t % STAGES;
    mbar_arrive_expect_tx(&full[slot], kTileBytes);
    bulk_g2s(ring + slot * kTileBytes, a.tiles + (t_begin + t) * kTileBytes, kTileBytes,
             &full[slot]);
  };
  int issued = 0;
  if (tid == 0)
    for (; issued < min(STAGES, ntiles); ++issued) issue(issued);

  float hi[QPT], lo[QPT];
  double s64[QPT];
#pragma unroll
  for (int k = 0; k < QPT; ++k) {
    hi[k] = lo[k] = 0.f;
    s64[k] = 0.0;
  }
  unsigned refined = 0, careful_tiles = 0;

  bool failed = false;
  int t = 0;
  for (; t < ntiles; ++t) {
    const int slot = t % STAGES;
    const bool landed = mbar_wait(&full[slot], (t / STAGES) & 1, a.err);
    float* tb = tbuf + (t & 1) * (kTileTransposedBytes / 4);
    // tbuf[t & 1] was last read for tile t - 2, which every thread finished
    // before the barrier of tile t - 1.
    if (landed) transpose_tile(ring + slot * kTileBytes, tb, tid, THREADS);
    if (!__syncthreads_and(landed)) {
      failed = true;
      break;
    }
    if (tid == 0 && t >= 1 && issued < ntiles) issue(issued++);
    mixed_tile_pairs<QPT, HALF>(ring + slot * kTileBytes, tb, (t_begin + t) * kTileFaces, a.tri64,
                          a.ld64, ox, oy, oz, qidx, hi, lo, s64, refined, careful_tiles);
  }

  if (failed) {
    if (tid == 0)
      for (int u = t; u < issued; ++u) mbar_wait(&full[u % STAGES], (u / STAGES) & 1, nullptr);
    __syncthreads();
    return;
  }
#pragma unroll
  for (int k = 0; k < QPT; ++k) {
    if (qidx[k] < 0) continue;
    const double total = static_cast<double>(hi[k]) + static_cast<double>(lo[k]) + s64[k];
    if (gridDim.y == 1)
      a.w[qidx[k]] = total / kTwoPi;
    else
      a.partial[static_cast<int64_t>(blockIdx.y) * a.nq + qidx[k]] = total;
  }
  if (a.stats) {
    unsigned r = refined;
    for (int off = 16; off; off >>= 1) r += __shfl_xor_sync(0xffffffffu, r, off);
    if ((tid & 31) == 0) {
      atomicAdd(&a.stats[0], static_cast<unsigned long long>(r));
      atomicAdd(&a.stats[1], static_cast<unsigned long long>(careful_tiles));
    }
  }
}

__global__ void sum_partials_kernel(const double* __restrict__ partial, int64_t nsplit, int64_t nq,
                                    double* __restrict__ w) {
  const int64_t qi = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (qi >= nq) return;
  double s = 0.0;
  for (int64_t y = 0; y < nsplit; ++y) s += partial[y * nq + qi];
  w[qi] = s / kTwoPi;
}

constexpr int kMixedThreads = 128, kMixedQpt = 2, kMixedStages = 4;

template <int THREADS, int QPT, int STAGES, bool HALF>
cudaError_t launch_mixed_variant(const MixedArgs& a, int64_t nsplit, cudaStream_t stream) {
  auto kernel = mixed_forward_kernel<THREADS, QPT, STAGES, HALF>;
  const size_t smem = static_cast<size_t>(STAGES) * kTileBytes + sizeof(uint64_t) * STAGES +
                      2 * kTileTransposedBytes;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  const int64_t per = static_cast<int64_t>(THREADS) * QPT;
  const int64_t blocks = (a.nq + per - 1) / per;
  kernel<<<dim3(static_cast<unsigned>(blocks), static_cast<unsigned>(nsplit)), THREADS, smem,
           stream>>>(a);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError();
}

int64_t blocks_for(int64_t n, int threads) { return std::max<int64_t>(1, (n + threads - 1) / threads); }

}  // namespace

size_t mixed_sort_scratch_bytes(int64_t n) {
  size_t temp = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, temp, static_cast<uint32_t*>(nullptr),
                                  static_cast<uint32_t*>(nullptr), static_cast<uint32_t*>(nullptr),
                                  static_cast<uint32_t*>(nullptr),
                                  static_cast<int>(std::max<int64_t>(n, 1)), 0, 30);
  const size_t n4 = ((static_cast<size_t>(std::max<int64_t>(n, 1)) * 4 + 255) / 256) * 256;
  return 256 + 4 * n4 + temp;
}

cudaError_t mixed_prepare_mesh(const double* tri, int64_t ld, int64_t nf, double kappa,
                               MixedMesh* m, void* scratch, size_t scratch_bytes,
                               cudaStream_t stream) {
  // scratch layout: box (6 u64) | keys_in | keys_out | vals_in | vals_out | cub temp
  if (scratch_bytes < mixed_sort_scratch_bytes(nf)) return cudaErrorInvalidValue;
  const int64_t ntiles = mixed_tiles(nf);
  m->nf = nf;
  m->ntiles = ntiles;
  m->ld64 = ntiles * kTileFaces;
  m->kappa = kappa;
  const size_t n4 = ((static_cast<size_t>(std::max<int64_t>(nf, 1)) * 4 + 255) / 256) * 256;
  unsigned char* s = static_cast<unsigned char*>(scratch);
  unsigned long long* box = reinterpret_cast<unsigned long long*>(s);
  uint32_t* keys_in = reinterpret_cast<uint32_t*>(s + 256);
  uint32_t* keys_out = reinterpret_cast<uint32_t*>(s + 256 + n4);
  uint32_t* vals_in = reinterpret_cast<uint32_t*>(s + 256 + 2 * n4);
  uint32_t* vals_out = reinterpret_cast<uint32_t*>(s + 256 + 3 * n4);
  void* temp = s + 256 + 4 * n4;
  size_t temp_bytes = scratch_bytes - (256 + 4 * n4);
  const int th = 256;
  if (nf > 0) {
    bbox_init_kernel<<<1, 32, 0, stream>>>(box);
    bbox_kernel<true><<<static_cast<unsigned>(std::min<int64_t>(blocks_for(nf, th), 1184)), th, 0,
                        stream>>>(tri, ld, nf, box);
    morton_kernel<true><<<static_cast<unsigned>(blocks_for(nf, th)), th, 0, stream>>>(
        tri, ld, nf, box, keys_in, vals_in);
    g_launches.fetch_add(3, std::memory_order_relaxed);
    cudaError_t e = cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys_in, keys_out, vals_in,
                                                    vals_out, static_cast<int>(nf), 0, 30, stream);
    if (e != cudaSuccess) return e;
  }
  build_tiles_kernel<<<static_cast<unsigned>(ntiles), kTileFaces, 0, stream>>>(
      tri, ld, nf, vals_out, kappa, m->tiles, m->tri64, m->ld64, m->face_of, nullptr, nullptr,
      m->reuse);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError();
}

MixedSplit plan_mixed(int64_t ntiles, int64_t nq, int sms) {
  MixedSplit p;
  const int64_t per = static_cast<int64_t>(kMixedThreads) * kMixedQpt;
  const int64_t qblocks = std::max<int64_t>(1, (nq + per - 1) / per);
  const int64_t target = static_cast<int64_t>(std::max(sms, 1)) * 8;
  int64_t nsplit = qblocks < target ? (target + qblocks - 1) / qblocks : 1;
  nsplit = std::max<int64_t>(1, std::min(nsplit, ntiles));
  p.tiles_per_split = (ntiles + nsplit - 1) / nsplit;
  p.nsplit = std::max<int64_t>(1, (ntiles + p.tiles_per_split - 1) / p.tiles_per_split);
  p.partial_doubles = p.nsplit > 1 ? p.nsplit * nq : 0;
  return p;
}

cudaError_t mixed_sort_queries(const double* q, int64_t nq, uint32_t* perm, void* scratch,
                               size_t scratch_bytes, cudaStream_t stream) {
  if (nq <= 0) return cudaSuccess;
  if (scratch_bytes < mixed_sort_scratch_bytes(nq)) return cudaErrorInvalidValue;
  const size_t n4 = ((static_cast<size_t>(nq) * 4 + 255) / 256) * 256;
  unsigned char* s = static_cast<unsigned char*>(scratch);
  unsigned long long* box = reinterpret_cast<unsigned long long*>(s);
  uint32_t* keys_in = reinterpret_cast<uint32_t*>(s + 256);
  uint32_t* keys_out = reinterpret_cast<uint32_t*>(s + 256 + n4);
  uint32_t* vals_in = reinterpret_cast<uint32_t*>(s + 256 + 2 * n4);
  void* temp = s + 256 + 4 * n4;
  size_t temp_bytes = scratch_bytes - (256 + 4 * n4);
  const int th = 256;
  bbox_init_kernel<<<1, 32, 0, stream>>>(box);
  bbox_kernel<false><<<static_cast<unsigned>(std::min<int64_t>(blocks_for(nq, th), 1184)), th, 0,
                       stream>>>(q, 0, nq, box);
  morton_kernel<false><<<static_cast<unsigned>(blocks_for(nq, th)), th, 0, stream>>>(
      q, 0, nq, box, keys_in, vals_in);
  g_launches.fetch_add(3, std::memory_order_relaxed);
  return cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys_in, keys_out, vals_in, perm,
                                         static_cast<int>(nq), 0, 30, stream);
}

cudaError_t mixed_forward_sorted(const MixedMesh& m, const double* q, const uint32_t* perm,
                                 int64_t nq, double* w, const MixedSplit& split, double* partial,
                                 unsigned long long* stats, int* err, cudaStream_t stream) {
  if (nq <= 0) return cudaSuccess;
  if (split.nsplit > 1 && !partial) return cudaErrorInvalidValue;
  if (split.nsplit > 65535) return cudaErrorInvalidConfiguration;
  MixedArgs a{m.tiles, m.ntiles, m.tri64, m.ld64, q, perm, nq, w, partial,
              split.tiles_per_split, stats, err};
  cudaError_t e =
      m.tile_faces == kHalfFaces
          ? launch_mixed_variant<kMixedThreads, kMixedQpt, kMixedStages, true>(a, split.nsplit,
                                                                               stream)
          : launch_mixed_variant<kMixedThreads, kMixedQpt, kMixedStages, false>(a, split.nsplit,
                                                                                stream);
  if (e != cudaSuccess || split.nsplit == 1) return e;
  sum_partials_kernel<<<static_cast<unsigned>(blocks_for(nq, 256)), 256, 0, stream>>>(
      partial, split.nsplit, nq, w);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError();
}

size_t mixed_forward_scratch_bytes(int64_t ntiles, int64_t nq, int sms) {
  const MixedSplit p = plan_mixed(ntiles, nq, sms);
  const size_t perm = ((static_cast<size_t>(std::max<int64_t>(nq, 1)) * 4 + 255) / 256) * 256;
  return perm + sizeof(double) * p.partial_doubles + mixed_sort_scratch_bytes(nq);
}

cudaError_t mixed_forward(const MixedMesh& m, const double* q, int64_t nq, double* w,
                          void* scratch, size_t scratch_bytes, int sms,
                          unsigned long long* stats, int* err, cudaStream_t stream) {
  if (nq <= 0) return cudaSuccess;
  if (scratch_bytes < mixed_forward_scratch_bytes(m.ntiles, nq, sms))
    return cudaErrorInvalidValue;
  const MixedSplit p = plan_mixed(m.ntiles, nq, sms);
  unsigned char* s = static_cast<unsigned char*>(scratch);
  uint32_t* perm = reinterpret_cast<uint32_t*>(s);
  const size_t perm_bytes = ((static_cast<size_t>(nq) * 4 + 255) / 256) * 256;
  double* partial = reinterpret_cast<double*>(s + perm_bytes);
  unsigned char* sort_scratch = s + perm_bytes + sizeof(double) * p.partial_doubles;
  cudaError_t e = mixed_sort_queries(q, nq, perm, sort_scratch, mixed_sort_scratch_bytes(nq),
                                     stream);
  if (e != cudaSuccess) return e;
  return mixed_forward_sorted(m, q, perm, nq, w, p, p.nsplit > 1 ? partial : nullptr, stats, err,
                              stream);
}

// ---- batched meshes -------------------------------------------------------
// Many meshes with their own query sets, of uneven sizes, in one persistent
// launch. The meshes are concatenated (vertices, faces, queries); faces and
// queries are Morton-ordered inside their own mesh by one radix sort each, on
// 64-bit keys (mesh id << 30 | 30-bit Morton code of the point in its mesh's
// box), so every mesh stays a contiguous segment. Each mesh is tiled on its
// own. The work is a list of items (mesh, block of Morton-ordered queries,
// range of that mesh's tiles) sized to ~target_pairs pairs and ordered largest
// first; a persistent grid takes items from one atomic counter, and every item
// writes its own slice of a partial-sum array, which a finishing kernel adds up
// per query in chunk order. The schedule is dynamic, the result is not: no slot
// is written twice and every sum runs in a fixed order.
struct BatchDevice {
  int64_t* F = nullptr;           // total_nf x 3, global vertex indices
  int32_t* face_mesh = nullptr;   // total_nf
  int32_t* query_mesh = nullptr;  // total_nq (original order == sorted segment order)
  int64_t* tile_first = nullptr;  // total_tiles: sorted position of the tile's first face
  int32_t* tile_count = nullptr;  // total_tiles
  double* tri = nullptr;          // 9 x ldt soup built from V and F
  unsigned long long* fbox = nullptr;  // nmesh x 6
  unsigned long long* qbox = nullptr;  // nmesh x 6
  uint64_t *fkeys_in = nullptr, *fkeys_out = nullptr;
  uint32_t *fvals_in = nullptr, *fvals_out = nullptr;
  uint64_t *qkeys_in = nullptr, *qkeys_out = nullptr;
  uint32_t *qvals_in = nullptr, *perm = nullptr;
  void* sort_temp = nullptr;
  size_t sort_temp_bytes = 0;
  MixedMesh mesh;                 // all tiles of all meshes
  BatchItem* items = nullptr;
  BatchMeshInfo* info = nullptr;  // nmesh
  unsigned int* counter = nullptr;
  double* partial = nullptr;
};

namespace {

__global__ void soup_from_indexed_kernel(const double* __restrict__ V,
                                         const int64_t* __restrict__ F, int64_t nf, int64_t ld,
                                         double* __restrict__ tri) {
  const int64_t f = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (f >= nf) return;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const int64_t v = F[3 * f + c];
#pragma unroll
    for (int x = 0; x < 3; ++x) tri[(3 * c + x) * ld + f] = V[3 * v + x];
  }
}

__global__ void batch_bbox_init_kernel(unsigned long long* box, int64_t nmesh) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < nmesh * 6) box[i] = (i % 6) < 3 ? ~0ull : 0ull;
}

__device__ __forceinline__ void point_of(const double* data, int64_t ld, int64_t i, bool centroid,
                                         double p[3]) {
#pragma unroll
  for (int x = 0; x < 3; ++x)
    p[x] = centroid ? (data[x * ld + i] + data[(3 + x) * ld + i] + data[(6 + x) * ld + i]) *
                          (1.0 / 3.0)
                    : data[3 * i + x];
}

// Per-mesh boxes: each thread scans 16 consecutive points (meshes are
// contiguous, so a run rarely changes mesh), a warp whose lanes all stayed in
// one mesh combines before its one set of atomics.
template <bool CENTROIDS>
__global__ void batch_bbox_kernel(const double* __restrict__ data, int64_t ld, int64_t n,
                                  const int32_t* __restrict__ mesh_of,
                                  unsigned long long* box) {
  constexpr int kRun = 16;
  const int64_t begin = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) * kRun;
  const int64_t end = min(n, begin + kRun);
  int cur = begin < n ? mesh_of[begin] : -1;
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  auto flush = [&](int m) {
    if (m < 0 || !isfinite(lo[0])) return;
    for (int x = 0; x < 3; ++x) {
      atomicMin(&box[6 * m + x], ordered_key(lo[x]));
      atomicMax(&box[6 * m + 3 + x], ordered_key(hi[x]));
    }
  };
  for (int64_t i = begin; i < end; ++i) {
    const int m = mesh_of[i];
    if (m != cur) {
      flush(cur);
      cur = m;
      for (int x = 0; x < 3; ++x) {
        lo[x] = INFINITY;
        hi[x] = -INFINITY;
      }
    }
    double p[3];
    point_of(data, ld, i, CENTROIDS, p);
    for (int x = 0; x < 3; ++x) {
      lo[x] = fmin(lo[x], p[x]);
      hi[x] = fmax(hi[x], p[x]);
    }
  }
  const int lead = __shfl_sync(0xffffffffu, cur, 0);
  if (__all_sync(0xffffffffu, cur == lead)) {
    for (int x = 0; x < 3; ++x) {
      lo[x] = warp_min(lo[x]);
      hi[x] = warp_max(hi[x]);
    }
    if ((threadIdx.x & 31) == 0) flush(cur);
  } else {
    flush(cur);
  }
}

template <bool CENTROIDS>
__global__ void batch_morton_kernel(const double* __restrict__ data, int64_t ld, int64_t n,
                                    const int32_t* __restrict__ mesh_of,
                                    const unsigned long long* __restrict__ box,
                                    uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double p[3];
  point_of(data, ld, i, CENTROIDS, p);
  const int m = mesh_of[i];
  keys[i] = (static_cast<uint64_t>(m) << 30) | morton30(p, box + 6 * m);
  vals[i] = static_cast<uint32_t>(i);
}

struct BatchArgs {
  const unsigned char* tiles;
  const double* tri64;
  int64_t ld64;
  const double* q;
  const uint32_t* perm;
  const BatchItem* items;
  int64_t n_items;
  unsigned int* counter;
  double* partial;
  unsigned long long* stats;
  int* err;
};

template <int THREADS, int QPT, int STAGES, bool HALF>
__global__ void __launch_bounds__(THREADS, QPT == 1 ? 6 : (QPT == 2 ? 4 : 3))
    batch_forward_kernel(const BatchArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* ring = smem_raw;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + STAGES * kTileBytes);
  // Two face-pair transposed tiles (this CTA's g-th tile uses tbuf[g & 1]).
  float* tbuf = reinterpret_cast<float*>(smem_raw + STAGES * kTileBytes + 8 * STAGES);
  __shared__ int64_t s_item;
  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(&full[s], 1);
    fence_barrier_init();
  }
  int64_t gt = 0;  // tiles consumed by this CTA so far: ring slot and phase
  unsigned refined = 0, careful_tiles = 0;
  bool failed = false;
  for (;;) {
    __syncthreads();  // everyone is done with the previous item and its tiles
    if (tid == 0) s_item = static_cast<int64_t>(atomicAdd(a.counter, 1u));
    __syncthreads();
    const int64_t item = s_item;
    if (item >= a.n_items) break;
    const BatchItem it = a.items[item];
    double ox[QPT], oy[QPT], oz[QPT];
    int64_t qidx[QPT];
#pragma unroll
    for (int k = 0; k < QPT; ++k) {
      const int64_t off = k * THREADS + tid;
      qidx[k] = off < it.q_count ? static_cast<int64_t>(a.perm[it.q_begin + off]) : -1;
      const int64_t i = qidx[k] >= 0 ? qidx[k] : static_cast<int64_t>(a.perm[it.q_begin]);
      ox[k] = a.q[3 * i];
      oy[k] = a.q[3 * i + 1];
      oz[k] = a.q[3 * i + 2];
    }
    float hi[QPT], lo[QPT];
    double s64[QPT];
#pragma unroll
    for (int k = 0; k < QPT; ++k) {
      hi[k] = lo[k] = 0.f;
      s64[k] = 0.0;
    }
    const int nt = it.t_count;
    auto issue = [&](int u) {
      const int slot = static_cast<int>((gt + u) % STAGES);
      mbar_arrive_expect_tx(&full[slot], kTileBytes);
      bulk_g2s(ring + slot * kTileBytes, a.tiles + (it.t_begin + u) * kTileBytes, kTileBytes,
               &full[slot]);
    };
    int issued = 0;
    if (tid == 0)
      for (; issued < min(STAGES, nt); ++issued) issue(issued);
    int u = 0;
    for (; u < nt; ++u) {
      const int slot = static_cast<int>((gt + u) % STAGES);
      const bool landed =
          mbar_wait(&full[slot], static_cast<uint32_t>(((gt + u) / STAGES) & 1), a.err);
      float* tb = tbuf + ((gt + u) & 1) * (kTileTransposedBytes / 4);
      // tbuf[g & 1] was last read for tile g - 2, finished by every thread before
      // the barrier of tile g - 1 (or of the item boundary).
      if (landed) transpose_tile(ring + slot * kTileBytes, tb, tid, THREADS);
      if (!__syncthreads_and(landed)) {
        failed = true;
        break;
      }
      if (tid == 0 && u >= 1 && issued < nt) issue(issued++);
      mixed_tile_pairs<QPT, HALF>(ring + slot * kTileBytes, tb, (it.t_begin + u) * kTileFaces,
                                  a.tri64,
                            a.ld64, ox, oy, oz, qidx, hi, lo, s64, refined, careful_tiles);
    }
    if (failed) {
      if (tid == 0)
        for (int w = u; w < issued; ++w)
          mbar_wait(&full[(gt + w) % STAGES], static_cast<uint32_t>(((gt + w) / STAGES) & 1),
                    nullptr);
      break;
    }
    gt += nt;
#pragma unroll
    for (int k = 0; k < QPT; ++k) {
      const int64_t off = k * THREADS + tid;
      if (off >= it.q_count) continue;
      a.partial[it.p_base + off] =
          static_cast<double>(hi[k]) + static_cast<double>(lo[k]) + s64[k];
    }
  }
  __syncthreads();
  if (a.stats) {
    unsigned r = refined;
    for (int off = 16; off; off >>= 1) r += __shfl_xor_sync(0xffffffffu, r, off);
    if ((tid & 31) == 0) {
      atomicAdd(&a.stats[0], static_cast<unsigned long long>(r));
      atomicAdd(&a.stats[1], static_cast<unsigned long long>(careful_tiles));
    }
  }
}

// W[perm[s]] = (sum over the mesh's tile chunks, in order) / (2 pi).
__global__ void batch_finish_kernel(const double* __restrict__ partial,
                                    const BatchMeshInfo* __restrict__ info,
                                    const int32_t* __restrict__ query_mesh,
                                    const uint32_t* __restrict__ perm, int64_t total_nq,
                                    double* __restrict__ w) {
  const int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s >= total_nq) return;
  const BatchMeshInfo mi = info[query_mesh[s]];
  const int64_t local = s - mi.q_off;
  double sum = 0.0;
  for (int64_t c = 0; c < mi.nchunk; ++c) sum += partial[mi.p_off + c * mi.nq + local];
  w[perm[s]] = sum / kTwoPi;
}

template <int QPT, bool HALF>
cudaError_t launch_batch_variant(const BatchArgs& a, int grid, cudaStream_t stream) {
  constexpr int kThreads = 128, kStages = 4;
  auto kernel = batch_forward_kernel<kThreads, QPT, kStages, HALF>;
  const size_t smem = static_cast<size_t>(kStages) * kTileBytes + sizeof(uint64_t) * kStages +
                      2 * kTileTransposedBytes;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  kernel<<<grid, kThreads, smem, stream>>>(a);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError();
}

template <int QPT, bool HALF>
int batch_grid(int sms, int ctas_per_sm) {
  constexpr int kThreads = 128, kStages = 4;
  const size_t smem = static_cast<size_t>(kStages) * kTileBytes + sizeof(uint64_t) * kStages +
                      2 * kTileTransposedBytes;
  int per_sm = 0;
  cudaFuncSetAttribute(batch_forward_kernel<kThreads, QPT, kStages, HALF>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm,
                                                batch_forward_kernel<kThreads, QPT, kStages, HALF>,
                                                kThreads, smem);
  if (ctas_per_sm > 0) per_sm = std::min(per_sm, ctas_per_sm);
  return std::max(1, per_sm) * std::max(1, sms);
}

template <typename T>
cudaError_t dmalloc(T** p, size_t count) {
  return dev_malloc(reinterpret_cast<void**>(p), sizeof(T) * std::max<size_t>(count, 1));
}

}  // namespace

cudaError_t batch_create(BatchState* b, int64_t nmesh, const int64_t* nv, const int64_t* nf,
                         const int64_t* nq, const int64_t* F, const BatchPlan& plan, int sms) {
  b->plan = plan;
  b->sms = sms;
  b->nmesh = nmesh;
  cudaGetDevice(&b->device);
  b->v_off.assign(nmesh + 1, 0);
  b->f_off.assign(nmesh + 1, 0);
  b->q_off.assign(nmesh + 1, 0);
  b->t_off.assign(nmesh + 1, 0);
  b->nv.assign(nv, nv + nmesh);
  b->nf.assign(nf, nf + nmesh);
  b->nq.assign(nq, nq + nmesh);
  b->ntile.assign(nmesh, 0);
  for (int64_t m = 0; m < nmesh; ++m) {
    b->ntile[m] = nf[m] > 0 ? (nf[m] + kTileFaces - 1) / kTileFaces : 0;
    b->v_off[m + 1] = b->v_off[m] + nv[m];
    b->f_off[m + 1] = b->f_off[m] + nf[m];
    b->q_off[m + 1] = b->q_off[m] + nq[m];
    b->t_off[m + 1] = b->t_off[m] + b->ntile[m];
  }
  b->total_nv = b->v_off[nmesh];
  b->total_nf = b->f_off[nmesh];
  b->total_nq = b->q_off[nmesh];
  b->total_tiles = b->t_off[nmesh];
  b->ldt = ((std::max<int64_t>(b->total_nf, 1) + 1) / 2) * 2;
  b->mesh_bits = 1;
  while ((int64_t(1) << b->mesh_bits) < nmesh) ++b->mesh_bits;

  // Work items and partial-sum layout.
  const int64_t per_block = int64_t(128) * plan.qpt;
  std::vector<BatchItem> items;
  std::vector<BatchMeshInfo> info(nmesh);
  int64_t p_off = 0;
  for (int64_t m = 0; m < nmesh; ++m) {
    const int64_t nt = b->ntile[m];
    int64_t chunk = nt;
    if (nt > 0) {
      const int64_t want = plan.target_pairs / (per_block * kTileFaces);
      chunk = std::max<int64_t>(1, std::min<int64_t>(nt, want));
      chunk = (nt + ((nt + chunk - 1) / chunk) - 1) / ((nt + chunk - 1) / chunk);  // even chunks
    }
    const int64_t nchunk = nt > 0 ? (nt + chunk - 1) / chunk : 0;
    info[m] = BatchMeshInfo{b->q_off[m], nq[m], p_off, nchunk};
    for (int64_t c = 0; c < nchunk; ++c) {
      const int64_t t0 = c * chunk, tn = std::min(chunk, nt - t0);
      for (int64_t q0 = 0; q0 < nq[m]; q0 += per_block) {
        BatchItem it;
        it.q_begin = b->q_off[m] + q0;
        it.t_begin = b->t_off[m] + t0;
        it.p_base = p_off + c * nq[m] + q0;
        it.q_count = static_cast<int32_t>(std::min(per_block, nq[m] - q0));
        it.t_count = static_cast<int32_t>(tn);
        items.push_back(it);
      }
    }
    p_off += nchunk * nq[m];
  }
  std::stable_sort(items.begin(), items.end(), [](const BatchItem& x, const BatchItem& y) {
    return int64_t(x.q_count) * x.t_count > int64_t(y.q_count) * y.t_count;
  });
  b->n_items = static_cast<int64_t>(items.size());
  b->total_partials = p_off;

  // Tile table and mesh ids.
  std::vector<int64_t> tile_first(std::max<int64_t>(b->total_tiles, 1));
  std::vector<int32_t> tile_count(std::max<int64_t>(b->total_tiles, 1));
  for (int64_t m = 0; m < nmesh; ++m)
    for (int64_t t = 0; t < b->ntile[m]; ++t) {
      tile_first[b->t_off[m] + t] = b->f_off[m] + t * kTileFaces;
      tile_count[b->t_off[m] + t] =
          static_cast<int32_t>(std::min<int64_t>(kTileFaces, nf[m] - t * kTileFaces));
    }
  std::vector<int32_t> face_mesh(std::max<int64_t>(b->total_nf, 1)),
      query_mesh(std::max<int64_t>(b->total_nq, 1));
  std::vector<int64_t> Fg(std::max<int64_t>(3 * b->total_nf, 1));
  for (int64_t m = 0; m < nmesh; ++m) {
    for (int64_t f = b->f_off[m]; f < b->f_off[m + 1]; ++f) {
      face_mesh[f] = static_cast<int32_t>(m);
      for (int c = 0; c < 3; ++c) Fg[3 * f + c] = F[3 * f + c] + b->v_off[m];
    }
    for (int64_t i = b->q_off[m]; i < b->q_off[m + 1]; ++i) query_mesh[i] = static_cast<int32_t>(m);
  }

  BatchDevice* d = new BatchDevice();
  b->dev = d;
  size_t tf = 0, tq = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tf, static_cast<uint64_t*>(nullptr),
                                  static_cast<uint64_t*>(nullptr), static_cast<uint32_t*>(nullptr),
                                  static_cast<uint32_t*>(nullptr),
                                  static_cast<int>(std::max<int64_t>(b->total_nf, 1)), 0,
                                  30 + b->mesh_bits);
  cub::DeviceRadixSort::SortPairs(nullptr, tq, static_cast<uint64_t*>(nullptr),
                                  static_cast<uint64_t*>(nullptr), static_cast<uint32_t*>(nullptr),
                                  static_cast<uint32_t*>(nullptr),
                                  static_cast<int>(std::max<int64_t>(b->total_nq, 1)), 0,
                                  30 + b->mesh_bits);
  d->sort_temp_bytes = std::max(tf, tq);
  const int64_t ld64 = std::max<int64_t>(b->total_tiles, 1) * kTileFaces;
  cudaError_t e;
  if ((e = dmalloc(&d->F, 3 * b->total_nf)) != cudaSuccess ||
      (e = dmalloc(&d->face_mesh, b->total_nf)) != cudaSuccess ||
      (e = dmalloc(&d->query_mesh, b->total_nq)) != cudaSuccess ||
      (e = dmalloc(&d->tile_first, b->total_tiles)) != cudaSuccess ||
      (e = dmalloc(&d->tile_count, b->total_tiles)) != cudaSuccess ||
      (e = dmalloc(&d->tri, 9 * b->ldt)) != cudaSuccess ||
      (e = dmalloc(&d->fbox, 6 * nmesh)) != cudaSuccess ||
      (e = dmalloc(&d->qbox, 6 * nmesh)) != cudaSuccess ||
      (e = dmalloc(&d->fkeys_in, b->total_nf)) != cudaSuccess ||
      (e = dmalloc(&d->fkeys_out, b->total_nf)) != cudaSuccess ||
      (e = dmalloc(&d->fvals_in, b->total_nf)) != cudaSuccess ||
      (e = dmalloc(&d->fvals_out, b->total_nf)) != cudaSuccess ||
      (e = dmalloc(&d->qkeys_in, b->total_nq)) != cudaSuccess ||
      (e = dmalloc(&d->qkeys_out, b->total_nq)) != cudaSuccess ||
      (e = dmalloc(&d->qvals_in, b->total_nq)) != cudaSuccess ||
      (e = dmalloc(&d->perm, b->total_nq)) != cudaSuccess ||
      (e = dev_malloc(&d->sort_temp, std::max<size_t>(d->sort_temp_bytes, 16))) != cudaSuccess ||
      (e = dmalloc(&d->mesh.tiles, static_cast<size_t>(std::max<int64_t>(b->total_tiles, 1)) *
                                       kTileBytes)) != cudaSuccess ||
      (e = dmalloc(&d->mesh.tri64, 9 * ld64)) != cudaSuccess ||
      (e = dmalloc(&d->mesh.face_of, ld64)) != cudaSuccess ||
      (e = dmalloc(&d->mesh.reuse, ld64)) != cudaSuccess ||
      (e = dmalloc(&d->items, b->n_items)) != cudaSuccess ||
      (e = dmalloc(&d->info, nmesh)) != cudaSuccess ||
      (e = dmalloc(&d->counter, 1)) != cudaSuccess ||
      (e = dmalloc(&d->partial, b->total_partials)) != cudaSuccess)
    return e;
  d->mesh.nf = b->total_nf;
  d->mesh.ntiles = b->total_tiles;
  d->mesh.ld64 = ld64;
  d->mesh.kappa = plan.kappa;
  if ((e = cudaMemcpy(d->F, Fg.data(), sizeof(int64_t) * Fg.size(), cudaMemcpyHostToDevice)) !=
          cudaSuccess ||
      (e = cudaMemcpy(d->face_mesh, face_mesh.data(), sizeof(int32_t) * face_mesh.size(),
                      cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(d->query_mesh, query_mesh.data(), sizeof(int32_t) * query_mesh.size(),
                      cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(d->tile_first, tile_first.data(), sizeof(int64_t) * tile_first.size(),
                      cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(d->tile_count, tile_count.data(), sizeof(int32_t) * tile_count.size(),
                      cudaMemcpyHostToDevice)) != cudaSuccess ||
      (items.size() && (e = cudaMemcpy(d->items, items.data(), sizeof(BatchItem) * items.size(),
                                       cudaMemcpyHostToDevice)) != cudaSuccess) ||
      (e = cudaMemcpy(d->info, info.data(), sizeof(BatchMeshInfo) * info.size(),
                      cudaMemcpyHostToDevice)) != cudaSuccess)
    return e;
  switch (plan.qpt) {
    case 1:
      b->grid = plan.tile_faces == kHalfFaces ? batch_grid<1, true>(sms, plan.ctas_per_sm)
                                              : batch_grid<1, false>(sms, plan.ctas_per_sm);
      break;
    case 4:
      b->grid = plan.tile_faces == kHalfFaces ? batch_grid<4, true>(sms, plan.ctas_per_sm)
                                              : batch_grid<4, false>(sms, plan.ctas_per_sm);
      break;
    default:
      b->grid = plan.tile_faces == kHalfFaces ? batch_grid<2, true>(sms, plan.ctas_per_sm)
                                              : batch_grid<2, false>(sms, plan.ctas_per_sm);
      break;
  }
  b->grid = static_cast<int>(std::min<int64_t>(b->grid, std::max<int64_t>(b->n_items, 1)));
  return cudaGetLastError();
}

void batch_destroy(BatchState* b) {
  BatchDevice* d = b->dev;
  if (!d) return;
  void* ptrs[] = {d->F, d->face_mesh, d->query_mesh, d->tile_first, d->tile_count, d->tri,
                  d->fbox, d->qbox, d->fkeys_in, d->fkeys_out, d->fvals_in, d->fvals_out,
                  d->qkeys_in, d->qkeys_out, d->qvals_in, d->perm, d->sort_temp,
                  d->mesh.tiles, d->mesh.tri64, d->mesh.face_of, d->mesh.reuse, d->items, d->info,
                  d->counter, d->partial};
  for (void* p : ptrs) cudaFree(p);
  delete d;
  b->dev = nullptr;
}

cudaError_t batch_forward(BatchState* b, const double* V, const double* q, double* w,
                          unsigned long long* stats, int* err, cudaStream_t stream) {
  BatchDevice* d = b->dev;
  const int th = 256;
  const int kbits = 30 + b->mesh_bits;
  cudaError_t e;
  if (b->total_nf > 0) {
    soup_from_indexed_kernel<<<static_cast<unsigned>(blocks_for(b->total_nf, th)), th, 0,
                               stream>>>(V, d->F, b->total_nf, b->ldt, d->tri);
    batch_bbox_init_kernel<<<static_cast<unsigned>(blocks_for(6 * b->nmesh, th)), th, 0,
                             stream>>>(d->fbox, b->nmesh);
    batch_bbox_kernel<true><<<static_cast<unsigned>(blocks_for((b->total_nf + 15) / 16, th)), th,
                              0, stream>>>(d->tri, b->ldt, b->total_nf, d->face_mesh, d->fbox);
    batch_morton_kernel<true><<<static_cast<unsigned>(blocks_for(b->total_nf, th)), th, 0,
                                stream>>>(d->tri, b->ldt, b->total_nf, d->face_mesh, d->fbox,
                                          d->fkeys_in, d->fvals_in);
    size_t tb = d->sort_temp_bytes;
    if ((e = cub::DeviceRadixSort::SortPairs(d->sort_temp, tb, d->fkeys_in, d->fkeys_out,
                                             d->fvals_in, d->fvals_out,
                                             static_cast<int>(b->total_nf), 0, kbits, stream)) !=
        cudaSuccess)
      return e;
    build_tiles_kernel<<<static_cast<unsigned>(b->total_tiles), kTileFaces, 0, stream>>>(
        d->tri, b->ldt, b->total_nf, d->fvals_out, b->plan.kappa, d->mesh.tiles, d->mesh.tri64,
        d->mesh.ld64, d->mesh.face_of, d->tile_first, d->tile_count, d->mesh.reuse);
    g_launches.fetch_add(5, std::memory_order_relaxed);
  }
  if (b->total_nq == 0) return cudaGetLastError();
  batch_bbox_init_kernel<<<static_cast<unsigned>(blocks_for(6 * b->nmesh, th)), th, 0, stream>>>(
      d->qbox, b->nmesh);
  batch_bbox_kernel<false><<<static_cast<unsigned>(blocks_for((b->total_nq + 15) / 16, th)), th,
                             0, stream>>>(q, 0, b->total_nq, d->query_mesh, d->qbox);
  batch_morton_kernel<false><<<static_cast<unsigned>(blocks_for(b->total_nq, th)), th, 0,
                               stream>>>(q, 0, b->total_nq, d->query_mesh, d->qbox, d->qkeys_in,
                                         d->qvals_in);
  size_t tb = d->sort_temp_bytes;
  if ((e = cub::DeviceRadixSort::SortPairs(d->sort_temp, tb, d->qkeys_in, d->qkeys_out,
                                           d->qvals_in, d->perm, static_cast<int>(b->total_nq), 0,
                                           kbits, stream)) != cudaSuccess)
    return e;
  g_launches.fetch_add(3, std::memory_order_relaxed);
  if ((e = cudaMemsetAsync(d->counter, 0, sizeof(unsigned int), stream)) != cudaSuccess) return e;
  BatchArgs a{d->mesh.tiles, d->mesh.tri64, d->mesh.ld64, q,     d->perm, d->items,
              b->n_items,    d->counter,    d->partial,   stats, err};
  if (b->n_items > 0) {
    const bool half = b->plan.tile_faces == kHalfFaces;
    switch (b->plan.qpt) {
      case 1:
        e = half ? launch_batch_variant<1, true>(a, b->grid, stream)
                 : launch_batch_variant<1, false>(a, b->grid, stream);
        break;
      case 4:
        e = half ? launch_batch_variant<4, true>(a, b->grid, stream)
                 : launch_batch_variant<4, false>(a, b->grid, stream);
        break;
      default:
        e = half ? launch_batch_variant<2, true>(a, b->grid, stream)
                 : launch_batch_variant<2, false>(a, b->grid, stream);
        break;
    }
    if (e != cudaSuccess) return e;
  }
  batch_finish_kernel<<<static_cast<unsigned>(blocks_for(b->total_nq, th)), th, 0, stream>>>(
      d->partial, d->info, d->query_mesh, d->perm, b->total_nq, w);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError();
}

size_t batch_morton_temp_bytes(int64_t n, int mesh_bits) {
  size_t bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, bytes, static_cast<uint64_t*>(nullptr),
                                  static_cast<uint64_t*>(nullptr), static_cast<uint32_t*>(nullptr),
                                  static_cast<uint32_t*>(nullptr),
                                  static_cast<int>(std::max<int64_t>(n, 1)), 0, 30 + mesh_bits);
  return bytes;
}

cudaError_t batch_morton_order(const double* pts, int64_t n, const int32_t* mesh_of,
                               int64_t nmesh, int mesh_bits, unsigned long long* box,
                               uint64_t* keys_in, uint64_t* keys_out, uint32_t* vals_in,
                               uint32_t* perm, void* temp, size_t temp_bytes,
                               cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  const int th = 256;
  batch_bbox_init_kernel<<<static_cast<unsigned>(blocks_for(6 * nmesh, th)), th, 0, stream>>>(
      box, nmesh);
  batch_bbox_kernel<false><<<static_cast<unsigned>(blocks_for((n + 15) / 16, th)), th, 0,
                             stream>>>(pts, 0, n, mesh_of, box);
  batch_morton_kernel<false><<<static_cast<unsigned>(blocks_for(n, th)), th, 0, stream>>>(
      pts, 0, n, mesh_of, box, keys_in, vals_in);
  g_launches.fetch_add(3, std::memory_order_relaxed);
  return cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys_in, keys_out, vals_in, perm,
                                         static_cast<int>(n), 0, 30 + mesh_bits, stream);
}

}  // namespace wn
