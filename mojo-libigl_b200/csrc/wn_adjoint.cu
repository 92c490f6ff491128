// Hand-written adjoint of the exact generalized winding number.
//
// Forward (lee101/mojo-libigl, src/capi.mojo:205-286): W(o) = sum_f Omega_f(o) / (4 pi) with
// Omega_f = 2 atan2(det, denom). For one face with a = A - o, b = B - o, c = C - o,
// la = |a| etc., and D_ab = la lb + a.b (likewise D_bc, D_ca), the solid angle's
// derivatives are (the boundary-variation formula of a flat triangle, each side
// integrated in closed form):
//   dOmega/dA = -[ (a x b) / (la D_ab) + (c x a) / (la D_ca) ]
//   dOmega/dB = -[ (a x b) / (lb D_ab) + (b x c) / (lb D_bc) ]
//   dOmega/dC = -[ (b x c) / (lc D_bc) + (c x a) / (lc D_ca) ]
//   dOmega/do = -(dOmega/dA + dOmega/dB + dOmega/dC)          (translation invariance)
// With ra = 1/la and W_ab = ra rb / (1 + (a.b) ra rb): 1/(la D_ab) = ra W_ab, 1/(lb D_ab) = rb W_ab.
// At a query on a vertex or on a side (la = 0 or D = 0) the derivative does not exist; such
// pairs contribute zero.
//
// Given dL/dW per query (g), the kernel returns dL/do per query and dL/d(corner) per face
// (9 values, the soup's SoA layout); a gather through a vertex -> (face, corner) list turns
// the latter into dL/dV. Nothing Q x F-sized is stored: every pair term is recomputed.
//
// Work split, deterministic, no floating-point atomics. Faces are cut into blocks of
// THREADS*FPT (each thread keeps FPT faces and their 9 gradient sums in registers), queries
// into groups. A CTA owns (face range r, query group g): it walks the face blocks of r; for
// each, it streams the queries of g through shared memory in chunks, every thread adds its
// faces' terms, and each query's dL/do share is reduced over the CTA in a fixed order (warp
// butterfly, then warps in index order) and added into dO_part[r][q], a row only this CTA
// touches. After the last chunk a block's face sums go to dF_part[g][corner][face]. Two
// finishing kernels add the partials over r and over g in index order.
#include <algorithm>
#include <cmath>
#include <vector>

#include "wn_adjoint.h"
#include "wn_batch.h"
#include "wn_common.cuh"
#include "wn_internal.h"
#include "wn_mixed.h"

namespace wn {
namespace {

constexpr double kInv4Pi = 0.079577471545947667884441881686257181;  // 1 / (4 pi)

// g * dOmega/d(A, B, C) of one pair in FP64 (see the file comment), added into gv[9]
// (corners A, B, C), and g * dOmega/do added into go[3]. Zero for padding faces and for
// pairs where the derivative does not exist; every factor is selected so that no
// inf * 0 can appear.
__device__ __forceinline__ void pair_grad_fp64(double ox, double oy, double oz, const double* v,
                                               double g, bool valid, double* gv, double* go) {
  const double ax = v[0] - ox, ay = v[1] - oy, az = v[2] - oz;
  const double bx = v[3] - ox, by = v[4] - oy, bz = v[5] - oz;
  const double cx = v[6] - ox, cy = v[7] - oy, cz = v[8] - oz;
  const double aa = ax * ax + ay * ay + az * az;
  const double bb = bx * bx + by * by + bz * bz;
  const double cc = cx * cx + cy * cy + cz * cz;
  const double ra = rsqrt(aa), rb = rsqrt(bb), rc = rsqrt(cc);
  const double rab = ra * rb, rbc = rb * rc, rca = rc * ra;
  const double dab = 1.0 + (ax * bx + ay * by + az * bz) * rab;
  const double dbc = 1.0 + (bx * cx + by * cy + bz * cz) * rbc;
  const double dca = 1.0 + (cx * ax + cy * ay + cz * az) * rca;
  const bool ok = valid && aa > 0.0 && bb > 0.0 && cc > 0.0 && dab > 0.0 && dbc > 0.0 &&
                  dca > 0.0;
  const double inv = ok ? g / (dab * dbc * dca) : 0.0;
  const double wab = ok ? rab * dbc * dca * inv : 0.0;
  const double wbc = ok ? rbc * dab * dca * inv : 0.0;
  const double wca = ok ? rca * dab * dbc * inv : 0.0;
  const double sa = ok ? ra : 0.0, sb = ok ? rb : 0.0, sc = ok ? rc : 0.0;
  const double xab0 = ay * bz - az * by, xab1 = az * bx - ax * bz, xab2 = ax * by - ay * bx;
  const double xbc0 = by * cz - bz * cy, xbc1 = bz * cx - bx * cz, xbc2 = bx * cy - by * cx;
  const double xca0 = cy * az - cz * ay, xca1 = cz * ax - cx * az, xca2 = cx * ay - cy * ax;
  const double kA1 = sa * wab, kA2 = sa * wca, kB1 = sb * wab, kB2 = sb * wbc;
  const double kC1 = sc * wbc, kC2 = sc * wca;
  gv[0] -= kA1 * xab0 + kA2 * xca0;
  gv[1] -= kA1 * xab1 + kA2 * xca1;
  gv[2] -= kA1 * xab2 + kA2 * xca2;
  gv[3] -= kB1 * xab0 + kB2 * xbc0;
  gv[4] -= kB1 * xab1 + kB2 * xbc1;
  gv[5] -= kB1 * xab2 + kB2 * xbc2;
  gv[6] -= kC1 * xbc0 + kC2 * xca0;
  gv[7] -= kC1 * xbc1 + kC2 * xca1;
  gv[8] -= kC1 * xbc2 + kC2 * xca2;
  const double sab = kA1 + kB1, sbc = kB2 + kC1, sca = kC2 + kA2;
  go[0] += sab * xab0 + sbc * xbc0 + sca * xca0;
  go[1] += sab * xab1 + sbc * xbc1 + sca * xca1;
  go[2] += sab * xab2 + sbc * xbc2 + sca * xca2;
}

struct AdjointArgs {
  const double* tri;  // 9 x ld
  int64_t ld, nf;
  const double* q;   // nq x 3
  const double* gw;  // nq
  int64_t nq;
  int64_t blocks_per_range;  // face blocks per face range (grid.x)
  int64_t queries_per_group;  // queries per group (grid.y)
  double* dO_part;  // [nranges][nq][3], zeroed before the launch
  double* dF_part;  // [ngroups][9][ld]
};

template <int THREADS, int FPT, int QC>
__global__ void __launch_bounds__(THREADS, 2) adjoint_fp64_kernel(const AdjointArgs a) {
  __shared__ double sq[QC][4];                 // x, y, z, g of the chunk's queries
  __shared__ double red[THREADS / 32][QC][3];  // per-warp dL/do shares
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int kBlockFaces = THREADS * FPT;
  const int64_t range = blockIdx.x, group = blockIdx.y;
  const int64_t nblocks = (a.nf + kBlockFaces - 1) / kBlockFaces;
  const int64_t b_begin = range * a.blocks_per_range;
  const int64_t b_end = min(nblocks, b_begin + a.blocks_per_range);
  const int64_t q_begin = group * a.queries_per_group;
  const int64_t q_end = min(a.nq, q_begin + a.queries_per_group);
  double* dO_row = a.dO_part + range * a.nq * 3;

  for (int64_t blk = b_begin; blk < b_end; ++blk) {
    double fv[FPT][9], acc[FPT][9];
    bool fvalid[FPT];
#pragma unroll
    for (int k = 0; k < FPT; ++k) {
      const int64_t f = blk * kBlockFaces + k * THREADS + tid;
      fvalid[k] = f < a.nf;
#pragma unroll
      for (int r = 0; r < 9; ++r) {
        fv[k][r] = fvalid[k] ? a.tri[r * a.ld + f] : 0.0;
        acc[k][r] = 0.0;
      }
    }
    for (int64_t c0 = q_begin; c0 < q_end; c0 += QC) {
      const int nc = static_cast<int>(q_end - c0 < QC ? q_end - c0 : QC);
      __syncthreads();  // previous chunk fully consumed
      if (tid < nc) {
        const int64_t qi = c0 + tid;
        sq[tid][0] = a.q[3 * qi];
        sq[tid][1] = a.q[3 * qi + 1];
        sq[tid][2] = a.q[3 * qi + 2];
        sq[tid][3] = a.gw[qi];
      }
      __syncthreads();
#pragma unroll 1
      for (int j = 0; j < nc; ++j) {
        const double ox = sq[j][0], oy = sq[j][1], oz = sq[j][2], g = sq[j][3];
        double go[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int k = 0; k < FPT; ++k) pair_grad_fp64(ox, oy, oz, fv[k], g, fvalid[k], acc[k], go);
        double dox = go[0], doy = go[1], doz = go[2];
        for (int off = 16; off; off >>= 1) {
          dox += __shfl_xor_sync(0xffffffffu, dox, off);
          doy += __shfl_xor_sync(0xffffffffu, doy, off);
          doz += __shfl_xor_sync(0xffffffffu, doz, off);
        }
        if (lane == 0) {
          red[warp][j][0] = dox;
          red[warp][j][1] = doy;
          red[warp][j][2] = doz;
        }
      }
      __syncthreads();
      for (int e = tid; e < nc * 3; e += THREADS) {
        const int j = e / 3, x = e % 3;
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < THREADS / 32; ++w) s += red[w][j][x];
        dO_row[(c0 + j) * 3 + x] += s;
      }
    }
#pragma unroll
    for (int k = 0; k < FPT; ++k) {
      const int64_t f = blk * kBlockFaces + k * THREADS + tid;
      if (!fvalid[k]) continue;
#pragma unroll
      for (int r = 0; r < 9; ++r) a.dF_part[(group * 9 + r) * a.ld + f] = acc[k][r];
    }
  }
}

// ---- mixed precision adjoint ---------------------------------------------
// Same decomposition over the prepared mesh of the mixed forward (wn_mixed.cu):
// 64-face tiles in Morton order with FP32 tile-local scaled coordinates, queries in
// Morton order. A face block is 4 tiles and a CTA has 4 warps: warp w keeps tile
// 4b + w, lane l its faces l and l + 32 as the two lanes of packed FP32x2
// arithmetic (sm_100 add/mul/fma .f32x2), so a query's far test against the tile
// is uniform over the warp. Far pairs are evaluated in FP32 in the tile's scaled
// frame; the tile's scale factor (derivatives scale as 1/length) is folded into the
// query's upstream gradient. A pair with a vertex closer than kappa * h_face is
// evaluated in FP64 from the sorted FP64 soup. Per-face sums are kept in FP32 over
// a few query chunks and in FP64 beyond; per-query sums over faces are reduced in a
// fixed order, FP32 shares of far pairs and FP64 shares of refined pairs (large
// near-surface terms cancel there) added in FP64.
//
// Per far pair, with a = A - o, e1 = B - A, e2 = C - A, n = e1 x e2 from the face
// record and g the query's (scaled) upstream gradient:
//   |a|^2, a.e1, a.e2 give |b|^2, |c|^2, a.b, b.c, c.a (as in the forward);
//   la = |a|^2 rsqrt(|a|^2) ...; D_ab = la lb + a.b ...; 1/D by rcp;
//   a x b = a x e1, c x a = e2 x a, b x c = n - a x b - c x a;
//   k_A1 = g ra / D_ab, k_A2 = g ra / D_ca, k_B1 = g rb / D_ab, k_B2 = g rb / D_bc,
//   k_C1 = g rc / D_bc, k_C2 = g rc / D_ca;
//   -g dOmega/dA = k_A1 (a x b) + k_A2 (c x a), -g dOmega/dB = k_B1 (a x b) + k_B2 (b x c),
//   -g dOmega/dC = k_C1 (b x c) + k_C2 (c x a),
//   g dOmega/do = (k_A1 + k_B1)(a x b) + (k_B2 + k_C1)(b x c) + (k_C2 + k_A2)(c x a):
// 83 FP32 operations (as 42 packed instructions per face pair) and 6 MUFU per pair.
struct MixedAdjointArgs {
  const unsigned char* tiles;
  int64_t ntiles;
  const double* tri64;  // sorted FP64 soup, 9 x ld64
  int64_t ld64;
  const double4* qs;      // nq queries in Morton order: x, y, z, g
  int64_t nq;
  int64_t blocks_per_range;   // 4-tile blocks per range (grid.x)
  int64_t queries_per_group;  // sorted query positions per group (grid.y)
  double* dO_part;  // [nranges][nq][3] by sorted position, zeroed before the launch
  double* dF_part;  // [ngroups][9][ld64] by sorted slot
};

// Queries in Morton order with their upstream gradient: xyz and g as one double4.
__global__ void gather_sorted_queries_kernel(const double* __restrict__ q,
                                             const double* __restrict__ gw,
                                             const uint32_t* __restrict__ perm, int64_t nq,
                                             double4* __restrict__ qs) {
  const int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s >= nq) return;
  const int64_t i = perm[s];
  qs[s] = make_double4(q[3 * i], q[3 * i + 1], q[3 * i + 2], gw[i]);
}

// Shared-memory layout of adjoint_faces_kernel (dynamic, QC queries per chunk).
constexpr int kFaThreads = 128;          // four warps, one 64-face tile each
constexpr int kFaTiles = kFaThreads / 32;
constexpr int kFaRow = kFaThreads + 4;   // padded row of per-thread dL/do shares
constexpr int kFaQc = 16;                // queries per chunk (4 CTAs per SM fit the smem)
constexpr int kFaFlushChunks = 4;        // FP32 face sums go to FP64 every 64 queries
constexpr int kFaFlushQueries = kFaFlushChunks * kFaQc;
static_assert(kFaThreads == 2 * kTileFaces, "two faces per thread cover a tile per warp");

template <int QC>
struct FaceAdjSmem {
  float dO32[QC * 3][kFaRow];         // per-thread FP32 dL/do shares, row 3*query + axis
  double acc64[18][kFaThreads];       // per-face FP64 sums (thread-private columns)
  double red64[kFaTiles][QC][3];      // per-warp FP64 shares of refined pairs
  double dsum[QC * 3];                // the chunk's dL/do sums before they go to global
  double4 q64[QC];                    // FP64 query and g (refinement)
  // Per (query, tile), as ready-made FP32x2 operands (both lanes alike): minus the
  // query in the tile's scaled frame, g * scale and its negation:
  // (-x, -x, -y, -y), (-z, -z, gs, gs), (-gs, -gs, 0, 0).
  float4 frame[QC][kFaTiles][3];
  int flag[QC][kFaTiles];             // 0: far, 1: careful (near test), 2: skip
  TileHeader th[kFaTiles];
};

// One refined (near) pair in FP64: g * dOmega into the face's FP64 sums in shared
// memory (thread-private column) and into go. Kept out of line: it is rare, and
// inlined it would raise the register count of the whole FP32 loop.
__device__ __noinline__ void refine_pair_grad(const double* __restrict__ tri64, int64_t ld64,
                                              int64_t slot, double4 o, double* acc_col,
                                              int stride, double* go) {
  double v[9], gv[9];
#pragma unroll
  for (int r = 0; r < 9; ++r) {
    v[r] = tri64[r * ld64 + slot];
    gv[r] = 0.0;
  }
  pair_grad_fp64(o.x, o.y, o.z, v, o.w, true, gv, go);
#pragma unroll
  for (int r = 0; r < 9; ++r) acc_col[r * stride] += gv[r];
}

__device__ __forceinline__ float2 f2(float x) { return make_float2(x, x); }
// Lane k of a float2 (k a compile-time constant after unrolling).
__device__ __forceinline__ float& lane_ref(float2& v, int k) { return k == 0 ? v.x : v.y; }
__device__ __forceinline__ float2 rsqrt2(float2 v) {
  float2 r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r.x) : "f"(v.x));
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r.y) : "f"(v.y));
  return r;
}
__device__ __forceinline__ float2 rcp2(float2 v) {
  float2 r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r.x) : "f"(v.x));
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r.y) : "f"(v.y));
  return r;
}
// u x v component u1 v2 - u2 v1 as one multiply and one FMA (packed).
__device__ __forceinline__ float2 cross_c(float2 u1, float2 v2, float2 u2, float2 v1) {
  return __ffma2_rn(u1, v2, __fmul2_rn(make_float2(-u2.x, -u2.y), v1));
}

// One query against this thread's two faces (the two lanes of every float2): adds
// -g dOmega/d(A, B, C) into acc and returns g dOmega/do in d. fr: the query's
// frame operands (see FaceAdjSmem::frame); fnn = -n. Every operand is a whole
// FP32x2 pair and no sign is flipped per pair: -a comes from one packed multiply,
// -(b x c) = a x b + c x a - n, and the two coefficients of b x c are formed with
// -g. With CAREFUL, a lane whose face has a vertex closer than sqrt(thr) takes
// g = 0 (and unit squared lengths, so every term is finite and zero); bit k of
// the result flags lane k.
template <bool CAREFUL>
__device__ __forceinline__ unsigned face_pair_terms(const float4 (&fr)[3], const float2 (&fa)[3],
                                                    const float2 (&fe1)[3], const float2 (&fe2)[3],
                                                    const float2 (&fnn)[3], const float2 (&fg)[3],
                                                    float thr0, float thr1, float2 (&acc)[9],
                                                    float2 (&d)[3]) {
  const float4 f0 = fr[0], f1 = fr[1], f2v = fr[2];
  const float2 ax = __fadd2_rn(fa[0], make_float2(f0.x, f0.y));
  const float2 ay = __fadd2_rn(fa[1], make_float2(f0.z, f0.w));
  const float2 az = __fadd2_rn(fa[2], make_float2(f1.x, f1.y));
  float2 g2 = make_float2(f1.z, f1.w), ng2 = make_float2(f2v.x, f2v.y);
  const float2 m1 = f2(-1.f), two = f2(2.f);
  float2 aa = __ffma2_rn(ax, ax, __ffma2_rn(ay, ay, __fmul2_rn(az, az)));
  const float2 s1 = __ffma2_rn(ax, fe1[0], __ffma2_rn(ay, fe1[1], __fmul2_rn(az, fe1[2])));
  const float2 s2 = __ffma2_rn(ax, fe2[0], __ffma2_rn(ay, fe2[1], __fmul2_rn(az, fe2[2])));
  const float2 ab = __fadd2_rn(aa, s1), ca = __fadd2_rn(aa, s2);
  float2 bb = __ffma2_rn(two, s1, __fadd2_rn(aa, fg[0]));
  float2 cc = __ffma2_rn(two, s2, __fadd2_rn(aa, fg[1]));
  const float2 bc = __fadd2_rn(ab, __fadd2_rn(s2, fg[2]));
  unsigned nb = 0u;
  if constexpr (CAREFUL) {
    const bool n0 = fminf(aa.x, fminf(bb.x, cc.x)) < thr0;
    const bool n1 = fminf(aa.y, fminf(bb.y, cc.y)) < thr1;
    nb = (n0 ? 1u : 0u) | (n1 ? 2u : 0u);
    g2 = make_float2(n0 ? 0.f : g2.x, n1 ? 0.f : g2.y);
    ng2 = make_float2(n0 ? 0.f : ng2.x, n1 ? 0.f : ng2.y);
    aa = make_float2(n0 ? 1.f : aa.x, n1 ? 1.f : aa.y);
    bb = make_float2(n0 ? 1.f : bb.x, n1 ? 1.f : bb.y);
    cc = make_float2(n0 ? 1.f : cc.x, n1 ? 1.f : cc.y);
  }
  const float2 ra = rsqrt2(aa), rb = rsqrt2(bb), rc = rsqrt2(cc);
  const float2 la = __fmul2_rn(aa, ra), lb = __fmul2_rn(bb, rb), lc = __fmul2_rn(cc, rc);
  const float2 iab = rcp2(__ffma2_rn(la, lb, ab));
  const float2 ibc = rcp2(__ffma2_rn(lb, lc, bc));
  const float2 ica = rcp2(__ffma2_rn(lc, la, ca));
  const float2 gab = __fmul2_rn(g2, iab), gca = __fmul2_rn(g2, ica);
  const float2 ngbc = __fmul2_rn(ng2, ibc);
  const float2 kA1 = __fmul2_rn(ra, gab), kA2 = __fmul2_rn(ra, gca);
  const float2 kB1 = __fmul2_rn(rb, gab), nkB2 = __fmul2_rn(rb, ngbc);
  const float2 nkC1 = __fmul2_rn(rc, ngbc), kC2 = __fmul2_rn(rc, gca);
  // a x b = a x e1 and c x a = e2 x a with -a; -(b x c) = a x b + c x a - n.
  const float2 nax = __fmul2_rn(ax, m1), nay = __fmul2_rn(ay, m1), naz = __fmul2_rn(az, m1);
  const float2 xab0 = __ffma2_rn(ay, fe1[2], __fmul2_rn(naz, fe1[1]));
  const float2 xab1 = __ffma2_rn(az, fe1[0], __fmul2_rn(nax, fe1[2]));
  const float2 xab2 = __ffma2_rn(ax, fe1[1], __fmul2_rn(nay, fe1[0]));
  const float2 xca0 = __ffma2_rn(fe2[1], az, __fmul2_rn(fe2[2], nay));
  const float2 xca1 = __ffma2_rn(fe2[2], ax, __fmul2_rn(fe2[0], naz));
  const float2 xca2 = __ffma2_rn(fe2[0], ay, __fmul2_rn(fe2[1], nax));
  const float2 nxbc0 = __fadd2_rn(__fadd2_rn(xab0, xca0), fnn[0]);
  const float2 nxbc1 = __fadd2_rn(__fadd2_rn(xab1, xca1), fnn[1]);
  const float2 nxbc2 = __fadd2_rn(__fadd2_rn(xab2, xca2), fnn[2]);
  acc[0] = __ffma2_rn(kA1, xab0, __ffma2_rn(kA2, xca0, acc[0]));
  acc[1] = __ffma2_rn(kA1, xab1, __ffma2_rn(kA2, xca1, acc[1]));
  acc[2] = __ffma2_rn(kA1, xab2, __ffma2_rn(kA2, xca2, acc[2]));
  acc[3] = __ffma2_rn(kB1, xab0, __ffma2_rn(nkB2, nxbc0, acc[3]));
  acc[4] = __ffma2_rn(kB1, xab1, __ffma2_rn(nkB2, nxbc1, acc[4]));
  acc[5] = __ffma2_rn(kB1, xab2, __ffma2_rn(nkB2, nxbc2, acc[5]));
  acc[6] = __ffma2_rn(nkC1, nxbc0, __ffma2_rn(kC2, xca0, acc[6]));
  acc[7] = __ffma2_rn(nkC1, nxbc1, __ffma2_rn(kC2, xca1, acc[7]));
  acc[8] = __ffma2_rn(nkC1, nxbc2, __ffma2_rn(kC2, xca2, acc[8]));
  const float2 sab = __fadd2_rn(kA1, kB1), nsbc = __fadd2_rn(nkB2, nkC1);
  const float2 sca = __fadd2_rn(kC2, kA2);
  d[0] = __ffma2_rn(sab, xab0, __ffma2_rn(nsbc, nxbc0, __fmul2_rn(sca, xca0)));
  d[1] = __ffma2_rn(sab, xab1, __ffma2_rn(nsbc, nxbc1, __fmul2_rn(sca, xca1)));
  d[2] = __ffma2_rn(sab, xab2, __ffma2_rn(nsbc, nxbc2, __fmul2_rn(sca, xca2)));
  return nb;
}

template <int QC>
__global__ void __launch_bounds__(kFaThreads, 4) adjoint_faces_kernel(const MixedAdjointArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  auto& sm = *reinterpret_cast<FaceAdjSmem<QC>*>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t nblocks = (a.ntiles + kFaTiles - 1) / kFaTiles;
  const int64_t range = blockIdx.x, group = blockIdx.y;
  const int64_t b_begin = range * a.blocks_per_range;
  const int64_t b_end = min(nblocks, b_begin + a.blocks_per_range);
  const int64_t q_begin = group * a.queries_per_group;
  const int64_t q_end = min(a.nq, q_begin + a.queries_per_group);
  double* dO_row = a.dO_part + range * a.nq * 3;

  for (int64_t blk = b_begin; blk < b_end; ++blk) {
    __syncthreads();  // previous block's shared data fully consumed
    if (tid < kFaTiles) {
      const int64_t t = blk * kFaTiles + tid;
      if (t < a.ntiles) {
        sm.th[tid] = *reinterpret_cast<const TileHeader*>(a.tiles + t * kTileBytes);
      } else {
        TileHeader empty{};
        empty.far_r2 = 0.0;  // every query is "far" from a missing tile
        empty.scale = 1.0;
        sm.th[tid] = empty;
      }
    }
    // This warp's tile; lane k of every float2 is face lane + 32 k. Padding faces get
    // a corner far away and zero edges: every term they give is exactly zero.
    const int64_t t = blk * kFaTiles + warp;
    const bool tile_ok = t < a.ntiles;
    const unsigned char* rec = a.tiles + (tile_ok ? t : 0) * kTileBytes;
    const int n = tile_ok ? reinterpret_cast<const TileHeader*>(rec)->n : 0;
    const float* thr_rec = reinterpret_cast<const float*>(rec + kTileHeaderBytes) + 16 * lane + 15;
    float4 r[2][4];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int j = lane + 32 * k;
      const float4* fr = reinterpret_cast<const float4*>(rec + kTileHeaderBytes) + 4 * j;
      r[k][0] = make_float4(1e18f, 1e18f, 1e18f, 0.f);
      r[k][1] = r[k][2] = make_float4(0.f, 0.f, 0.f, 0.f);
      r[k][3] = make_float4(0.f, 0.f, 0.f, -1.f);
      if (j < n) {
        r[k][0] = fr[0];
        r[k][1] = fr[1];
        r[k][2] = fr[2];
        r[k][3] = fr[3];
      }
    }
    // Each field of the two faces as one FP32x2 value, built whole (fnn = -n).
    auto pr = [&](float a, float b) { return make_float2(a, b); };
    const float2 fa[3] = {pr(r[0][0].x, r[1][0].x), pr(r[0][0].y, r[1][0].y),
                          pr(r[0][0].z, r[1][0].z)};
    const float2 fe1[3] = {pr(r[0][0].w, r[1][0].w), pr(r[0][1].x, r[1][1].x),
                           pr(r[0][1].y, r[1][1].y)};
    const float2 fe2[3] = {pr(r[0][1].z, r[1][1].z), pr(r[0][1].w, r[1][1].w),
                           pr(r[0][2].x, r[1][2].x)};
    const float2 fnn[3] = {pr(-r[0][2].y, -r[1][2].y), pr(-r[0][2].z, -r[1][2].z),
                           pr(-r[0][2].w, -r[1][2].w)};
    const float2 fg[3] = {pr(r[0][3].x, r[1][3].x), pr(r[0][3].y, r[1][3].y),
                          pr(r[0][3].z, r[1][3].z)};
    const int64_t slot0 = (tile_ok ? t : 0) * kTileFaces + lane;
#pragma unroll
    for (int r = 0; r < 18; ++r) sm.acc64[r][tid] = 0.0;
    float2 acc[9];
#pragma unroll
    for (int r = 0; r < 9; ++r) acc[r] = f2(0.f);

    int chunks = 0;
    for (int64_t c0 = q_begin; c0 < q_end; c0 += QC) {
      const int nc = static_cast<int>(q_end - c0 < QC ? q_end - c0 : QC);
      __syncthreads();  // previous chunk's shared data fully consumed (and the headers landed)
      for (int item = tid; item < QC * kFaTiles; item += kFaThreads) {
        const int jq = item / kFaTiles, tt = item % kFaTiles;
        if (jq < nc) {
          const double4 o = a.qs[c0 + jq];
          const TileHeader& th = sm.th[tt];
          const double dx = o.x - th.cx, dy = o.y - th.cy, dz = o.z - th.cz;
          const double d2 = dx * dx + dy * dy + dz * dz;
          // Beyond 2^40 tile radii the tile's terms are below 2^-80 of a near one and
          // squared FP32 distances could overflow: the tile is skipped for this query.
          const bool skip = d2 * th.scale * th.scale > 1.2089258196146292e24;
          const float lx = static_cast<float>(dx * th.scale);
          const float ly = static_cast<float>(dy * th.scale);
          const float lz = static_cast<float>(dz * th.scale);
          const float gs = static_cast<float>(o.w * th.scale);
          sm.frame[jq][tt][0] = make_float4(-lx, -lx, -ly, -ly);
          sm.frame[jq][tt][1] = make_float4(-lz, -lz, gs, gs);
          sm.frame[jq][tt][2] = make_float4(-gs, -gs, 0.f, 0.f);
          sm.flag[jq][tt] = skip ? 2 : (d2 >= th.far_r2 ? 0 : 1);
          if (tt == 0) sm.q64[jq] = o;
        }
      }
      for (int e = tid; e < kFaTiles * QC * 3; e += kFaThreads) (&sm.red64[0][0][0])[e] = 0.0;
      __syncthreads();
      static_assert(QC <= 32, "one mask bit per query of a chunk");
      unsigned near0 = 0u, near1 = 0u;  // bit jq: the pair (query jq, face k) is refined
      // This warp's far and careful queries of the chunk (flags of its tile), taken in
      // two branch-free loops; skipped queries only store zero shares.
      const int myflag = lane < nc ? sm.flag[lane][warp] : 2;
      const unsigned far_q = __ballot_sync(0xffffffffu, myflag == 0);
      const unsigned careful_q = __ballot_sync(0xffffffffu, myflag == 1);
      const unsigned skip_q = __ballot_sync(0xffffffffu, myflag == 2 && lane < nc);
#pragma unroll 1
      for (unsigned m = far_q; m; m &= m - 1u) {
        const int jq = __ffs(m) - 1;
        float2 d[3];
        face_pair_terms<false>(sm.frame[jq][warp], fa, fe1, fe2, fnn, fg, 0.f, 0.f, acc, d);
        sm.dO32[3 * jq][tid] = d[0].x + d[0].y;
        sm.dO32[3 * jq + 1][tid] = d[1].x + d[1].y;
        sm.dO32[3 * jq + 2][tid] = d[2].x + d[2].y;
      }
      if (careful_q) {
        // Careful visits: pairs with a vertex closer than kappa * h_face are refined
        // in FP64 below; their FP32 terms come out as zero here.
        const float thr0 = lane < n ? __ldg(thr_rec) : -1.f;  // padding: never near
        const float thr1 = lane + 32 < n ? __ldg(thr_rec + 16 * 32) : -1.f;
#pragma unroll 1
        for (unsigned m = careful_q; m; m &= m - 1u) {
          const int jq = __ffs(m) - 1;
          float2 d[3];
          const unsigned nb = face_pair_terms<true>(sm.frame[jq][warp], fa, fe1, fe2, fnn, fg,
                                                    thr0, thr1, acc, d);
          near0 |= (nb & 1u) << jq;
          near1 |= (nb >> 1) << jq;
          sm.dO32[3 * jq][tid] = d[0].x + d[0].y;
          sm.dO32[3 * jq + 1][tid] = d[1].x + d[1].y;
          sm.dO32[3 * jq + 2][tid] = d[2].x + d[2].y;
        }
      }
      for (unsigned m = skip_q; m; m &= m - 1u) {
        const int jq = __ffs(m) - 1;
        sm.dO32[3 * jq][tid] = 0.f;
        sm.dO32[3 * jq + 1][tid] = 0.f;
        sm.dO32[3 * jq + 2][tid] = 0.f;
      }
      // Near pairs in FP64, query by query with the warp's lanes in step; each
      // query's FP64 dL/do shares are reduced over the warp in a fixed order.
      for (unsigned pending = __reduce_or_sync(0xffffffffu, near0 | near1); pending;
           pending &= pending - 1u) {
        const int jq = __ffs(pending) - 1;
        double go[3] = {0.0, 0.0, 0.0};
        if ((near0 >> jq) & 1u)
          refine_pair_grad(a.tri64, a.ld64, slot0, sm.q64[jq], &sm.acc64[0][tid], kFaThreads, go);
        if ((near1 >> jq) & 1u)
          refine_pair_grad(a.tri64, a.ld64, slot0 + 32, sm.q64[jq], &sm.acc64[9][tid],
                           kFaThreads, go);
        for (int off = 16; off; off >>= 1) {
          go[0] += __shfl_xor_sync(0xffffffffu, go[0], off);
          go[1] += __shfl_xor_sync(0xffffffffu, go[1], off);
          go[2] += __shfl_xor_sync(0xffffffffu, go[2], off);
        }
        if (lane == 0) {
          sm.red64[warp][jq][0] = go[0];
          sm.red64[warp][jq][1] = go[1];
          sm.red64[warp][jq][2] = go[2];
        }
      }
      __syncthreads();
      // Each (query, axis) row of 128 FP32 shares is summed by 4 lanes (32 shares each,
      // in index order), the 4 partial sums by a fixed butterfly; the FP64 shares of
      // refined pairs are added in warp order. Loop bounds are uniform per warp.
      for (int base = 0; base + 8 * warp < QC * 3; base += kFaThreads / 4) {
        const int row = base + (tid >> 2), part = tid & 3;
        const float4* src = reinterpret_cast<const float4*>(&sm.dO32[row][32 * part]);
        float4 s4 = src[0];
#pragma unroll
        for (int i = 1; i < 8; ++i) {
          const float4 v = src[i];
          s4.x += v.x;
          s4.y += v.y;
          s4.z += v.z;
          s4.w += v.w;
        }
        float v = (s4.x + s4.y) + (s4.z + s4.w);
        v += __shfl_xor_sync(0xffffffffu, v, 1);
        v += __shfl_xor_sync(0xffffffffu, v, 2);
        if (part == 0 && row < nc * 3) {
          const int jq = row / 3, x = row % 3;
          double sum = static_cast<double>(v);
#pragma unroll
          for (int w = 0; w < kFaTiles; ++w) sum += sm.red64[w][jq][x];
          sm.dsum[row] = sum;
        }
      }
      // FP32 face sums (minus g dOmega/dX, scale folded in) into FP64 every few chunks.
      if (++chunks == kFaFlushChunks || c0 + QC >= q_end) {
        chunks = 0;
#pragma unroll
        for (int r = 0; r < 9; ++r) {
          sm.acc64[r][tid] -= static_cast<double>(acc[r].x);
          sm.acc64[9 + r][tid] -= static_cast<double>(acc[r].y);
          acc[r] = f2(0.f);
        }
      }
      __syncthreads();
      for (int e = tid; e < nc * 3; e += kFaThreads) dO_row[c0 * 3 + e] += sm.dsum[e];
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      if (lane + 32 * k >= n) continue;
#pragma unroll
      for (int r = 0; r < 9; ++r)
        a.dF_part[(group * 9 + r) * a.ld64 + slot0 + 32 * k] = sm.acc64[9 * k + r][tid];
    }
  }
}

// dq[perm[s]] = (1/4pi) sum_r dO_part[r][s] (sorted positions back to input order).
__global__ void finish_dq_sorted_kernel(const double* __restrict__ part, int64_t nranges,
                                        int64_t nq, const uint32_t* __restrict__ perm,
                                        double* __restrict__ dq) {
  const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= nq * 3) return;
  double s = 0.0;
  for (int64_t r = 0; r < nranges; ++r) s += part[r * nq * 3 + e];
  dq[3 * static_cast<int64_t>(perm[e / 3]) + e % 3] = s * kInv4Pi;
}

// dtri[row][face_of[slot]] = (1/4pi) sum_g dF_part[g][row][slot] (sorted slots to input faces).
__global__ void finish_dtri_sorted_kernel(const double* __restrict__ part, int64_t ngroups,
                                          int64_t ld64, const uint32_t* __restrict__ face_of,
                                          int64_t ld, double* __restrict__ dtri) {
  const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= 9 * ld64) return;
  const int64_t r = e / ld64, sl = e % ld64;
  const uint32_t f = face_of[sl];
  if (f == 0xffffffffu) return;
  double s = 0.0;
  for (int64_t g = 0; g < ngroups; ++g) s += part[(g * 9 + r) * ld64 + sl];
  dtri[r * ld + f] = s * kInv4Pi;
}

// ---- boundary-edge adjoint ------------------------------------------------
// For an indexed mesh the per-face terms above telescope. Write a face's
// derivative as a sum over its three directed sides P -> Q (p = P - o, q = Q - o,
// D = |p||q| + p.q):
//   side P -> Q adds  -(p x q)/(|p| D) to dOmega/dP  and  -(p x q)/(|q| D) to dOmega/dQ.
// The reversed side Q -> P of a neighbouring face adds exactly the negatives, so
// at both endpoints the two cancel. Summed over the mesh only the net boundary
// survives: every undirected edge {u, v} enters with multiplicity
// m = #(u -> v) - #(v -> u), and edges with m = 0 drop out. This kernel evaluates
// those edges (endpoints P, Q and m in a 7 x le SoA); its per-edge sums over the
// queries go to dedge (6 x le: dL/dP, dL/dQ) and the per-query sums over edges to dq.
// Same work split and fixed reduction order as adjoint_fp64_kernel.
struct EdgeAdjointArgs {
  const double* edges;  // 7 x le: Px, Py, Pz, Qx, Qy, Qz, m
  int64_t le, ne;
  const double* q;
  const double* gw;
  int64_t nq;
  int64_t blocks_per_range, queries_per_group;
  double* dO_part;  // [nranges][nq][3], zeroed
  double* dE_part;  // [ngroups][6][le]
};

template <int THREADS, int EPT, int QC>
__global__ void __launch_bounds__(THREADS, 2) adjoint_edges_kernel(const EdgeAdjointArgs a) {
  __shared__ double sq[QC][4];
  __shared__ double red[THREADS / 32][QC][3];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int kBlockEdges = THREADS * EPT;
  const int64_t nblocks = (a.ne + kBlockEdges - 1) / kBlockEdges;
  const int64_t range = blockIdx.x, group = blockIdx.y;
  const int64_t b_begin = range * a.blocks_per_range;
  const int64_t b_end = min(nblocks, b_begin + a.blocks_per_range);
  const int64_t q_begin = group * a.queries_per_group;
  const int64_t q_end = min(a.nq, q_begin + a.queries_per_group);
  double* dO_row = a.dO_part + range * a.nq * 3;
  for (int64_t blk = b_begin; blk < b_end; ++blk) {
    double ev[EPT][7], acc[EPT][6];
#pragma unroll
    for (int k = 0; k < EPT; ++k) {
      const int64_t e = blk * kBlockEdges + k * THREADS + tid;
      const bool valid = e < a.ne;
#pragma unroll
      for (int r = 0; r < 7; ++r) ev[k][r] = valid ? a.edges[r * a.le + e] : 0.0;
#pragma unroll
      for (int r = 0; r < 6; ++r) acc[k][r] = 0.0;
    }
    for (int64_t c0 = q_begin; c0 < q_end; c0 += QC) {
      const int nc = static_cast<int>(q_end - c0 < QC ? q_end - c0 : QC);
      __syncthreads();
      if (tid < nc) {
        const int64_t qi = c0 + tid;
        sq[tid][0] = a.q[3 * qi];
        sq[tid][1] = a.q[3 * qi + 1];
        sq[tid][2] = a.q[3 * qi + 2];
        sq[tid][3] = a.gw[qi];
      }
      __syncthreads();
#pragma unroll 1
      for (int j = 0; j < nc; ++j) {
        const double ox = sq[j][0], oy = sq[j][1], oz = sq[j][2], g = sq[j][3];
        double dox = 0.0, doy = 0.0, doz = 0.0;
#pragma unroll
        for (int k = 0; k < EPT; ++k) {
          const double px = ev[k][0] - ox, py = ev[k][1] - oy, pz = ev[k][2] - oz;
          const double qx = ev[k][3] - ox, qy = ev[k][4] - oy, qz = ev[k][5] - oz;
          const double pp = px * px + py * py + pz * pz;
          const double qq = qx * qx + qy * qy + qz * qz;
          const double rp = rsqrt(pp), rq = rsqrt(qq);
          const double rpq = rp * rq;
          const double d = 1.0 + (px * qx + py * qy + pz * qz) * rpq;
          // Zero for padding (m = 0) and where the derivative does not exist.
          const bool ok = ev[k][6] != 0.0 && pp > 0.0 && qq > 0.0 && d > 0.0;
          const double w = ok ? g * ev[k][6] * rpq / d : 0.0;
          const double cp = ok ? rp * w : 0.0, cq = ok ? rq * w : 0.0;
          const double x0 = py * qz - pz * qy, x1 = pz * qx - px * qz, x2 = px * qy - py * qx;
          acc[k][0] -= cp * x0;
          acc[k][1] -= cp * x1;
          acc[k][2] -= cp * x2;
          acc[k][3] -= cq * x0;
          acc[k][4] -= cq * x1;
          acc[k][5] -= cq * x2;
          const double c = cp + cq;
          dox += c * x0;
          doy += c * x1;
          doz += c * x2;
        }
        for (int off = 16; off; off >>= 1) {
          dox += __shfl_xor_sync(0xffffffffu, dox, off);
          doy += __shfl_xor_sync(0xffffffffu, doy, off);
          doz += __shfl_xor_sync(0xffffffffu, doz, off);
        }
        if (lane == 0) {
          red[warp][j][0] = dox;
          red[warp][j][1] = doy;
          red[warp][j][2] = doz;
        }
      }
      __syncthreads();
      for (int e = tid; e < nc * 3; e += THREADS) {
        const int j = e / 3, x = e % 3;
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < THREADS / 32; ++w) s += red[w][j][x];
        dO_row[(c0 + j) * 3 + x] += s;
      }
    }
#pragma unroll
    for (int k = 0; k < EPT; ++k) {
      const int64_t e = blk * kBlockEdges + k * THREADS + tid;
      if (e >= a.ne) continue;
#pragma unroll
      for (int r = 0; r < 6; ++r) a.dE_part[(group * 6 + r) * a.le + e] = acc[k][r];
    }
  }
}

// dedge[row][e] = (1/4pi) sum_g dE_part[g][row][e].
__global__ void finish_dedge_kernel(const double* __restrict__ part, int64_t ngroups, int64_t le,
                                    int64_t ne, double* __restrict__ dedge) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= 6 * ne) return;
  const int64_t r = i / ne, e = i % ne;
  double s = 0.0;
  for (int64_t g = 0; g < ngroups; ++g) s += part[(g * 6 + r) * le + e];
  dedge[r * le + e] = s * kInv4Pi;
}

// dq[q] = (1/4pi) sum_r dO_part[r][q] (r in index order).
__global__ void finish_dq_kernel(const double* __restrict__ part, int64_t nranges, int64_t nq,
                                 double* __restrict__ dq) {
  const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= nq * 3) return;
  double s = 0.0;
  for (int64_t r = 0; r < nranges; ++r) s += part[r * nq * 3 + e];
  dq[e] = s * kInv4Pi;
}

// dtri[row][f] = (1/4pi) sum_g dF_part[g][row][f] (g in index order).
__global__ void finish_dtri_kernel(const double* __restrict__ part, int64_t ngroups, int64_t ld,
                                   int64_t nf, double* __restrict__ dtri) {
  const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= 9 * nf) return;
  const int64_t r = e / nf, f = e % nf;
  double s = 0.0;
  for (int64_t g = 0; g < ngroups; ++g) s += part[(g * 9 + r) * ld + f];
  dtri[r * ld + f] = s * kInv4Pi;
}

// dV[v][x] = sum over the vertex's (face, corner) entries, in list order.
__global__ void gather_vertex_kernel(const double* __restrict__ dtri, int64_t ld, int corners,
                                     const int64_t* __restrict__ indptr,
                                     const int64_t* __restrict__ entries, int64_t nv,
                                     double* __restrict__ dV) {
  const int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int64_t e = indptr[v]; e < indptr[v + 1]; ++e) {
    const int64_t f = entries[e] / corners, c = entries[e] % corners;
    s0 += dtri[(3 * c) * ld + f];
    s1 += dtri[(3 * c + 1) * ld + f];
    s2 += dtri[(3 * c + 2) * ld + f];
  }
  dV[3 * v] = s0;
  dV[3 * v + 1] = s1;
  dV[3 * v + 2] = s2;
}

constexpr int kAdjThreads = 128, kAdjFpt = 2, kAdjQc = 64;

int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

}  // namespace

// Split nblocks element blocks into ranges (grid.x) and nq queries into groups
// (grid.y) so that the grid is a whole number of waves of `slots` resident CTAs.
AdjointPlan plan_waves(int64_t nblocks, int64_t nq, int64_t slots, int64_t qc) {
  AdjointPlan p;
  nblocks = std::max<int64_t>(1, nblocks);
  slots = std::max<int64_t>(1, slots);
  const int64_t nranges = std::min<int64_t>(nblocks, 16);
  p.blocks_per_range = cdiv(nblocks, nranges);
  p.nranges = cdiv(nblocks, p.blocks_per_range);
  const int64_t max_groups = std::max<int64_t>(1, std::min<int64_t>(cdiv(nq, qc), 65535));
  // Two whole waves: nranges * ngroups <= 2 * slots, as close to it as possible, so
  // that no wave runs nearly empty.
  const int64_t ngroups = std::max<int64_t>(1, std::min(max_groups, (2 * slots) / p.nranges));
  p.queries_per_group = cdiv(std::max<int64_t>(nq, 1), ngroups);
  p.ngroups = cdiv(std::max<int64_t>(nq, 1), p.queries_per_group);
  return p;
}

// Like plan_waves, but the split between face ranges and query groups balances the
// two partial arrays the split creates: nranges * nq * 3 doubles of dL/do partials
// against ngroups * elem_doubles of per-element partials (elem_doubles = 9 * ld for
// faces), for about two waves of `slots` resident CTAs.
AdjointPlan plan_balanced(int64_t nblocks, int64_t nq, int64_t slots, int64_t qc,
                          int64_t elem_doubles) {
  AdjointPlan p;
  nblocks = std::max<int64_t>(1, nblocks);
  nq = std::max<int64_t>(1, nq);
  const int64_t target = 2 * std::max<int64_t>(1, slots);
  const double r = std::sqrt(static_cast<double>(target) * static_cast<double>(elem_doubles) /
                             (3.0 * static_cast<double>(nq)));
  const int64_t nranges =
      std::max<int64_t>(1, std::min<int64_t>(std::min(nblocks, target), std::llround(r)));
  p.blocks_per_range = cdiv(nblocks, nranges);
  p.nranges = cdiv(nblocks, p.blocks_per_range);
  const int64_t max_groups = std::max<int64_t>(1, std::min<int64_t>(cdiv(nq, qc), 65535));
  const int64_t ngroups = std::max<int64_t>(1, std::min(max_groups, target / p.nranges));
  p.queries_per_group = cdiv(nq, ngroups);
  p.ngroups = cdiv(nq, p.queries_per_group);
  return p;
}

int resident_ctas(const void* kernel, int threads, size_t smem, int sms) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) !=
          cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  return per_sm * std::max(sms, 1);
}

AdjointPlan plan_adjoint(int64_t nf, int64_t nq, int sms) {
  const int slots = resident_ctas(
      reinterpret_cast<const void*>(adjoint_fp64_kernel<kAdjThreads, kAdjFpt, kAdjQc>),
      kAdjThreads, 0, sms);
  return plan_waves(cdiv(nf, kAdjThreads * kAdjFpt), nq, slots, kAdjQc);
}

size_t adjoint_scratch_bytes(const AdjointPlan& p, int64_t ld, int64_t nq) {
  // dO partials, dF partials, and the Morton-ordered (query, g) copy of the mixed path.
  return sizeof(double) * (static_cast<size_t>(p.nranges) * nq * 3 +
                           static_cast<size_t>(p.ngroups) * 9 * ld) +
         sizeof(double4) * static_cast<size_t>(std::max<int64_t>(nq, 1)) + 256;
}

cudaError_t adjoint_fp64(const AdjointPlan& p, const double* tri, int64_t ld, int64_t nf,
                         const double* q, int64_t nq, const double* gw, double* dq, double* dtri,
                         void* scratch, size_t scratch_bytes, cudaStream_t stream) {
  if (nq <= 0 || nf <= 0) {
    cudaError_t e = cudaSuccess;
    if (nq > 0) e = cudaMemsetAsync(dq, 0, sizeof(double) * 3 * nq, stream);
    if (e == cudaSuccess && nf > 0) e = cudaMemsetAsync(dtri, 0, sizeof(double) * 9 * ld, stream);
    return e;
  }
  if (scratch_bytes < adjoint_scratch_bytes(p, ld, nq)) return cudaErrorInvalidValue;
  double* dO_part = static_cast<double*>(scratch);
  double* dF_part = dO_part + static_cast<size_t>(p.nranges) * nq * 3;
  cudaError_t e =
      cudaMemsetAsync(dO_part, 0, sizeof(double) * static_cast<size_t>(p.nranges) * nq * 3, stream);
  if (e != cudaSuccess) return e;
  AdjointArgs a{tri, ld, nf, q, gw, nq, p.blocks_per_range, p.queries_per_group, dO_part, dF_part};
  adjoint_fp64_kernel<kAdjThreads, kAdjFpt, kAdjQc>
      <<<dim3(static_cast<unsigned>(p.nranges), static_cast<unsigned>(p.ngroups)), kAdjThreads, 0,
         stream>>>(a);
  finish_dq_kernel<<<static_cast<unsigned>(cdiv(nq * 3, 256)), 256, 0, stream>>>(dO_part, p.nranges,
                                                                               nq, dq);
  finish_dtri_kernel<<<static_cast<unsigned>(cdiv(9 * nf, 256)), 256, 0, stream>>>(
      dF_part, p.ngroups, ld, nf, dtri);
  g_launches.fetch_add(3, std::memory_order_relaxed);
  return cudaGetLastError();
}

AdjointPlan plan_adjoint_edges(int64_t ne, int64_t nq, int sms) {
  const int slots = resident_ctas(
      reinterpret_cast<const void*>(adjoint_edges_kernel<kAdjThreads, kAdjFpt, kAdjQc>),
      kAdjThreads, 0, sms);
  return plan_waves(cdiv(ne, kAdjThreads * kAdjFpt), nq, slots, kAdjQc);
}

size_t adjoint_edges_scratch_bytes(const AdjointPlan& p, int64_t le, int64_t nq) {
  return sizeof(double) * (static_cast<size_t>(p.nranges) * nq * 3 +
                           static_cast<size_t>(p.ngroups) * 6 * le) + 256;
}

cudaError_t adjoint_edges(const AdjointPlan& p, const double* edges, int64_t le, int64_t ne,
                          const double* q, int64_t nq, const double* gw, double* dq,
                          double* dedge, void* scratch, size_t scratch_bytes,
                          cudaStream_t stream) {
  cudaError_t e = cudaSuccess;
  if (nq > 0) e = cudaMemsetAsync(dq, 0, sizeof(double) * 3 * nq, stream);
  if (e == cudaSuccess && ne > 0) e = cudaMemsetAsync(dedge, 0, sizeof(double) * 6 * le, stream);
  if (e != cudaSuccess || nq <= 0 || ne <= 0) return e;
  if (scratch_bytes < adjoint_edges_scratch_bytes(p, le, nq)) return cudaErrorInvalidValue;
  double* dO_part = static_cast<double*>(scratch);
  double* dE_part = dO_part + static_cast<size_t>(p.nranges) * nq * 3;
  e = cudaMemsetAsync(dO_part, 0, sizeof(double) * static_cast<size_t>(p.nranges) * nq * 3,
                      stream);
  if (e != cudaSuccess) return e;
  EdgeAdjointArgs a{edges, le, ne, q, gw, nq, p.blocks_per_range, p.queries_per_group,
                    dO_part, dE_part};
  adjoint_edges_kernel<kAdjThreads, kAdjFpt, kAdjQc>
      <<<dim3(static_cast<unsigned>(p.nranges), static_cast<unsigned>(p.ngroups)), kAdjThreads, 0,
         stream>>>(a);
  finish_dq_kernel<<<static_cast<unsigned>(cdiv(nq * 3, 256)), 256, 0, stream>>>(dO_part, p.nranges,
                                                                               nq, dq);
  finish_dedge_kernel<<<static_cast<unsigned>(cdiv(6 * ne, 256)), 256, 0, stream>>>(
      dE_part, p.ngroups, le, ne, dedge);
  g_launches.fetch_add(3, std::memory_order_relaxed);
  return cudaGetLastError();
}

AdjointPlan plan_adjoint_mixed(int64_t ntiles, int64_t nq, int sms) {
  auto kernel = adjoint_faces_kernel<kFaQc>;
  const int smem = static_cast<int>(sizeof(FaceAdjSmem<kFaQc>));
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  const int slots = resident_ctas(reinterpret_cast<const void*>(kernel), kFaThreads, smem, sms);
  return plan_balanced(cdiv(ntiles, kFaTiles), nq, slots, kFaQc,
                       9 * std::max<int64_t>(ntiles, 1) * kTileFaces);
}

cudaError_t adjoint_mixed(const AdjointPlan& p, const MixedMesh& m, const double* q,
                          const uint32_t* perm, int64_t nq, const double* gw, double* dq,
                          double* dtri, int64_t ld, void* scratch, size_t scratch_bytes,
                          cudaStream_t stream) {
  cudaError_t e = cudaSuccess;
  if (nq > 0) e = cudaMemsetAsync(dq, 0, sizeof(double) * 3 * nq, stream);
  if (e == cudaSuccess && m.nf > 0) e = cudaMemsetAsync(dtri, 0, sizeof(double) * 9 * ld, stream);
  if (e != cudaSuccess || nq <= 0 || m.nf <= 0) return e;
  if (scratch_bytes < adjoint_scratch_bytes(p, m.ld64, nq)) return cudaErrorInvalidValue;
  double* dO_part = static_cast<double*>(scratch);
  double* dF_part = dO_part + static_cast<size_t>(p.nranges) * nq * 3;
  e = cudaMemsetAsync(dO_part, 0, sizeof(double) * static_cast<size_t>(p.nranges) * nq * 3,
                      stream);
  if (e != cudaSuccess) return e;
  const size_t qs_off =
      ((reinterpret_cast<uintptr_t>(dF_part + static_cast<size_t>(p.ngroups) * 9 * m.ld64) + 255) &
       ~static_cast<uintptr_t>(255)) - reinterpret_cast<uintptr_t>(scratch);
  double4* qs = reinterpret_cast<double4*>(static_cast<unsigned char*>(scratch) + qs_off);
  gather_sorted_queries_kernel<<<static_cast<unsigned>(cdiv(nq, 256)), 256, 0, stream>>>(
      q, gw, perm, nq, qs);
  MixedAdjointArgs a{m.tiles, m.ntiles, m.tri64, m.ld64, qs, nq,
                     p.blocks_per_range, p.queries_per_group, dO_part, dF_part};
  auto kernel = adjoint_faces_kernel<kFaQc>;
  const int smem = static_cast<int>(sizeof(FaceAdjSmem<kFaQc>));
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  kernel<<<dim3(static_cast<unsigned>(p.nranges), static_cast<unsigned>(p.ngroups)), kFaThreads,
           smem, stream>>>(a);
  finish_dq_sorted_kernel<<<static_cast<unsigned>(cdiv(nq * 3, 256)), 256, 0, stream>>>(
      dO_part, p.nranges, nq, perm, dq);
  finish_dtri_sorted_kernel<<<static_cast<unsigned>(cdiv(9 * m.ld64, 256)), 256, 0, stream>>>(
      dF_part, p.ngroups, m.ld64, m.face_of, ld, dtri);
  g_launches.fetch_add(4, std::memory_order_relaxed);
  return cudaGetLastError();
}

namespace {

// ---- mixed-precision boundary-edge adjoint -----------------------------------
// The boundary-edge adjoint with the per-face mixed adjoint's precision split.
// Edges are ordered along a Morton curve of their midpoints and cut into tiles of
// 64; per tile an FP64 centre, a power-of-two scale ~ 1/radius and the squared
// far radius (r + kappa h)^2 (h = the tile's longest edge); per edge, in the
// tile's scaled FP32 frame, P, e = Q - P, |e|^2 and the multiplicity m. A pair
// (query, edge) is near when an endpoint lies within kappa |e| of the query; near
// pairs are evaluated in FP64 from the sorted FP64 edges, the rest in FP32: with
// p = P - o, q = p + e, D = |p||q| + p.q (no cancellation at kappa >= 3: p and q
// point the same way), k_P = g m r_p / D, k_Q = g m r_q / D, x = p x e (= p x q):
//   -g m dOmega/dP += k_P x,  -g m dOmega/dQ += k_Q x,  g m dOmega/do += (k_P + k_Q) x,
// 37 FP32 operations (as 19 packed instructions per edge pair) and 3 MUFU per
// pair. Work split, fixed-order reductions and partial arrays as in the per-face
// mixed adjoint; the outputs are those of adjoint_edges.
struct EdgeRec {
  float px, py, pz;  // endpoint P minus the tile centre, times the tile's scale
  float ex, ey, ez;  // Q - P (formed in FP64, then rounded)
  float ee;          // |Q - P|^2
  float m;           // net multiplicity (0 for padding)
};
static_assert(sizeof(EdgeRec) == 32, "edge record is 32 bytes");
constexpr int kEdgeTileBytes = static_cast<int>(sizeof(TileHeader) + kTileFaces * sizeof(EdgeRec));

// AoS midpoints of the edges (7 x le SoA: P, Q, m), for the Morton sort.
__global__ void edge_midpoints_kernel(const double* __restrict__ edges, int64_t le, int64_t ne,
                                      double* __restrict__ mid) {
  const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= ne) return;
#pragma unroll
  for (int x = 0; x < 3; ++x) mid[3 * e + x] = 0.5 * (edges[x * le + e] + edges[(3 + x) * le + e]);
}

__device__ __forceinline__ double warp_max_d(double v) {
  for (int off = 16; off; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
  return v;
}
__device__ __forceinline__ double warp_min_d(double v) {
  for (int off = 16; off; off >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, off));
  return v;
}

// One CTA of 64 threads per tile: edges order[first + j], j < count, in Morton
// order, with first = 64 t and count = min(64, ne - first), or (batched meshes,
// whose tiles do not cross a mesh) both from tile_first / tile_count.
__global__ void __launch_bounds__(kTileFaces) build_edge_tiles_kernel(
    const double* __restrict__ edges, int64_t le, int64_t ne, const uint32_t* __restrict__ order,
    double kappa, unsigned char* __restrict__ tiles, double* __restrict__ e64, int64_t ld64,
    uint32_t* __restrict__ edge_of, const int64_t* __restrict__ tile_first = nullptr,
    const int32_t* __restrict__ tile_count = nullptr) {
  __shared__ double red[8][kTileFaces / 32];
  const int j = threadIdx.x, warp = j >> 5, lane = j & 31;
  const int64_t tile = blockIdx.x;
  const int64_t slot = tile * kTileFaces + j;
  const int64_t first = tile_first ? tile_first[tile] : tile * kTileFaces;
  const int64_t left = ne - first;
  const int64_t count = tile_count ? tile_count[tile] : (left < kTileFaces ? left : kTileFaces);
  const bool valid = j < count;
  const int64_t e = valid ? order[first + j] : 0;
  double v[7];
#pragma unroll
  for (int r = 0; r < 7; ++r) v[r] = valid ? edges[r * le + e] : 0.0;
  double lo[3], hi[3];
#pragma unroll
  for (int x = 0; x < 3; ++x) {
    lo[x] = warp_min_d(valid ? fmin(v[x], v[3 + x]) : INFINITY);
    hi[x] = warp_max_d(valid ? fmax(v[x], v[3 + x]) : -INFINITY);
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
    const double l = fmin(red[x][0], red[x][1]), h = fmax(red[3 + x][0], red[3 + x][1]);
    c[x] = isfinite(l) ? 0.5 * (l + h) : 0.0;
  }
  __syncthreads();
  double r2 = 0.0, h2 = 0.0;
  if (valid) {
    for (int k = 0; k < 2; ++k) {
      const double dx = v[3 * k] - c[0], dy = v[3 * k + 1] - c[1], dz = v[3 * k + 2] - c[2];
      r2 = fmax(r2, dx * dx + dy * dy + dz * dz);
    }
    const double ex = v[3] - v[0], ey = v[4] - v[1], ez = v[5] - v[2];
    h2 = ex * ex + ey * ey + ez * ez;
  }
  double rt = warp_max_d(sqrt(r2)), ht = warp_max_d(sqrt(h2));
  if (lane == 0) {
    red[6][warp] = rt;
    red[7][warp] = ht;
  }
  __syncthreads();
  rt = fmax(red[6][0], red[6][1]);
  ht = fmax(red[7][0], red[7][1]);
  int ex2 = 0;
  if (rt > 0.0) frexp(rt, &ex2);
  const double scale = ldexp(1.0, -ex2);
  unsigned char* rec = tiles + tile * kEdgeTileBytes;
  if (j == 0) {
    TileHeader th{};
    th.cx = c[0];
    th.cy = c[1];
    th.cz = c[2];
    const double far = rt + kappa * ht;
    th.far_r2 = far * far;
    th.scale = scale;
    th.n = static_cast<int32_t>(count);
    th.r = static_cast<float>(rt);
    th.h = static_cast<float>(ht);
    *reinterpret_cast<TileHeader*>(rec) = th;
  }
  EdgeRec er;
  const double ex = (v[3] - v[0]) * scale, ey = (v[4] - v[1]) * scale, ez = (v[5] - v[2]) * scale;
  er.px = valid ? static_cast<float>((v[0] - c[0]) * scale) : 1e18f;
  er.py = valid ? static_cast<float>((v[1] - c[1]) * scale) : 1e18f;
  er.pz = valid ? static_cast<float>((v[2] - c[2]) * scale) : 1e18f;
  er.ex = static_cast<float>(ex);
  er.ey = static_cast<float>(ey);
  er.ez = static_cast<float>(ez);
  er.ee = static_cast<float>(ex * ex + ey * ey + ez * ez);
  er.m = static_cast<float>(v[6]);
  reinterpret_cast<EdgeRec*>(rec + sizeof(TileHeader))[j] = er;
#pragma unroll
  for (int r = 0; r < 7; ++r) e64[r * ld64 + slot] = v[r];
  edge_of[slot] = valid ? static_cast<uint32_t>(e) : 0xffffffffu;
}

// g m dOmega of one (query, edge) pair in FP64, the FP64 edge kernel's formula:
// -g w dOmega/dP into gv[0..2], -g w dOmega/dQ into gv[3..5], g m dOmega/do into go,
// with w = m, or w = 1 when `unit` (edges welded by position: per-endpoint sums
// unweighted, the multiplicity only in dOmega/do).
__device__ __noinline__ void refine_edge_grad(const double* __restrict__ e64, int64_t ld64,
                                              int64_t slot, double4 o, double* acc_col,
                                              int stride, double* go, bool unit) {
  double v[7];
#pragma unroll
  for (int r = 0; r < 7; ++r) v[r] = e64[r * ld64 + slot];
  const double px = v[0] - o.x, py = v[1] - o.y, pz = v[2] - o.z;
  const double qx = v[3] - o.x, qy = v[4] - o.y, qz = v[5] - o.z;
  const double pp = px * px + py * py + pz * pz;
  const double qq = qx * qx + qy * qy + qz * qz;
  const double rp = rsqrt(pp), rq = rsqrt(qq);
  const double rpq = rp * rq;
  const double d = 1.0 + (px * qx + py * qy + pz * qz) * rpq;
  const bool ok = (unit || v[6] != 0.0) && pp > 0.0 && qq > 0.0 && d > 0.0;
  const double w = ok ? o.w * (unit ? 1.0 : v[6]) * rpq / d : 0.0;
  const double cp = ok ? rp * w : 0.0, cq = ok ? rq * w : 0.0;
  const double x0 = py * qz - pz * qy, x1 = pz * qx - px * qz, x2 = px * qy - py * qx;
  acc_col[0] -= cp * x0;
  acc_col[stride] -= cp * x1;
  acc_col[2 * stride] -= cp * x2;
  acc_col[3 * stride] -= cq * x0;
  acc_col[4 * stride] -= cq * x1;
  acc_col[5 * stride] -= cq * x2;
  const double cs = unit ? (cp + cq) * v[6] : cp + cq;
  go[0] += cs * x0;
  go[1] += cs * x1;
  go[2] += cs * x2;
}

struct MixedEdgeArgs {
  const unsigned char* tiles;  // ntiles * kEdgeTileBytes
  int64_t ntiles;
  const double* e64;  // sorted FP64 edges, 7 x ld64 (P, Q, m)
  int64_t ld64;
  const double4* qs;  // nq queries in Morton order: x, y, z, g
  int64_t nq;
  float kappa2;  // kappa^2: a pair is near when min(|p|^2, |q|^2) <= kappa^2 |e|^2
  int64_t blocks_per_range, queries_per_group;
  double* dO_part;  // [nranges][nq][3] by sorted position, zeroed before the launch
  double* dE_part;  // [ngroups][6][ld64] by sorted slot
};

template <int QC, bool DQ = true>
struct EdgeAdjSmem {
  float dO32[DQ ? QC * 3 : 1][kFaRow];  // per-thread FP32 dL/do shares, row 3*query + axis
  double acc64[12][kFaThreads];  // per-edge FP64 sums (thread-private columns)
  double red64[kFaTiles][QC][3];
  double dsum[QC * 3];
  double4 q64[QC];
  float4 frame[QC][kFaTiles][2];  // (-x, -x, -y, -y), (-z, -z, gs, gs) as FP32x2 operands
  int flag[QC][kFaTiles];
  TileHeader th[kFaTiles];
};

// One query against this thread's two edges (the two lanes of every float2): adds
// -g m dOmega/dP and -g m dOmega/dQ into acc and returns g m dOmega/do in d, every
// operand a whole FP32x2 pair, no per-pair sign flip (-p from one packed multiply).
// With CAREFUL, a lane whose edge has an endpoint within kappa |e| (k2ee = kappa^2
// |e|^2, valid = the lane holds an edge) takes g = 0 and unit squared lengths, so
// its terms are finite and zero; bit k of the result flags lane k. With UNIT the
// per-endpoint sums take weight 1 and only dOmega/do the multiplicity m; without DQ
// (UNIT over edges whose m are all 0, so that every dOmega/do term is exactly 0) d is
// left untouched.
template <bool CAREFUL, bool UNIT, bool DQ = true>
__device__ __forceinline__ unsigned edge_pair_terms(const float4 (&fr)[2], const float2 (&fp)[3],
                                                    const float2 (&fe)[3],
                                                    const float2 (&fne)[3], float2 fee, float2 fm,
                                                    float2 k2ee, bool valid0, bool valid1,
                                                    float2 (&acc)[6], float2 (&d)[3]) {
  const float4 f0 = fr[0], f1 = fr[1];
  const float2 px = __fadd2_rn(fp[0], make_float2(f0.x, f0.y));
  const float2 py = __fadd2_rn(fp[1], make_float2(f0.z, f0.w));
  const float2 pz = __fadd2_rn(fp[2], make_float2(f1.x, f1.y));
  float2 gm = UNIT ? make_float2(f1.z, f1.w) : __fmul2_rn(make_float2(f1.z, f1.w), fm);
  float2 pp = __ffma2_rn(px, px, __ffma2_rn(py, py, __fmul2_rn(pz, pz)));
  const float2 s = __ffma2_rn(px, fe[0], __ffma2_rn(py, fe[1], __fmul2_rn(pz, fe[2])));
  const float2 pq = __fadd2_rn(pp, s);
  float2 qq = __ffma2_rn(f2(2.f), s, __fadd2_rn(pp, fee));
  unsigned nb = 0u;
  if constexpr (CAREFUL) {
    const bool n0 = valid0 && fminf(pp.x, qq.x) <= k2ee.x;
    const bool n1 = valid1 && fminf(pp.y, qq.y) <= k2ee.y;
    nb = (n0 ? 1u : 0u) | (n1 ? 2u : 0u);
    gm = make_float2(n0 ? 0.f : gm.x, n1 ? 0.f : gm.y);
    pp = make_float2(n0 ? 1.f : pp.x, n1 ? 1.f : pp.y);
    qq = make_float2(n0 ? 1.f : qq.x, n1 ? 1.f : qq.y);
  }
  const float2 rp = rsqrt2(pp), rq = rsqrt2(qq);
  const float2 lp = __fmul2_rn(pp, rp), lq = __fmul2_rn(qq, rq);
  const float2 gD = __fmul2_rn(gm, rcp2(__ffma2_rn(lp, lq, pq)));
  const float2 kp = __fmul2_rn(rp, gD), kq = __fmul2_rn(rq, gD);
  // x = p x e. With dL/do the tile's -e saves negating p per pair ((-a) b and a (-b)
  // round alike); without it the kernel's register budget is tighter than the three
  // packed negations, which cost fewer instructions than the moves -e brings there.
  float2 x0, x1, x2;
  if constexpr (DQ) {
    x0 = __ffma2_rn(py, fe[2], __fmul2_rn(pz, fne[1]));
    x1 = __ffma2_rn(pz, fe[0], __fmul2_rn(px, fne[2]));
    x2 = __ffma2_rn(px, fe[1], __fmul2_rn(py, fne[0]));
  } else {
    const float2 m1 = f2(-1.f);
    const float2 npx = __fmul2_rn(px, m1), npy = __fmul2_rn(py, m1), npz = __fmul2_rn(pz, m1);
    x0 = __ffma2_rn(py, fe[2], __fmul2_rn(npz, fe[1]));
    x1 = __ffma2_rn(pz, fe[0], __fmul2_rn(npx, fe[2]));
    x2 = __ffma2_rn(px, fe[1], __fmul2_rn(npy, fe[0]));
  }
  acc[0] = __ffma2_rn(kp, x0, acc[0]);
  acc[1] = __ffma2_rn(kp, x1, acc[1]);
  acc[2] = __ffma2_rn(kp, x2, acc[2]);
  acc[3] = __ffma2_rn(kq, x0, acc[3]);
  acc[4] = __ffma2_rn(kq, x1, acc[4]);
  acc[5] = __ffma2_rn(kq, x2, acc[5]);
  if constexpr (DQ) {
    const float2 cs = UNIT ? __fmul2_rn(__fadd2_rn(kp, kq), fm) : __fadd2_rn(kp, kq);
    d[0] = __fmul2_rn(cs, x0);
    d[1] = __fmul2_rn(cs, x1);
    d[2] = __fmul2_rn(cs, x2);
  }
  return nb;
}

__device__ __forceinline__ int jq_of(unsigned mask) { return __ffs(mask) - 1; }

// The work of one CTA: blocks [b_begin, b_end) of kFaTiles edge tiles of one mesh
// against its sorted queries [q_begin, q_end). Indices are local to the mesh: its
// tiles, FP64 edge slots (row stride ld64) and sorted queries start at the pointers.
struct EdgeWork {
  const unsigned char* tiles;
  int64_t ntiles;
  const double* e64;
  int64_t ld64;
  const double4* qs;
  float kappa2;
  int64_t b_begin, b_end, q_begin, q_end;
  double* dO_row;    // this edge range's dL/do partials, [sorted position][3], accumulated
  double* dE_group;  // this query group's per-slot sums, [6][de_ld], written
  int64_t de_ld;
};

// NODQ (with UNIT, for callers that need no dL/do: every net multiplicity is 0)
// compiles the dL/do path out, so that the per-query shares take no shared memory
// and 96 registers fit five CTAs per SM.
template <int QC, bool UNIT, bool NODQ>
__device__ __forceinline__ void edge_adjoint_cta(const EdgeWork& a,
                                                 EdgeAdjSmem<QC, !NODQ>& sm) {
  static_assert(UNIT || !NODQ, "dL/do is dropped only in the unit-weight mode");
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t b_begin = a.b_begin, b_end = a.b_end;
  const int64_t q_begin = a.q_begin, q_end = a.q_end;
  double* dO_row = a.dO_row;

  for (int64_t blk = b_begin; blk < b_end; ++blk) {
    __syncthreads();  // previous block's shared data fully consumed
    if (tid < kFaTiles) {
      const int64_t t = blk * kFaTiles + tid;
      if (t < a.ntiles) {
        sm.th[tid] = *reinterpret_cast<const TileHeader*>(a.tiles + t * kEdgeTileBytes);
      } else {
        TileHeader empty{};
        empty.far_r2 = 0.0;
        empty.scale = 1.0;
        sm.th[tid] = empty;
      }
    }
    // This warp's tile; lane k of every float2 is edge lane + 32 k (padding edges
    // carry a far corner, a zero edge and m = 0: every term they give is zero).
    const int64_t t = blk * kFaTiles + warp;
    const bool tile_ok = t < a.ntiles;
    const unsigned char* rec = a.tiles + (tile_ok ? t : 0) * kEdgeTileBytes;
    const int n = tile_ok ? reinterpret_cast<const TileHeader*>(rec)->n : 0;
    float4 r[2][2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int j = lane + 32 * k;
      const float4* er = reinterpret_cast<const float4*>(rec + sizeof(TileHeader)) + 2 * j;
      r[k][0] = make_float4(1e18f, 1e18f, 1e18f, 0.f);
      r[k][1] = make_float4(0.f, 0.f, 0.f, 0.f);
      if (j < n) {
        r[k][0] = er[0];
        r[k][1] = er[1];
      }
    }
    // Each field of the two edges as one FP32x2 value, built whole.
    const float2 fp[3] = {make_float2(r[0][0].x, r[1][0].x), make_float2(r[0][0].y, r[1][0].y),
                          make_float2(r[0][0].z, r[1][0].z)};
    const float2 fe[3] = {make_float2(r[0][0].w, r[1][0].w), make_float2(r[0][1].x, r[1][1].x),
                          make_float2(r[0][1].y, r[1][1].y)};
    const float2 fne[3] = {__fmul2_rn(fe[0], f2(-1.f)), __fmul2_rn(fe[1], f2(-1.f)),
                           __fmul2_rn(fe[2], f2(-1.f))};
    const float2 fee = make_float2(r[0][1].z, r[1][1].z);
    const float2 fm = make_float2(r[0][1].w, r[1][1].w);
    // Welded sides whose net multiplicities are all 0 in this block (every side of a
    // closed soup) give dOmega/do terms that are exactly 0: the block skips them.
    const bool no_dq = NODQ || (UNIT && __syncthreads_and(fm.x == 0.f && fm.y == 0.f));
    const int64_t slot0 = (tile_ok ? t : 0) * kTileFaces + lane;
#pragma unroll
    for (int r = 0; r < 12; ++r) sm.acc64[r][tid] = 0.0;
    float2 acc[6];
#pragma unroll
    for (int r = 0; r < 6; ++r) acc[r] = f2(0.f);
    const float2 k2ee = __fmul2_rn(f2(a.kappa2), fee);

    int chunks = 0;
    for (int64_t c0 = q_begin; c0 < q_end; c0 += QC) {
      const int nc = static_cast<int>(q_end - c0 < QC ? q_end - c0 : QC);
      __syncthreads();
      for (int item = tid; item < QC * kFaTiles; item += kFaThreads) {
        const int jq = item / kFaTiles, tt = item % kFaTiles;
        if (jq < nc) {
          const double4 o = a.qs[c0 + jq];
          const TileHeader& th = sm.th[tt];
          const double dx = o.x - th.cx, dy = o.y - th.cy, dz = o.z - th.cz;
          const double d2 = dx * dx + dy * dy + dz * dz;
          const bool skip = d2 * th.scale * th.scale > 1.2089258196146292e24;
          const float lx = static_cast<float>(dx * th.scale);
          const float ly = static_cast<float>(dy * th.scale);
          const float lz = static_cast<float>(dz * th.scale);
          const float gs = static_cast<float>(o.w * th.scale);
          sm.frame[jq][tt][0] = make_float4(-lx, -lx, -ly, -ly);
          sm.frame[jq][tt][1] = make_float4(-lz, -lz, gs, gs);
          sm.flag[jq][tt] = skip ? 2 : (d2 >= th.far_r2 ? 0 : 1);
          if (tt == 0) sm.q64[jq] = o;
        }
      }
      if (!no_dq)
        for (int e = tid; e < kFaTiles * QC * 3; e += kFaThreads) (&sm.red64[0][0][0])[e] = 0.0;
      __syncthreads();
      static_assert(QC <= 32, "one mask bit per query of a chunk");
      unsigned near0 = 0u, near1 = 0u;
      const int myflag = lane < nc ? sm.flag[lane][warp] : 2;
      const unsigned far_q = __ballot_sync(0xffffffffu, myflag == 0);
      const unsigned careful_q = __ballot_sync(0xffffffffu, myflag == 1);
      const unsigned skip_q = __ballot_sync(0xffffffffu, myflag == 2 && lane < nc);
      if constexpr (UNIT) {
        if (no_dq) {
          float2 d[3];
          // Four, then two queries per pass (in increasing order, as one at a time
          // would add them): the later ones' arithmetic overlaps the first's latencies.
          unsigned rest = far_q;
#pragma unroll 1
          for (unsigned m = rest; __popc(m) >= 4;) {
            const int j0 = jq_of(m);
            m &= m - 1u;
            const int j1 = jq_of(m);
            m &= m - 1u;
            const int j2 = jq_of(m);
            m &= m - 1u;
            const int j3 = jq_of(m);
            m &= m - 1u;
            rest = m;
            edge_pair_terms<false, true, false>(sm.frame[j0][warp], fp, fe, fne, fee, fm, k2ee,
                                                true, true, acc, d);
            edge_pair_terms<false, true, false>(sm.frame[j1][warp], fp, fe, fne, fee, fm, k2ee,
                                                true, true, acc, d);
            edge_pair_terms<false, true, false>(sm.frame[j2][warp], fp, fe, fne, fee, fm, k2ee,
                                                true, true, acc, d);
            edge_pair_terms<false, true, false>(sm.frame[j3][warp], fp, fe, fne, fee, fm, k2ee,
                                                true, true, acc, d);
          }
#pragma unroll 1
          for (unsigned m = rest; m;) {
            const int j0 = jq_of(m);
            m &= m - 1u;
            if (m) {
              const int j1 = jq_of(m);
              m &= m - 1u;
              edge_pair_terms<false, true, false>(sm.frame[j0][warp], fp, fe, fne, fee, fm, k2ee,
                                                  true, true, acc, d);
              edge_pair_terms<false, true, false>(sm.frame[j1][warp], fp, fe, fne, fee, fm, k2ee,
                                                  true, true, acc, d);
            } else {
              edge_pair_terms<false, true, false>(sm.frame[j0][warp], fp, fe, fne, fee, fm, k2ee,
                                                  true, true, acc, d);
            }
          }
#pragma unroll 1
          for (unsigned m = careful_q; m; m &= m - 1u) {
            const int jq = jq_of(m);
            const unsigned nb = edge_pair_terms<true, true, false>(
                sm.frame[jq][warp], fp, fe, fne, fee, fm, k2ee, lane < n, lane + 32 < n, acc, d);
            near0 |= (nb & 1u) << jq;
            near1 |= (nb >> 1) << jq;
          }
          for (unsigned pending = __reduce_or_sync(0xffffffffu, near0 | near1); pending;
               pending &= pending - 1u) {
            const int jq = jq_of(pending);
            double go[3] = {0.0, 0.0, 0.0};  // exactly 0 here: all m are 0
            if ((near0 >> jq) & 1u)
              refine_edge_grad(a.e64, a.ld64, slot0, sm.q64[jq], &sm.acc64[0][tid], kFaThreads,
                               go, true);
            if ((near1 >> jq) & 1u)
              refine_edge_grad(a.e64, a.ld64, slot0 + 32, sm.q64[jq], &sm.acc64[6][tid],
                               kFaThreads, go, true);
          }
          if (++chunks == kFaFlushQueries / QC || c0 + QC >= q_end) {
            chunks = 0;
#pragma unroll
            for (int r = 0; r < 6; ++r) {
              sm.acc64[r][tid] -= static_cast<double>(acc[r].x);
              sm.acc64[6 + r][tid] -= static_cast<double>(acc[r].y);
              acc[r] = f2(0.f);
            }
          }
          continue;
        }
      }
#pragma unroll 1
      for (unsigned m = far_q; m;) {
        const int j0 = jq_of(m);
        m &= m - 1u;
        float2 d[3];
        if (m) {
          const int j1 = jq_of(m);
          m &= m - 1u;
          float2 d1[3];
          edge_pair_terms<false, UNIT>(sm.frame[j0][warp], fp, fe, fne, fee, fm, k2ee, true, true,
                                       acc, d);
          edge_pair_terms<false, UNIT>(sm.frame[j1][warp], fp, fe, fne, fee, fm, k2ee, true, true,
                                       acc, d1);
          sm.dO32[3 * j1][tid] = d1[0].x + d1[0].y;
          sm.dO32[3 * j1 + 1][tid] = d1[1].x + d1[1].y;
          sm.dO32[3 * j1 + 2][tid] = d1[2].x + d1[2].y;
        } else {
          edge_pair_terms<false, UNIT>(sm.frame[j0][warp], fp, fe, fne, fee, fm, k2ee, true, true,
                                       acc, d);
        }
        sm.dO32[3 * j0][tid] = d[0].x + d[0].y;
        sm.dO32[3 * j0 + 1][tid] = d[1].x + d[1].y;
        sm.dO32[3 * j0 + 2][tid] = d[2].x + d[2].y;
      }
#pragma unroll 1
      for (unsigned m = careful_q; m; m &= m - 1u) {
        // Careful visits: pairs with an endpoint within kappa |e| are refined in FP64
        // below; their FP32 terms come out as zero here.
        const int jq = __ffs(m) - 1;
        float2 d[3];
        const unsigned nb = edge_pair_terms<true, UNIT>(sm.frame[jq][warp], fp, fe, fne, fee, fm,
                                                        k2ee, lane < n, lane + 32 < n, acc, d);
        near0 |= (nb & 1u) << jq;
        near1 |= (nb >> 1) << jq;
        sm.dO32[3 * jq][tid] = d[0].x + d[0].y;
        sm.dO32[3 * jq + 1][tid] = d[1].x + d[1].y;
        sm.dO32[3 * jq + 2][tid] = d[2].x + d[2].y;
      }
      for (unsigned m = skip_q; m; m &= m - 1u) {
        const int jq = __ffs(m) - 1;
        sm.dO32[3 * jq][tid] = 0.f;
        sm.dO32[3 * jq + 1][tid] = 0.f;
        sm.dO32[3 * jq + 2][tid] = 0.f;
      }
      for (unsigned pending = __reduce_or_sync(0xffffffffu, near0 | near1); pending;
           pending &= pending - 1u) {
        const int jq = __ffs(pending) - 1;
        double go[3] = {0.0, 0.0, 0.0};
        if ((near0 >> jq) & 1u)
          refine_edge_grad(a.e64, a.ld64, slot0, sm.q64[jq], &sm.acc64[0][tid], kFaThreads, go,
                           UNIT);
        if ((near1 >> jq) & 1u)
          refine_edge_grad(a.e64, a.ld64, slot0 + 32, sm.q64[jq], &sm.acc64[6][tid], kFaThreads,
                           go, UNIT);
        for (int off = 16; off; off >>= 1) {
          go[0] += __shfl_xor_sync(0xffffffffu, go[0], off);
          go[1] += __shfl_xor_sync(0xffffffffu, go[1], off);
          go[2] += __shfl_xor_sync(0xffffffffu, go[2], off);
        }
        if (lane == 0) {
          sm.red64[warp][jq][0] = go[0];
          sm.red64[warp][jq][1] = go[1];
          sm.red64[warp][jq][2] = go[2];
        }
      }
      __syncthreads();
      for (int base = 0; base + 8 * warp < QC * 3; base += kFaThreads / 4) {
        const int row = base + (tid >> 2), part = tid & 3;
        const float4* src = reinterpret_cast<const float4*>(&sm.dO32[row][32 * part]);
        float4 s4 = src[0];
#pragma unroll
        for (int i = 1; i < 8; ++i) {
          const float4 v = src[i];
          s4.x += v.x;
          s4.y += v.y;
          s4.z += v.z;
          s4.w += v.w;
        }
        float v = (s4.x + s4.y) + (s4.z + s4.w);
        v += __shfl_xor_sync(0xffffffffu, v, 1);
        v += __shfl_xor_sync(0xffffffffu, v, 2);
        if (part == 0 && row < nc * 3) {
          const int jq = row / 3, x = row % 3;
          double sum = static_cast<double>(v);
#pragma unroll
          for (int w = 0; w < kFaTiles; ++w) sum += sm.red64[w][jq][x];
          sm.dsum[row] = sum;
        }
      }
      if (++chunks == kFaFlushQueries / QC || c0 + QC >= q_end) {
        chunks = 0;
#pragma unroll
        for (int r = 0; r < 6; ++r) {
          sm.acc64[r][tid] -= static_cast<double>(acc[r].x);
          sm.acc64[6 + r][tid] -= static_cast<double>(acc[r].y);
          acc[r] = f2(0.f);
        }
      }
      __syncthreads();
      for (int e = tid; e < nc * 3; e += kFaThreads) dO_row[c0 * 3 + e] += sm.dsum[e];
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      if (lane + 32 * k >= n) continue;
#pragma unroll
      for (int r = 0; r < 6; ++r)
        a.dE_group[r * a.de_ld + slot0 + 32 * k] = sm.acc64[6 * k + r][tid];
    }
  }
}

// Five CTAs per SM (96 registers): without dL/do nothing spills; with it a few cold
// values do (16-28 bytes) and it still runs faster than at four CTAs and 122
// registers (open c3: 55.4 -> 53.0 ms, C4 edges 6.6-6.9 -> 6.4-6.6 ms).
template <int QC, bool UNIT, bool NODQ = false>
__global__ void __launch_bounds__(kFaThreads, 5)
    adjoint_edges_mixed_kernel(const MixedEdgeArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  auto& sm = *reinterpret_cast<EdgeAdjSmem<QC, !NODQ>*>(smem_raw);
  const int64_t nblocks = (a.ntiles + kFaTiles - 1) / kFaTiles;
  const int64_t range = blockIdx.x, group = blockIdx.y;
  EdgeWork w;
  w.tiles = a.tiles;
  w.ntiles = a.ntiles;
  w.e64 = a.e64;
  w.ld64 = a.ld64;
  w.qs = a.qs;
  w.kappa2 = a.kappa2;
  w.b_begin = range * a.blocks_per_range;
  w.b_end = min(nblocks, w.b_begin + a.blocks_per_range);
  w.q_begin = group * a.queries_per_group;
  w.q_end = min(a.nq, w.q_begin + a.queries_per_group);
  w.dO_row = a.dO_part + range * a.nq * 3;
  w.dE_group = a.dE_part + group * 6 * a.ld64;
  w.de_ld = a.ld64;
  edge_adjoint_cta<QC, UNIT, NODQ>(w, sm);
}

// dedge[row][edge_of[slot]] = (1/4pi) sum_g dE_part[g][row][slot] (sorted slots to input edges).
__global__ void finish_dedge_sorted_kernel(const double* __restrict__ part, int64_t ngroups,
                                           int64_t ld64, const uint32_t* __restrict__ edge_of,
                                           int64_t le, double* __restrict__ dedge) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= 6 * ld64) return;
  const int64_t r = i / ld64, sl = i % ld64;
  const uint32_t e = edge_of[sl];
  if (e == 0xffffffffu) return;
  double s = 0.0;
  for (int64_t g = 0; g < ngroups; ++g) s += part[(g * 6 + r) * ld64 + sl];
  dedge[r * le + e] = s * kInv4Pi;
}

constexpr int kEaQc = kFaQc;
constexpr int kEaQcNoDq = 32;  // without dL/do shares a 32-query chunk is cheap in shared memory

// Scratch layout of adjoint_edges_mixed (each piece 256-byte aligned).
struct EdgeMixedLayout {
  size_t mid, eperm, sort, tiles, e64, edge_of, qperm, qs, dO, dE, total;
};

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

EdgeMixedLayout edge_mixed_layout(const AdjointPlan& p, int64_t ne, int64_t nq) {
  const int64_t ntiles = std::max<int64_t>(1, cdiv(ne, kTileFaces));
  const int64_t ld64 = ntiles * kTileFaces;
  EdgeMixedLayout l{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t at = off;
    off += align256(std::max<size_t>(bytes, 1));
    return at;
  };
  l.mid = take(sizeof(double) * 3 * static_cast<size_t>(ne));
  l.eperm = take(sizeof(uint32_t) * static_cast<size_t>(ne));
  l.sort = take(std::max(mixed_sort_scratch_bytes(ne), mixed_sort_scratch_bytes(nq)));
  l.tiles = take(static_cast<size_t>(ntiles) * kEdgeTileBytes);
  l.e64 = take(sizeof(double) * 7 * static_cast<size_t>(ld64));
  l.edge_of = take(sizeof(uint32_t) * static_cast<size_t>(ld64));
  l.qperm = take(sizeof(uint32_t) * static_cast<size_t>(nq));
  l.qs = take(sizeof(double4) * static_cast<size_t>(nq));
  l.dO = take(sizeof(double) * static_cast<size_t>(p.nranges) * nq * 3);
  l.dE = take(sizeof(double) * static_cast<size_t>(p.ngroups) * 6 * ld64);
  l.total = off;
  return l;
}

}  // namespace

AdjointPlan plan_adjoint_edges_mixed(int64_t ne, int64_t nq, int sms, bool no_dq) {
  auto kernel = no_dq ? adjoint_edges_mixed_kernel<kEaQcNoDq, true, true>
                      : adjoint_edges_mixed_kernel<kEaQc, false>;
  const int smem = static_cast<int>(no_dq ? sizeof(EdgeAdjSmem<kEaQcNoDq, false>)
                                          : sizeof(EdgeAdjSmem<kEaQc>));
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  const int slots = resident_ctas(reinterpret_cast<const void*>(kernel), kFaThreads, smem, sms);
  const int64_t ntiles = std::max<int64_t>(1, cdiv(ne, kTileFaces));
  return plan_balanced(cdiv(ntiles, kFaTiles), nq, slots, no_dq ? kEaQcNoDq : kEaQc,
                       6 * ntiles * kTileFaces);
}

size_t adjoint_edges_mixed_scratch_bytes(const AdjointPlan& p, int64_t ne, int64_t nq) {
  return edge_mixed_layout(p, ne, nq).total;
}

cudaError_t adjoint_edges_mixed(const AdjointPlan& p, const double* edges, int64_t le, int64_t ne,
                                const double* q, int64_t nq, const double* gw, double kappa,
                                bool unit, double* dq, double* dedge, void* scratch,
                                size_t scratch_bytes, cudaStream_t stream) {
  cudaError_t e = cudaSuccess;
  const bool no_dq = dq == nullptr;  // unit weights only: dL/do not wanted
  if (no_dq && !unit) return cudaErrorInvalidValue;
  if (nq > 0 && !no_dq) e = cudaMemsetAsync(dq, 0, sizeof(double) * 3 * nq, stream);
  if (e == cudaSuccess && ne > 0) e = cudaMemsetAsync(dedge, 0, sizeof(double) * 6 * le, stream);
  if (e != cudaSuccess || nq <= 0 || ne <= 0) return e;
  const EdgeMixedLayout l = edge_mixed_layout(p, ne, nq);
  if (scratch_bytes < l.total) return cudaErrorInvalidValue;
  unsigned char* s = static_cast<unsigned char*>(scratch);
  double* mid = reinterpret_cast<double*>(s + l.mid);
  uint32_t* eperm = reinterpret_cast<uint32_t*>(s + l.eperm);
  unsigned char* tiles = s + l.tiles;
  double* e64 = reinterpret_cast<double*>(s + l.e64);
  uint32_t* edge_of = reinterpret_cast<uint32_t*>(s + l.edge_of);
  uint32_t* qperm = reinterpret_cast<uint32_t*>(s + l.qperm);
  double4* qs = reinterpret_cast<double4*>(s + l.qs);
  double* dO_part = reinterpret_cast<double*>(s + l.dO);
  double* dE_part = reinterpret_cast<double*>(s + l.dE);
  const size_t sort_bytes = l.tiles - l.sort;
  const int64_t ntiles = cdiv(ne, kTileFaces);
  const int64_t ld64 = ntiles * kTileFaces;
  edge_midpoints_kernel<<<static_cast<unsigned>(cdiv(ne, 256)), 256, 0, stream>>>(edges, le, ne,
                                                                                mid);
  if ((e = mixed_sort_queries(mid, ne, eperm, s + l.sort, sort_bytes, stream)) != cudaSuccess)
    return e;
  build_edge_tiles_kernel<<<static_cast<unsigned>(ntiles), kTileFaces, 0, stream>>>(
      edges, le, ne, eperm, kappa, tiles, e64, ld64, edge_of);
  if ((e = mixed_sort_queries(q, nq, qperm, s + l.sort, sort_bytes, stream)) != cudaSuccess)
    return e;
  gather_sorted_queries_kernel<<<static_cast<unsigned>(cdiv(nq, 256)), 256, 0, stream>>>(
      q, gw, qperm, nq, qs);
  if (!no_dq &&
      (e = cudaMemsetAsync(dO_part, 0, sizeof(double) * static_cast<size_t>(p.nranges) * nq * 3,
                           stream)) != cudaSuccess)
    return e;
  MixedEdgeArgs a{tiles, ntiles, e64, ld64, qs, nq, static_cast<float>(kappa * kappa),
                  p.blocks_per_range, p.queries_per_group, dO_part, dE_part};
  auto kernel = no_dq ? adjoint_edges_mixed_kernel<kEaQcNoDq, true, true>
                      : (unit ? adjoint_edges_mixed_kernel<kEaQc, true>
                              : adjoint_edges_mixed_kernel<kEaQc, false>);
  const int smem = static_cast<int>(no_dq ? sizeof(EdgeAdjSmem<kEaQcNoDq, false>)
                                          : sizeof(EdgeAdjSmem<kEaQc>));
  if ((e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) !=
      cudaSuccess)
    return e;
  kernel<<<dim3(static_cast<unsigned>(p.nranges), static_cast<unsigned>(p.ngroups)), kFaThreads,
           smem, stream>>>(a);
  if (!no_dq)
    finish_dq_sorted_kernel<<<static_cast<unsigned>(cdiv(nq * 3, 256)), 256, 0, stream>>>(
        dO_part, p.nranges, nq, qperm, dq);
  finish_dedge_sorted_kernel<<<static_cast<unsigned>(cdiv(6 * ld64, 256)), 256, 0, stream>>>(
      dE_part, p.ngroups, ld64, edge_of, le, dedge);
  g_launches.fetch_add(no_dq ? 6 : 7, std::memory_order_relaxed);
  return cudaGetLastError();
}

cudaError_t gather_vertex_grad(const double* dtri, int64_t ld, int corners,
                               const int64_t* indptr, const int64_t* entries, int64_t nv,
                               double* dV, cudaStream_t stream) {
  if (nv <= 0) return cudaSuccess;
  gather_vertex_kernel<<<static_cast<unsigned>(cdiv(nv, 256)), 256, 0, stream>>>(
      dtri, ld, corners, indptr, entries, nv, dV);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError();
}

// ---- batched boundary-edge adjoint ------------------------------------------
// Every mesh's net boundary edges (computed once from the faces on the host)
// are concatenated; work items (mesh, range of edges, group of queries) are
// taken from an atomic counter by a persistent grid. An item owns one row of
// the mesh's per-range dL/do partials and one row of its per-group edge
// partials, so the schedule is dynamic but every sum is in a fixed order.
struct BatchEdgeItem {
  int64_t e_begin, e_end;  // global edge indices
  int64_t q_begin, q_end;  // global query indices
  int64_t do_row;          // dO_part offset of this item's row, in doubles, minus 3*q_off
  int64_t de_row;          // dE_part offset of this item's group, in doubles, minus e_off
  int64_t ne;              // edges in the mesh (row stride of the group block)
};

struct BatchEdgeMesh {
  int64_t e_off, ne, q_off, nq, nranges, ngroups, do_off, de_off;
};

// Mixed path: mesh m's edges fill tiles [tile_off, tile_off + ntile) (slots 64 per
// tile, ld = 64 ntile per mesh) in its own Morton order; its sorted queries are
// positions [q_off, q_off + nq) of the batch's.
struct BatchMixedMesh {
  int64_t tile_off, ntile, q_off, nq, nranges, ngroups, do_off, de_off;
};

// One CTA's work on the mixed path (the fields of EdgeWork, mesh-relative).
struct BatchMixedItem {
  int64_t tile_off, ntiles, q_off;
  int64_t b_begin, b_end, q_begin, q_end;
  int64_t do_row;   // dO offset of this range's row (mesh-local sorted positions)
  int64_t de_base;  // dE offset of this group's [6][de_ld] block
  int64_t de_ld;
};

struct BatchEdges {
  int64_t ne_total = 0, le = 1, n_items = 0, do_doubles = 0, de_doubles = 0;
  int grid = 0;
  int64_t* ends = nullptr;      // ne_total x 2, global vertex indices
  double* mult = nullptr;       // ne_total
  double* edges = nullptr;      // 7 x le SoA (positions filled per call)
  double* dedge = nullptr;      // 6 x le
  int64_t* indptr = nullptr;    // total_nv + 1
  int64_t* entries = nullptr;   // 2 * ne_total
  BatchEdgeItem* items = nullptr;
  BatchEdgeMesh* meshes = nullptr;
  int32_t* query_mesh = nullptr;  // total_nq
  int32_t* edge_mesh = nullptr;   // ne_total
  unsigned int* counter = nullptr;
  double* dO_part = nullptr;
  double* dE_part = nullptr;
  // Mixed path (the default).
  bool fp64 = false;
  int64_t nt = 0, m_items = 0, m_do = 0, m_de = 0;
  int64_t* tile_first = nullptr;   // nt: sorted position of the tile's first edge
  int32_t* tile_count = nullptr;   // nt
  int32_t* tile_mesh = nullptr;    // nt
  BatchMixedMesh* mmeshes = nullptr;
  BatchMixedItem* mitems = nullptr;
  double* mid = nullptr;           // ne_total x 3 edge midpoints
  unsigned long long* box = nullptr;
  uint64_t* keys_in = nullptr;
  uint64_t* keys_out = nullptr;
  uint32_t* vals_in = nullptr;
  uint32_t* eperm = nullptr;       // ne_total
  uint32_t* qperm = nullptr;       // total_nq
  void* temp = nullptr;
  size_t temp_bytes = 0;
  unsigned char* tiles = nullptr;  // nt x kEdgeTileBytes
  double* e64 = nullptr;           // 7 x 64 nt
  uint32_t* edge_of = nullptr;     // 64 nt
  double4* qs = nullptr;           // total_nq
  double* mdO = nullptr;
  double* mdE = nullptr;
};

namespace {

constexpr int64_t kBatchEdgeRange = 2048;   // edges per item
constexpr int64_t kBatchQueryGroup = 2048;  // queries per item

__global__ void batch_edge_positions_kernel(const double* __restrict__ V,
                                            const int64_t* __restrict__ ends,
                                            const double* __restrict__ mult, int64_t ne,
                                            int64_t le, double* __restrict__ edges) {
  const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  const int64_t u = ends[2 * e], v = ends[2 * e + 1];
#pragma unroll
  for (int x = 0; x < 3; ++x) {
    edges[x * le + e] = V[3 * u + x];
    edges[(3 + x) * le + e] = V[3 * v + x];
  }
  edges[6 * le + e] = mult[e];
}

struct BatchEdgeArgs {
  const double* edges;
  int64_t le;
  const double* q;
  const double* gw;
  const BatchEdgeItem* items;
  int64_t n_items;
  unsigned int* counter;
  double* dO_part;
  double* dE_part;
};

template <int THREADS, int EPT, int QC>
__global__ void __launch_bounds__(THREADS, 2) batch_edges_kernel(const BatchEdgeArgs a) {
  __shared__ double sq[QC][4];
  __shared__ double red[THREADS / 32][QC][3];
  __shared__ int64_t s_item;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int kBlockEdges = THREADS * EPT;
  for (;;) {
    __syncthreads();
    if (tid == 0) s_item = static_cast<int64_t>(atomicAdd(a.counter, 1u));
    __syncthreads();
    const int64_t item = s_item;
    if (item >= a.n_items) break;
    const BatchEdgeItem it = a.items[item];
    for (int64_t b0 = it.e_begin; b0 < it.e_end; b0 += kBlockEdges) {
      double ev[EPT][7], acc[EPT][6];
#pragma unroll
      for (int k = 0; k < EPT; ++k) {
        const int64_t e = b0 + k * THREADS + tid;
        const bool valid = e < it.e_end;
#pragma unroll
        for (int r = 0; r < 7; ++r) ev[k][r] = valid ? a.edges[r * a.le + e] : 0.0;
#pragma unroll
        for (int r = 0; r < 6; ++r) acc[k][r] = 0.0;
      }
      for (int64_t c0 = it.q_begin; c0 < it.q_end; c0 += QC) {
        const int nc = static_cast<int>(it.q_end - c0 < QC ? it.q_end - c0 : QC);
        __syncthreads();
        if (tid < nc) {
          const int64_t qi = c0 + tid;
          sq[tid][0] = a.q[3 * qi];
          sq[tid][1] = a.q[3 * qi + 1];
          sq[tid][2] = a.q[3 * qi + 2];
          sq[tid][3] = a.gw[qi];
        }
        __syncthreads();
#pragma unroll 1
        for (int j = 0; j < nc; ++j) {
          const double ox = sq[j][0], oy = sq[j][1], oz = sq[j][2], g = sq[j][3];
          double dox = 0.0, doy = 0.0, doz = 0.0;
#pragma unroll
          for (int k = 0; k < EPT; ++k) {
            const double px = ev[k][0] - ox, py = ev[k][1] - oy, pz = ev[k][2] - oz;
            const double qx = ev[k][3] - ox, qy = ev[k][4] - oy, qz = ev[k][5] - oz;
            const double pp = px * px + py * py + pz * pz;
            const double qq = qx * qx + qy * qy + qz * qz;
            const double rp = rsqrt(pp), rq = rsqrt(qq);
            const double rpq = rp * rq;
            const double d = 1.0 + (px * qx + py * qy + pz * qz) * rpq;
            const bool ok = ev[k][6] != 0.0 && pp > 0.0 && qq > 0.0 && d > 0.0;
            const double w = ok ? g * ev[k][6] * rpq / d : 0.0;
            const double cp = ok ? rp * w : 0.0, cq = ok ? rq * w : 0.0;
            const double x0 = py * qz - pz * qy, x1 = pz * qx - px * qz, x2 = px * qy - py * qx;
            acc[k][0] -= cp * x0;
            acc[k][1] -= cp * x1;
            acc[k][2] -= cp * x2;
            acc[k][3] -= cq * x0;
            acc[k][4] -= cq * x1;
            acc[k][5] -= cq * x2;
            const double c = cp + cq;
            dox += c * x0;
            doy += c * x1;
            doz += c * x2;
          }
          for (int off = 16; off; off >>= 1) {
            dox += __shfl_xor_sync(0xffffffffu, dox, off);
            doy += __shfl_xor_sync(0xffffffffu, doy, off);
            doz += __shfl_xor_sync(0xffffffffu, doz, off);
          }
          if (lane == 0) {
            red[warp][j][0] = dox;
            red[warp][j][1] = doy;
            red[warp][j][2] = doz;
          }
        }
        __syncthreads();
        for (int e = tid; e < nc * 3; e += THREADS) {
          const int j = e / 3, x = e % 3;
          double sum = 0.0;
#pragma unroll
          for (int w = 0; w < THREADS / 32; ++w) sum += red[w][j][x];
          a.dO_part[it.do_row + (c0 + j) * 3 + x] += sum;
        }
      }
#pragma unroll
      for (int k = 0; k < EPT; ++k) {
        const int64_t e = b0 + k * THREADS + tid;
        if (e >= it.e_end) continue;
#pragma unroll
        for (int r = 0; r < 6; ++r) a.dE_part[it.de_row + r * it.ne + e] = acc[k][r];
      }
    }
  }
}

__global__ void batch_finish_dq_kernel(const double* __restrict__ dO_part,
                                       const BatchEdgeMesh* __restrict__ meshes,
                                       const int32_t* __restrict__ query_mesh, int64_t total_nq,
                                       double* __restrict__ dq) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= total_nq * 3) return;
  const int64_t qi = i / 3, x = i % 3;
  const BatchEdgeMesh mm = meshes[query_mesh[qi]];
  double s = 0.0;
  for (int64_t r = 0; r < mm.nranges; ++r)
    s += dO_part[mm.do_off + (r * mm.nq + (qi - mm.q_off)) * 3 + x];
  dq[i] = s * kInv4Pi;
}

__global__ void batch_finish_dedge_kernel(const double* __restrict__ dE_part,
                                          const BatchEdgeMesh* __restrict__ meshes,
                                          const int32_t* __restrict__ edge_mesh, int64_t ne_total,
                                          int64_t le, double* __restrict__ dedge) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= ne_total * 6) return;
  const int64_t e = i / 6, r = i % 6;
  const BatchEdgeMesh mm = meshes[edge_mesh[e]];
  double s = 0.0;
  for (int64_t g = 0; g < mm.ngroups; ++g)
    s += dE_part[mm.de_off + (g * 6 + r) * mm.ne + (e - mm.e_off)];
  dedge[r * le + e] = s * kInv4Pi;
}

constexpr int64_t kBatchMixedBlocks = 16;     // largest item: 4-tile blocks per range
constexpr int64_t kBatchMixedQueries = 4096;  // (4,096 edges) and sorted queries per group
static_assert(kBatchMixedQueries % kFaFlushQueries == 0, "groups hold whole FP32 flushes");

struct BatchMixedArgs {
  const BatchMixedItem* items;
  const unsigned char* tiles;
  const double* e64;
  int64_t ld64;
  const double4* qs;
  float kappa2;
  double* dO;
  double* dE;
};

// The mixed edge adjoint's CTA over work items: item blockIdx.x is one (mesh, edge
// range, query group) of one mesh, whose sums go to the mesh's own partial rows.
template <int QC>
__global__ void __launch_bounds__(kFaThreads, 4) batch_edges_mixed_kernel(const BatchMixedArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  auto& sm = *reinterpret_cast<EdgeAdjSmem<QC, true>*>(smem_raw);
  const BatchMixedItem it = a.items[blockIdx.x];
  EdgeWork w;
  w.tiles = a.tiles + it.tile_off * kEdgeTileBytes;
  w.ntiles = it.ntiles;
  w.e64 = a.e64 + it.tile_off * kTileFaces;
  w.ld64 = a.ld64;
  w.qs = a.qs + it.q_off;
  w.kappa2 = a.kappa2;
  w.b_begin = it.b_begin;
  w.b_end = it.b_end;
  w.q_begin = it.q_begin;
  w.q_end = it.q_end;
  w.dO_row = a.dO + it.do_row;
  w.dE_group = a.dE + it.de_base;
  w.de_ld = it.de_ld;
  edge_adjoint_cta<QC, false, false>(w, sm);
}

// dq[qperm[s]] = (1/4pi) sum over the mesh's ranges of dO at sorted position s
// (sorted positions are grouped by mesh as the input queries are).
__global__ void batch_mixed_finish_dq_kernel(const double* __restrict__ dO,
                                             const BatchMixedMesh* __restrict__ meshes,
                                             const int32_t* __restrict__ query_mesh,
                                             const uint32_t* __restrict__ qperm,
                                             int64_t total_nq, double* __restrict__ dq) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= total_nq * 3) return;
  const int64_t sp = i / 3, x = i % 3;
  const BatchMixedMesh mm = meshes[query_mesh[sp]];
  double s = 0.0;
  for (int64_t r = 0; r < mm.nranges; ++r)
    s += dO[mm.do_off + (r * mm.nq + (sp - mm.q_off)) * 3 + x];
  dq[3 * static_cast<int64_t>(qperm[sp]) + x] = s * kInv4Pi;
}

// dedge[row][edge_of[slot]] = (1/4pi) sum over the mesh's groups of dE at the slot.
__global__ void batch_mixed_finish_dedge_kernel(const double* __restrict__ dE,
                                                const BatchMixedMesh* __restrict__ meshes,
                                                const int32_t* __restrict__ tile_mesh,
                                                const uint32_t* __restrict__ edge_of, int64_t nt,
                                                int64_t le, double* __restrict__ dedge) {
  const int64_t slots = nt * kTileFaces;
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= 6 * slots) return;
  const int64_t r = i / slots, sl = i % slots;
  const uint32_t e = edge_of[sl];
  if (e == 0xffffffffu) return;
  const BatchMixedMesh mm = meshes[tile_mesh[sl / kTileFaces]];
  const int64_t ld = mm.ntile * kTileFaces, local = sl - mm.tile_off * kTileFaces;
  double s = 0.0;
  for (int64_t g = 0; g < mm.ngroups; ++g) s += dE[mm.de_off + (g * 6 + r) * ld + local];
  dedge[r * le + e] = s * kInv4Pi;
}

}  // namespace

cudaError_t batch_edges_create(BatchState* b, const int64_t* F) {
  BatchEdges* E = new BatchEdges();
  b->edges = E;
  std::vector<int64_t> ends;
  std::vector<double> mult;
  std::vector<BatchEdgeMesh> meshes(b->nmesh);
  std::vector<int32_t> edge_mesh;
  for (int64_t m = 0; m < b->nmesh; ++m) {
    // Net multiplicity of every undirected edge {u < v}: +1 per u -> v, -1 per v -> u.
    std::vector<std::pair<int64_t, int>> keyed;
    keyed.reserve(3 * b->nf[m]);
    const int64_t nvm = std::max<int64_t>(b->nv[m], 1);
    for (int64_t f = b->f_off[m]; f < b->f_off[m + 1]; ++f)
      for (int c = 0; c < 3; ++c) {
        const int64_t u = F[3 * f + c], v = F[3 * f + (c + 1) % 3];
        if (u == v) continue;
        keyed.emplace_back(std::min(u, v) * nvm + std::max(u, v), u < v ? 1 : -1);
      }
    std::sort(keyed.begin(), keyed.end());
    const int64_t e_off = static_cast<int64_t>(mult.size());
    for (size_t i = 0; i < keyed.size();) {
      size_t j = i;
      int net = 0;
      for (; j < keyed.size() && keyed[j].first == keyed[i].first; ++j) net += keyed[j].second;
      if (net != 0) {
        ends.push_back(keyed[i].first / nvm + b->v_off[m]);
        ends.push_back(keyed[i].first % nvm + b->v_off[m]);
        mult.push_back(static_cast<double>(net));
        edge_mesh.push_back(static_cast<int32_t>(m));
      }
      i = j;
    }
    BatchEdgeMesh& mm = meshes[m];
    mm.e_off = e_off;
    mm.ne = static_cast<int64_t>(mult.size()) - e_off;
    mm.q_off = b->q_off[m];
    mm.nq = b->nq[m];
    mm.nranges = mm.ne > 0 ? (mm.ne + kBatchEdgeRange - 1) / kBatchEdgeRange : 0;
    mm.ngroups = mm.nq > 0 ? (mm.nq + kBatchQueryGroup - 1) / kBatchQueryGroup : 0;
  }
  E->ne_total = static_cast<int64_t>(mult.size());
  E->le = std::max<int64_t>(E->ne_total, 1);
  std::vector<BatchEdgeItem> items;
  int64_t do_off = 0, de_off = 0;
  for (int64_t m = 0; m < b->nmesh; ++m) {
    BatchEdgeMesh& mm = meshes[m];
    mm.do_off = do_off;
    mm.de_off = de_off;
    if (mm.ne > 0 && mm.nq > 0) {
      for (int64_t r = 0; r < mm.nranges; ++r)
        for (int64_t g = 0; g < mm.ngroups; ++g) {
          BatchEdgeItem it;
          it.e_begin = mm.e_off + r * kBatchEdgeRange;
          it.e_end = std::min(mm.e_off + mm.ne, it.e_begin + kBatchEdgeRange);
          it.q_begin = mm.q_off + g * kBatchQueryGroup;
          it.q_end = std::min(mm.q_off + mm.nq, it.q_begin + kBatchQueryGroup);
          it.do_row = do_off + r * mm.nq * 3 - 3 * mm.q_off;
          it.de_row = de_off + g * 6 * mm.ne - mm.e_off;
          it.ne = mm.ne;
          items.push_back(it);
        }
      do_off += mm.nranges * mm.nq * 3;
      de_off += mm.ngroups * 6 * mm.ne;
    }
  }
  std::stable_sort(items.begin(), items.end(), [](const BatchEdgeItem& x, const BatchEdgeItem& y) {
    return (x.e_end - x.e_begin) * (x.q_end - x.q_begin) >
           (y.e_end - y.e_begin) * (y.q_end - y.q_begin);
  });
  E->n_items = static_cast<int64_t>(items.size());
  E->do_doubles = do_off;
  E->de_doubles = de_off;
  // Vertex -> (2*edge + end) list, grouped by global vertex id.
  std::vector<int64_t> indptr(b->total_nv + 1, 0), entries(ends.size());
  for (int64_t v : ends) ++indptr[v + 1];
  for (int64_t v = 0; v < b->total_nv; ++v) indptr[v + 1] += indptr[v];
  {
    std::vector<int64_t> fill(indptr.begin(), indptr.end() - 1);
    for (size_t i = 0; i < ends.size(); ++i) entries[fill[ends[i]]++] = static_cast<int64_t>(i);
  }
  std::vector<int32_t> query_mesh(std::max<int64_t>(b->total_nq, 1));
  for (int64_t m = 0; m < b->nmesh; ++m)
    for (int64_t i = b->q_off[m]; i < b->q_off[m + 1]; ++i) query_mesh[i] = static_cast<int32_t>(m);

  auto up = [](auto** dst, const auto& src, size_t min_count) -> cudaError_t {
    using T = typename std::remove_reference<decltype(src)>::type::value_type;
    const size_t n = std::max(src.size(), min_count);
    cudaError_t e = dev_malloc(reinterpret_cast<void**>(dst), sizeof(T) * std::max<size_t>(n, 1));
    if (e == cudaSuccess && !src.empty())
      e = cudaMemcpy(*dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice);
    return e;
  };
  cudaError_t e;
  if ((e = up(&E->ends, ends, 2)) != cudaSuccess || (e = up(&E->mult, mult, 1)) != cudaSuccess ||
      (e = up(&E->indptr, indptr, 1)) != cudaSuccess ||
      (e = up(&E->entries, entries, 1)) != cudaSuccess ||
      (e = up(&E->items, items, 1)) != cudaSuccess ||
      (e = up(&E->meshes, meshes, 1)) != cudaSuccess ||
      (e = up(&E->query_mesh, query_mesh, 1)) != cudaSuccess ||
      (e = up(&E->edge_mesh, edge_mesh, 1)) != cudaSuccess ||
      (e = dev_malloc(reinterpret_cast<void**>(&E->edges), sizeof(double) * 7 * E->le)) !=
          cudaSuccess ||
      (e = dev_malloc(reinterpret_cast<void**>(&E->dedge), sizeof(double) * 6 * E->le)) !=
          cudaSuccess ||
      (e = dev_malloc(reinterpret_cast<void**>(&E->counter), sizeof(unsigned int))) !=
          cudaSuccess ||
      (e = dev_malloc(reinterpret_cast<void**>(&E->dO_part),
                      sizeof(double) * std::max<int64_t>(E->do_doubles, 1))) != cudaSuccess ||
      (e = dev_malloc(reinterpret_cast<void**>(&E->dE_part),
                      sizeof(double) * std::max<int64_t>(E->de_doubles, 1))) != cudaSuccess)
    return e;
  // Mixed path: every mesh's edges in whole 64-edge tiles of their own, and (edge
  // range, query group) items per mesh, largest first.
  std::vector<BatchMixedMesh> mmeshes(b->nmesh);
  std::vector<int64_t> tile_first;
  std::vector<int32_t> tile_count, tile_mesh;
  std::vector<BatchMixedItem> mitems;
  {
    // Item size: the largest that still gives at least 8 items per SM (halving the
    // longer side, edges or queries, down to one block or one FP32 flush of queries).
    int64_t br = kBatchMixedBlocks, qg = kBatchMixedQueries;
    auto items_for = [&](int64_t r, int64_t g) {
      int64_t n = 0;
      for (int64_t m = 0; m < b->nmesh; ++m)
        if (meshes[m].ne > 0 && meshes[m].nq > 0)
          n += cdiv(cdiv(cdiv(meshes[m].ne, kTileFaces), kFaTiles), r) * cdiv(meshes[m].nq, g);
      return n;
    };
    const int64_t want = 8 * std::max(1, b->sms);
    while (items_for(br, qg) < want && (br > 1 || qg > kFaFlushQueries)) {
      if (qg > kFaFlushQueries && (qg >= br * kFaTiles * kTileFaces || br == 1))
        qg /= 2;
      else
        br /= 2;
    }
    int64_t mdo = 0, mde = 0, toff = 0;
    for (int64_t m = 0; m < b->nmesh; ++m) {
      const BatchEdgeMesh& em = meshes[m];
      BatchMixedMesh& mm = mmeshes[m];
      mm.tile_off = toff;
      mm.ntile = cdiv(em.ne, kTileFaces);
      mm.q_off = em.q_off;
      mm.nq = em.nq;
      for (int64_t t = 0; t < mm.ntile; ++t) {
        tile_first.push_back(em.e_off + t * kTileFaces);
        tile_count.push_back(static_cast<int32_t>(std::min<int64_t>(kTileFaces,
                                                                    em.ne - t * kTileFaces)));
        tile_mesh.push_back(static_cast<int32_t>(m));
      }
      toff += mm.ntile;
      const bool work = em.ne > 0 && em.nq > 0;
      const int64_t nblocks = cdiv(mm.ntile, kFaTiles), ld = mm.ntile * kTileFaces;
      mm.nranges = work ? cdiv(nblocks, br) : 0;
      mm.ngroups = work ? cdiv(em.nq, qg) : 0;
      mm.do_off = mdo;
      mm.de_off = mde;
      for (int64_t r = 0; r < mm.nranges; ++r)
        for (int64_t g = 0; g < mm.ngroups; ++g) {
          BatchMixedItem it;
          it.tile_off = mm.tile_off;
          it.ntiles = mm.ntile;
          it.q_off = mm.q_off;
          it.b_begin = r * br;
          it.b_end = std::min(nblocks, it.b_begin + br);
          it.q_begin = g * qg;
          it.q_end = std::min(em.nq, it.q_begin + qg);
          it.do_row = mdo + r * em.nq * 3;
          it.de_base = mde + g * 6 * ld;
          it.de_ld = ld;
          mitems.push_back(it);
        }
      mdo += mm.nranges * em.nq * 3;
      mde += mm.ngroups * 6 * ld;
    }
    E->nt = toff;
    E->m_do = mdo;
    E->m_de = mde;
  }
  std::stable_sort(mitems.begin(), mitems.end(),
                   [](const BatchMixedItem& x, const BatchMixedItem& y) {
                     return (x.b_end - x.b_begin) * (x.q_end - x.q_begin) >
                            (y.b_end - y.b_begin) * (y.q_end - y.q_begin);
                   });
  E->m_items = static_cast<int64_t>(mitems.size());
  const int64_t nkeys = std::max<int64_t>({E->ne_total, b->total_nq, 1});
  E->temp_bytes = batch_morton_temp_bytes(nkeys, b->mesh_bits);
  const int64_t nt1 = std::max<int64_t>(E->nt, 1);
  if ((e = up(&E->tile_first, tile_first, 1)) != cudaSuccess ||
      (e = up(&E->tile_count, tile_count, 1)) != cudaSuccess ||
      (e = up(&E->tile_mesh, tile_mesh, 1)) != cudaSuccess ||
      (e = up(&E->mmeshes, mmeshes, 1)) != cudaSuccess ||
      (e = up(&E->mitems, mitems, 1)) != cudaSuccess ||
      (e = dev_malloc(reinterpret_cast<void**>(&E->mid),
                      sizeof(double) * 3 * std::max<int64_t>(E->ne_total, 1))) != cudaSuccess ||
      (e = dev_malloc(reinterpret_cast<void**>(&E->box),
                      sizeof(unsigned long long) * 6 * std::max<int64_t>(b->nmesh, 1))) !=
          cudaSuccess ||
      (e = dev_malloc(reinterpret_cast<void**>(&E->keys_in), sizeof(uint64_t) * nkeys)) !=
          cudaSuccess ||
      (e = dev_malloc(reinterpret_cast<void**>(&E->keys_out), sizeof(uint64_t) * nkeys)) !=
          cudaSuccess ||
      (e = dev_malloc(reinterpret_cast<void**>(&E->vals_in), sizeof(uint32_t) * nkeys)) !=
          cudaSuccess ||
      (e = dev_malloc(reinterpret_cast<void**>(&E->eperm),
                      sizeof(uint32_t) * std::max<int64_t>(E->ne_total, 1))) != cudaSuccess ||
      (e = dev_malloc(reinterpret_cast<void**>(&E->qperm),
                      sizeof(uint32_t) * std::max<int64_t>(b->total_nq, 1))) != cudaSuccess ||
      (e = dev_malloc(&E->temp, std::max<size_t>(E->temp_bytes, 16))) != cudaSuccess ||
      (e = dev_malloc(reinterpret_cast<void**>(&E->tiles),
                      static_cast<size_t>(kEdgeTileBytes) * nt1)) != cudaSuccess ||
      (e = dev_malloc(reinterpret_cast<void**>(&E->e64),
                      sizeof(double) * 7 * kTileFaces * nt1)) != cudaSuccess ||
      (e = dev_malloc(reinterpret_cast<void**>(&E->edge_of),
                      sizeof(uint32_t) * kTileFaces * nt1)) != cudaSuccess ||
      (e = dev_malloc(reinterpret_cast<void**>(&E->qs),
                      sizeof(double4) * std::max<int64_t>(b->total_nq, 1))) != cudaSuccess ||
      (e = dev_malloc(reinterpret_cast<void**>(&E->mdO),
                      sizeof(double) * std::max<int64_t>(E->m_do, 1))) != cudaSuccess ||
      (e = dev_malloc(reinterpret_cast<void**>(&E->mdE),
                      sizeof(double) * std::max<int64_t>(E->m_de, 1))) != cudaSuccess)
    return e;
  if ((e = cudaFuncSetAttribute(batch_edges_mixed_kernel<kEaQc>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(sizeof(EdgeAdjSmem<kEaQc>)))) != cudaSuccess)
    return e;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, batch_edges_kernel<kAdjThreads, kAdjFpt, kAdjQc>, kAdjThreads, 0);
  E->grid = static_cast<int>(
      std::min<int64_t>(std::max(1, per_sm) * std::max(1, b->sms), std::max<int64_t>(E->n_items, 1)));
  return cudaGetLastError();
}

int64_t batch_boundary_edges(const BatchState* b) { return b->edges ? b->edges->ne_total : 0; }
int64_t batch_edge_items(const BatchState* b) {
  return b->edges ? (b->edges->fp64 ? b->edges->n_items : b->edges->m_items) : 0;
}
void batch_set_adjoint_fp64(BatchState* b, bool fp64) {
  if (b->edges) b->edges->fp64 = fp64;
}
bool batch_adjoint_fp64(const BatchState* b) { return b->edges && b->edges->fp64; }

void batch_edges_destroy(BatchState* b) {
  BatchEdges* E = b->edges;
  if (!E) return;
  void* ptrs[] = {E->ends,     E->mult,       E->edges,     E->dedge,      E->indptr,
                  E->entries,  E->items,      E->meshes,    E->query_mesh, E->edge_mesh,
                  E->counter,  E->dO_part,    E->dE_part,   E->tile_first, E->tile_count,
                  E->tile_mesh, E->mmeshes,   E->mitems,    E->mid,        E->box,
                  E->keys_in,  E->keys_out,   E->vals_in,   E->eperm,      E->qperm,
                  E->temp,     E->tiles,      E->e64,       E->edge_of,    E->qs,
                  E->mdO,      E->mdE};
  for (void* p : ptrs) cudaFree(p);
  delete E;
  b->edges = nullptr;
}

cudaError_t batch_backward(BatchState* b, const double* V, const double* q, const double* gw,
                           double* dq, double* dV, cudaStream_t stream) {
  BatchEdges* E = b->edges;
  if (!E) return cudaErrorInvalidValue;
  cudaError_t e;
  if (b->total_nq > 0 &&
      (e = cudaMemsetAsync(dq, 0, sizeof(double) * 3 * b->total_nq, stream)) != cudaSuccess)
    return e;
  if (b->total_nv > 0 &&
      (e = cudaMemsetAsync(dV, 0, sizeof(double) * 3 * b->total_nv, stream)) != cudaSuccess)
    return e;
  if (E->ne_total == 0 || b->total_nq == 0) return cudaSuccess;
  batch_edge_positions_kernel<<<static_cast<unsigned>(cdiv(E->ne_total, 256)), 256, 0, stream>>>(
      V, E->ends, E->mult, E->ne_total, E->le, E->edges);
  if (!E->fp64) {
    // Mixed: each mesh's edges and queries in their own Morton order, 64-edge tiles,
    // then (range, group) items with fixed-order sums as the single-mesh path.
    edge_midpoints_kernel<<<static_cast<unsigned>(cdiv(E->ne_total, 256)), 256, 0, stream>>>(
        E->edges, E->le, E->ne_total, E->mid);
    if ((e = batch_morton_order(E->mid, E->ne_total, E->edge_mesh, b->nmesh, b->mesh_bits,
                                E->box, E->keys_in, E->keys_out, E->vals_in, E->eperm, E->temp,
                                E->temp_bytes, stream)) != cudaSuccess)
      return e;
    build_edge_tiles_kernel<<<static_cast<unsigned>(E->nt), kTileFaces, 0, stream>>>(
        E->edges, E->le, E->ne_total, E->eperm, b->plan.kappa, E->tiles, E->e64,
        E->nt * kTileFaces, E->edge_of, E->tile_first, E->tile_count);
    if ((e = batch_morton_order(q, b->total_nq, E->query_mesh, b->nmesh, b->mesh_bits, E->box,
                                E->keys_in, E->keys_out, E->vals_in, E->qperm, E->temp,
                                E->temp_bytes, stream)) != cudaSuccess)
      return e;
    gather_sorted_queries_kernel<<<static_cast<unsigned>(cdiv(b->total_nq, 256)), 256, 0,
                                   stream>>>(q, gw, E->qperm, b->total_nq, E->qs);
    if ((e = cudaMemsetAsync(E->mdO, 0, sizeof(double) * std::max<int64_t>(E->m_do, 1),
                             stream)) != cudaSuccess)
      return e;
    const double kappa = b->plan.kappa;
    BatchMixedArgs ma{E->mitems, E->tiles, E->e64, E->nt * kTileFaces, E->qs,
                      static_cast<float>(kappa * kappa), E->mdO, E->mdE};
    if (E->m_items > 0)
      batch_edges_mixed_kernel<kEaQc>
          <<<static_cast<unsigned>(E->m_items), kFaThreads,
             static_cast<int>(sizeof(EdgeAdjSmem<kEaQc>)), stream>>>(ma);
    batch_mixed_finish_dq_kernel<<<static_cast<unsigned>(cdiv(3 * b->total_nq, 256)), 256, 0,
                                   stream>>>(E->mdO, E->mmeshes, E->query_mesh, E->qperm,
                                             b->total_nq, dq);
    batch_mixed_finish_dedge_kernel<<<static_cast<unsigned>(cdiv(6 * E->nt * kTileFaces, 256)),
                                      256, 0, stream>>>(E->mdE, E->mmeshes, E->tile_mesh,
                                                        E->edge_of, E->nt, E->le, E->dedge);
    gather_vertex_kernel<<<static_cast<unsigned>(cdiv(b->total_nv, 256)), 256, 0, stream>>>(
        E->dedge, E->le, 2, E->indptr, E->entries, b->total_nv, dV);
    g_launches.fetch_add(E->m_items > 0 ? 7 : 6, std::memory_order_relaxed);
    return cudaGetLastError();
  }
  if ((e = cudaMemsetAsync(E->dO_part, 0, sizeof(double) * std::max<int64_t>(E->do_doubles, 1),
                           stream)) != cudaSuccess ||
      (e = cudaMemsetAsync(E->counter, 0, sizeof(unsigned int), stream)) != cudaSuccess)
    return e;
  BatchEdgeArgs a{E->edges, E->le, q, gw, E->items, E->n_items, E->counter, E->dO_part,
                  E->dE_part};
  if (E->n_items > 0)
    batch_edges_kernel<kAdjThreads, kAdjFpt, kAdjQc><<<E->grid, kAdjThreads, 0, stream>>>(a);
  batch_finish_dq_kernel<<<static_cast<unsigned>(cdiv(3 * b->total_nq, 256)), 256, 0, stream>>>(
      E->dO_part, E->meshes, E->query_mesh, b->total_nq, dq);
  batch_finish_dedge_kernel<<<static_cast<unsigned>(cdiv(6 * E->ne_total, 256)), 256, 0,
                              stream>>>(E->dE_part, E->meshes, E->edge_mesh, E->ne_total, E->le,
                                        E->dedge);
  gather_vertex_kernel<<<static_cast<unsigned>(cdiv(b->total_nv, 256)), 256, 0, stream>>>(
      E->dedge, E->le, 2, E->indptr, E->entries, b->total_nv, dV);
  g_launches.fetch_add(5, std::memory_order_relaxed);
  return cudaGetLastError();
}

}  // namespace wn
