// Plain FP64 forward: the exact generalized winding number of a triangle soup.
//
// Replaces the reference's two-kernel GPU path (lee101/mojo-libigl,
// src/capi.mojo:297-398: one thread per (face, query) writing an nf x nq FP64
// angle buffer, then one thread per query summing it). Here one fused kernel:
//   * each CTA owns THREADS*QPT queries, QPT per thread, held in registers;
//   * the CTA streams the face SoA (9 rows x ld doubles) through a STAGES-deep
//     ring of shared-memory tiles filled by 1-D bulk copies (cp.async.bulk,
//     completion on an mbarrier; no cluster multicast);
//   * every thread evaluates its QPT queries against each face of the tile,
//     reading the face by shared-memory broadcast;
//   * pair terms are bit-identical to the reference (wn_pair.cuh); the angles
//     are summed either by the argument-of-product accumulator (default) or by
//     one atan2 per pair;
//   * no nf x nq buffer exists. When there are too few queries to fill the
//     GPU the face range is split over grid.y and a second kernel sums the
//     per-split partial angles in split order (deterministic, no atomics).
#include <algorithm>

#include "wn_common.cuh"
#include "wn_internal.h"
#include "wn_mixed.h"
#include "wn_pair.cuh"

namespace wn {
namespace {

struct Fp64Args {
  const double* tri;
  int64_t ld;
  int64_t nf;
  const double* q;
  int64_t nq;
  int64_t f_chunk;
  double* w;        // final output when gridDim.y == 1
  double* partial;  // [gridDim.y][nq] angle sums when gridDim.y > 1
  int* err;
};

// Sum of atan2 over faces [f_begin, f_end) read straight from global memory;
// the recovery path for an accumulator marked bad.
__device__ double direct_sum_global(const Fp64Args& a, int64_t f_begin, int64_t f_end, double ox,
                                    double oy, double oz) {
  double s = 0.0;
  for (int64_t f = f_begin; f < f_end; ++f) {
    const double* t = a.tri + f;
    double det, denom;
    pair_terms_exact(ox, oy, oz, t[0], t[a.ld], t[2 * a.ld], t[3 * a.ld], t[4 * a.ld],
                     t[5 * a.ld], t[6 * a.ld], t[7 * a.ld], t[8 * a.ld], det, denom);
    s += atan2(det, denom);
  }
  return s;
}

template <int THREADS, int QPT, int TF, int STAGES, int MODE>
__global__ void __launch_bounds__(THREADS) fp64_forward_kernel(const Fp64Args a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double* tiles = reinterpret_cast<double*>(smem_raw);  // [STAGES][9][TF]
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + sizeof(double) * STAGES * 9 * TF);

  const int tid = threadIdx.x;
  const int64_t q_base = static_cast<int64_t>(blockIdx.x) * (THREADS * QPT);
  const int64_t f_begin = static_cast<int64_t>(blockIdx.y) * a.f_chunk;
  const int64_t f_end = min(a.nf, f_begin + a.f_chunk);
  const int ntiles = f_end > f_begin ? static_cast<int>((f_end - f_begin + TF - 1) / TF) : 0;

  double ox[QPT], oy[QPT], oz[QPT];
#pragma unroll
  for (int k = 0; k < QPT; ++k) {
    const int64_t qi = q_base + tid + k * THREADS;
    const bool valid = qi < a.nq;
    ox[k] = valid ? a.q[3 * qi] : 0.0;
    oy[k] = valid ? a.q[3 * qi + 1] : 0.0;
    oz[k] = valid ? a.q[3 * qi + 2] : 0.0;
  }

  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(&full[s], 1);
    fence_barrier_init();
  }
  __syncthreads();

  // Tile t covers faces [f_begin + t*TF, +n); each of the 9 rows is one bulk
  // copy of round_up(n, 2) doubles. Alignment: ld and f_chunk are even and TF
  // is even, so every source offset is a multiple of 2 doubles (16 bytes).
  auto issue = [&](int t) {
    const int slot = t % STAGES;
    const int64_t f0 = f_begin + static_cast<int64_t>(t) * TF;
    const int64_t n = min(static_cast<int64_t>(TF), f_end - f0);
    const uint32_t bytes = static_cast<uint32_t>(((n + 1) & ~int64_t(1)) * sizeof(double));
    mbar_arrive_expect_tx(&full[slot], 9u * bytes);
#pragma unroll
    for (int r = 0; r < 9; ++r)
      bulk_g2s(tiles + (slot * 9 + r) * TF, a.tri + r * a.ld + f0, bytes, &full[slot]);
  };
  int issued = 0;
  if (tid == 0) {
    for (; issued < min(STAGES, ntiles); ++issued) issue(issued);
  }

  ArgAcc acc[QPT];
  double sum[QPT];
#pragma unroll
  for (int k = 0; k < QPT; ++k) {
    argacc_init(acc[k]);
    sum[k] = 0.0;
  }

  bool failed = false;
  int t = 0;
  for (; t < ntiles; ++t) {
    const int slot = t % STAGES;
    const bool landed = mbar_wait(&full[slot], (t / STAGES) & 1, a.err);
    // Every thread has finished tile t-1 past this barrier, so its slot is free.
    if (!__syncthreads_and(landed)) {
      failed = true;
      break;
    }
    if (tid == 0 && t >= 1 && issued < ntiles) issue(issued++);

    const double* s = tiles + slot * 9 * TF;
    const int64_t f0 = f_begin + static_cast<int64_t>(t) * TF;
    const int n = static_cast<int>(min(static_cast<int64_t>(TF), f_end - f0));
#pragma unroll 1
    for (int j = 0; j < n; ++j) {
      const double Ax = s[j], Ay = s[TF + j], Az = s[2 * TF + j];
      const double Bx = s[3 * TF + j], By = s[4 * TF + j], Bz = s[5 * TF + j];
      const double Cx = s[6 * TF + j], Cy = s[7 * TF + j], Cz = s[8 * TF + j];
#pragma unroll
      for (int k = 0; k < QPT; ++k) {
        double det, denom;
        pair_terms_exact(ox[k], oy[k], oz[k], Ax, Ay, Az, Bx, By, Bz, Cx, Cy, Cz, det, denom);
        if (MODE == kFp64ArgProd)
          argacc_push(acc[k], denom, det);
        else
          sum[k] += atan2(det, denom);
      }
    }
  }

  if (failed) {
    // Leave no bulk copy in flight into this CTA's shared memory.
    if (tid == 0)
      for (int u = t; u < issued; ++u) mbar_wait(&full[u % STAGES], (u / STAGES) & 1, nullptr);
    __syncthreads();
    return;
  }

#pragma unroll
  for (int k = 0; k < QPT; ++k) {
    const int64_t qi = q_base + tid + k * THREADS;
    if (qi >= a.nq) continue;
    double angle;
    if (MODE == kFp64ArgProd) {
      angle = acc[k].bad ? direct_sum_global(a, f_begin, f_end, ox[k], oy[k], oz[k])
                         : atan2(acc[k].zi, acc[k].zr) + static_cast<double>(acc[k].k) * kTwoPi;
    } else {
      angle = sum[k];
    }
    if (gridDim.y == 1)
      a.w[qi] = angle / kTwoPi;
    else
      a.partial[static_cast<int64_t>(blockIdx.y) * a.nq + qi] = angle;
  }
}

__global__ void sum_splits_kernel(const double* __restrict__ partial, int64_t nsplit, int64_t nq,
                                  double* __restrict__ w) {
  const int64_t qi = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (qi >= nq) return;
  double s = 0.0;
  for (int64_t y = 0; y < nsplit; ++y) s += partial[y * nq + qi];
  w[qi] = s / kTwoPi;
}

// ---- FP64 over a prepared mesh, with corner reuse ---------------------------
// Same bit-exact pair terms and argument-of-product sum, but the faces come from a
// prepared mesh (wn_mixed.cu): Morton-ordered 64-face tiles whose faces are
// ordered as strips, with a per-face code telling which corners equal a corner
// of the previous face. a = v - o and |a| (three subtractions, three products,
// two sums and a correctly rounded sqrt) depend only on the vertex and the
// query, so a repeated corner is copied instead of recomputed: the same bits,
// about 40% fewer FP64 instructions per pair on a typical mesh.
struct Fp64TiledArgs {
  const double* tri64;  // 9 x ld64, tile-major sorted soup
  int64_t ld64;
  const uint8_t* reuse;  // ld64 codes
  int64_t ntiles;
  const double* q;
  int64_t nq;
  int64_t tiles_per_split;
  double* w;
  double* partial;
  int* err;
};

constexpr int kFp64TileBytes = 9 * kTileFaces * 8 + kTileFaces;  // coordinates + codes

__device__ __forceinline__ Corner pick_corner(unsigned code, const Corner& c0, const Corner& c1,
                                              const Corner& c2) {
  return code == 0 ? c0 : (code == 1 ? c1 : c2);
}

// Corner `pos` of face j when its reuse code M is known at compile time: one of
// the previous face's corners (M = 0..2) or a new one computed from the tile.
template <unsigned M>
__device__ __forceinline__ Corner corner_of(const Corner& p0, const Corner& p1, const Corner& p2,
                                            double ox, double oy, double oz, const double* s,
                                            int pos, int j) {
  if constexpr (M == 3)
    return corner_exact(ox, oy, oz, s[(3 * pos) * kTileFaces + j],
                        s[(3 * pos + 1) * kTileFaces + j], s[(3 * pos + 2) * kTileFaces + j]);
  else if constexpr (M == 0)
    return p0;
  else if constexpr (M == 1)
    return p1;
  else
    return p2;
}

// The three corners of face j. The code is the same for every lane (all lanes
// walk the same face), so a switch over it is a uniform branch, and each case
// names its corners at compile time: no per-register selects. The cases are
// the 28 codes whose reused corners are distinct with at most two of them (a
// face that shares all three corners with the previous one is a duplicate and
// takes the generic path).
__device__ __forceinline__ void face_corners(unsigned code, const Corner& p0, const Corner& p1,
                                             const Corner& p2, double ox, double oy, double oz,
                                             const double* s, int j, Corner& c0, Corner& c1,
                                             Corner& c2) {
#define WN_FACE_CASE(A, B, C)                                 \
  case (A) | ((B) << 2) | ((C) << 4):                         \
    c0 = corner_of<A>(p0, p1, p2, ox, oy, oz, s, 0, j);       \
    c1 = corner_of<B>(p0, p1, p2, ox, oy, oz, s, 1, j);       \
    c2 = corner_of<C>(p0, p1, p2, ox, oy, oz, s, 2, j);       \
    return;
  switch (code) {
    WN_FACE_CASE(3, 3, 3)
    WN_FACE_CASE(0, 3, 3) WN_FACE_CASE(1, 3, 3) WN_FACE_CASE(2, 3, 3)
    WN_FACE_CASE(3, 0, 3) WN_FACE_CASE(3, 1, 3) WN_FACE_CASE(3, 2, 3)
    WN_FACE_CASE(3, 3, 0) WN_FACE_CASE(3, 3, 1) WN_FACE_CASE(3, 3, 2)
    WN_FACE_CASE(3, 0, 1) WN_FACE_CASE(3, 0, 2) WN_FACE_CASE(3, 1, 0)
    WN_FACE_CASE(3, 1, 2) WN_FACE_CASE(3, 2, 0) WN_FACE_CASE(3, 2, 1)
    WN_FACE_CASE(0, 3, 1) WN_FACE_CASE(0, 3, 2) WN_FACE_CASE(1, 3, 0)
    WN_FACE_CASE(1, 3, 2) WN_FACE_CASE(2, 3, 0) WN_FACE_CASE(2, 3, 1)
    WN_FACE_CASE(0, 1, 3) WN_FACE_CASE(0, 2, 3) WN_FACE_CASE(1, 0, 3)
    WN_FACE_CASE(1, 2, 3) WN_FACE_CASE(2, 0, 3) WN_FACE_CASE(2, 1, 3)
    default:
      break;
  }
#undef WN_FACE_CASE
  Corner c[3];
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    const unsigned cm = (code >> (2 * m)) & 3u;
    c[m] = cm == 3u ? corner_exact(ox, oy, oz, s[(3 * m) * kTileFaces + j],
                                   s[(3 * m + 1) * kTileFaces + j],
                                   s[(3 * m + 2) * kTileFaces + j])
                    : pick_corner(cm, p0, p1, p2);
  }
  c0 = c[0];
  c1 = c[1];
  c2 = c[2];
}

template <int THREADS, int QPT, int STAGES>
__global__ void __launch_bounds__(THREADS) fp64_tiled_kernel(const Fp64TiledArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* ring = smem_raw;  // [STAGES][kFp64TileBytes]
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + STAGES * kFp64TileBytes);
  const int tid = threadIdx.x;
  const int64_t q_base = static_cast<int64_t>(blockIdx.x) * (THREADS * QPT);
  const int64_t t_begin = static_cast<int64_t>(blockIdx.y) * a.tiles_per_split;
  const int64_t t_left = a.ntiles - t_begin < a.tiles_per_split ? a.ntiles - t_begin
                                                                 : a.tiles_per_split;
  const int ntiles = static_cast<int>(t_left > 0 ? t_left : 0);
  double ox[QPT], oy[QPT], oz[QPT];
#pragma unroll
  for (int k = 0; k < QPT; ++k) {
    const int64_t qi = q_base + k * THREADS + tid;
    const bool valid = qi < a.nq;
    ox[k] = valid ? a.q[3 * qi] : 0.0;
    oy[k] = valid ? a.q[3 * qi + 1] : 0.0;
    oz[k] = valid ? a.q[3 * qi + 2] : 0.0;
  }
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(&full[s], 1);
    fence_barrier_init();
  }
  __syncthreads();
  // Tile t: 9 coordinate rows of 64 doubles (512 bytes each, 16-byte aligned since
  // ld64 is a multiple of 64) and 64 reuse codes.
  auto issue = [&](int t) {
    const int slot = t % STAGES;
    unsigned char* dst = ring + slot * kFp64TileBytes;
    const int64_t base = (t_begin + t) * kTileFaces;
    mbar_arrive_expect_tx(&full[slot], kFp64TileBytes);
#pragma unroll
    for (int r = 0; r < 9; ++r)
      bulk_g2s(dst + r * kTileFaces * 8, a.tri64 + r * a.ld64 + base, kTileFaces * 8, &full[slot]);
    bulk_g2s(dst + 9 * kTileFaces * 8, a.reuse + base, kTileFaces, &full[slot]);
  };
  int issued = 0;
  if (tid == 0)
    for (; issued < min(STAGES, ntiles); ++issued) issue(issued);
  ArgAcc acc[QPT];
  Corner p0[QPT], p1[QPT], p2[QPT];
#pragma unroll
  for (int k = 0; k < QPT; ++k) {
    argacc_init(acc[k]);
    p0[k] = p1[k] = p2[k] = Corner{0, 0, 0, 0};
  }
  bool failed = false;
  int t = 0;
  for (; t < ntiles; ++t) {
    const int slot = t % STAGES;
    const bool landed = mbar_wait(&full[slot], (t / STAGES) & 1, a.err);
    if (!__syncthreads_and(landed)) {
      failed = true;
      break;
    }
    if (tid == 0 && t >= 1 && issued < ntiles) issue(issued++);
    const double* s = reinterpret_cast<const double*>(ring + slot * kFp64TileBytes);
    const uint8_t* codes = ring + slot * kFp64TileBytes + 9 * kTileFaces * 8;
#pragma unroll 1
    for (int j = 0; j < kTileFaces; ++j) {
      const unsigned code = codes[j];
      if (code == 0xffu) break;  // padding: the rest of the tile is empty
#pragma unroll
      for (int k = 0; k < QPT; ++k) {
        Corner c0, c1, c2;
        face_corners(code, p0[k], p1[k], p2[k], ox[k], oy[k], oz[k], s, j, c0, c1, c2);
        double det, denom;
        face_exact(c0, c1, c2, det, denom);
        argacc_push(acc[k], denom, det);
        p0[k] = c0;
        p1[k] = c1;
        p2[k] = c2;
      }
    }
  }
  if (failed) {
    if (tid == 0)
      for (int u = t; u < issued; ++u) mbar_wait(&full[u % STAGES], (u / STAGES) & 1, nullptr);
    __syncthreads();
    return;
  }
#pragma unroll
  for (int k = 0; k < QPT; ++k) {
    const int64_t qi = q_base + k * THREADS + tid;
    if (qi >= a.nq) continue;
    double angle;
    if (!acc[k].bad) {
      angle = atan2(acc[k].zi, acc[k].zr) + static_cast<double>(acc[k].k) * kTwoPi;
    } else {
      // Recovery: one atan2 per pair over this slice, from global memory.
      angle = 0.0;
      for (int64_t f = t_begin * kTileFaces; f < (t_begin + ntiles) * kTileFaces; ++f) {
        if (a.reuse[f] == 0xffu) continue;
        const double* v = a.tri64 + f;
        const int64_t L = a.ld64;
        double det, denom;
        pair_terms_exact(ox[k], oy[k], oz[k], v[0], v[L], v[2 * L], v[3 * L], v[4 * L],
                         v[5 * L], v[6 * L], v[7 * L], v[8 * L], det, denom);
        angle += atan2(det, denom);
      }
    }
    if (gridDim.y == 1)
      a.w[qi] = angle / kTwoPi;
    else
      a.partial[static_cast<int64_t>(blockIdx.y) * a.nq + qi] = angle;
  }
}

template <int THREADS, int QPT, int TF, int STAGES, int MODE>
cudaError_t launch_variant(const Fp64Plan& p, const Fp64Args& a, cudaStream_t stream) {
  auto kernel = fp64_forward_kernel<THREADS, QPT, TF, STAGES, MODE>;
  const size_t smem = sizeof(double) * STAGES * 9 * TF + sizeof(uint64_t) * STAGES;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  dim3 grid(static_cast<unsigned>(p.qblocks), static_cast<unsigned>(p.nsplit));
  kernel<<<grid, THREADS, smem, stream>>>(a);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError();
}

}  // namespace

Fp64Plan plan_fp64(int64_t nf, int64_t nq, int sms, int force_nsplit) {
  Fp64Plan p;
  const int64_t per_block = static_cast<int64_t>(p.threads) * p.qpt;
  p.qblocks = std::max<int64_t>(1, (nq + per_block - 1) / per_block);
  const int64_t tiles = std::max<int64_t>(1, (nf + p.tile_faces - 1) / p.tile_faces);
  // Aim for >= 4 resident-CTA waves' worth of CTAs across the SMs.
  const int64_t target = static_cast<int64_t>(std::max(sms, 1)) * 8;
  int64_t nsplit = 1;
  if (force_nsplit > 0)
    nsplit = force_nsplit;
  else if (p.qblocks < target)
    nsplit = (target + p.qblocks - 1) / p.qblocks;
  nsplit = std::max<int64_t>(1, std::min(nsplit, tiles));
  const int64_t tiles_per_split = (tiles + nsplit - 1) / nsplit;
  p.f_chunk = tiles_per_split * p.tile_faces;
  p.nsplit = std::max<int64_t>(1, (nf + p.f_chunk - 1) / p.f_chunk);
  p.scratch_doubles = p.nsplit > 1 ? p.nsplit * nq : 0;
  return p;
}

constexpr int kTiledThreads = 128, kTiledQpt = 1, kTiledStages = 4;

Fp64TiledPlan plan_fp64_tiled(int64_t ntiles, int64_t nq, int sms) {
  Fp64TiledPlan p;
  const int64_t per = static_cast<int64_t>(kTiledThreads) * kTiledQpt;
  const int64_t qblocks = std::max<int64_t>(1, (nq + per - 1) / per);
  const int64_t target = static_cast<int64_t>(std::max(sms, 1)) * 8;
  int64_t nsplit = qblocks < target ? (target + qblocks - 1) / qblocks : 1;
  nsplit = std::max<int64_t>(1, std::min(nsplit, std::max<int64_t>(ntiles, 1)));
  p.tiles_per_split = (std::max<int64_t>(ntiles, 1) + nsplit - 1) / nsplit;
  p.nsplit = std::max<int64_t>(1, (std::max<int64_t>(ntiles, 1) + p.tiles_per_split - 1) /
                                      p.tiles_per_split);
  p.qblocks = qblocks;
  p.scratch_doubles = p.nsplit > 1 ? p.nsplit * nq : 0;
  return p;
}

cudaError_t launch_fp64_tiled(const Fp64TiledPlan& p, const MixedMesh& m, const double* q,
                              int64_t nq, double* w, double* scratch, int* err,
                              cudaStream_t stream) {
  if (nq <= 0) return cudaSuccess;
  if (!m.reuse || (p.nsplit > 1 && !scratch) || p.nsplit > 65535)
    return cudaErrorInvalidValue;
  constexpr int kThreads = kTiledThreads, kStages = kTiledStages;
  Fp64TiledArgs a{m.tri64, m.ld64, m.reuse, m.ntiles, q, nq, p.tiles_per_split, w, scratch, err};
  auto kernel = fp64_tiled_kernel<kThreads, kTiledQpt, kStages>;
  const size_t smem = static_cast<size_t>(kStages) * kFp64TileBytes + sizeof(uint64_t) * kStages;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  kernel<<<dim3(static_cast<unsigned>(p.qblocks), static_cast<unsigned>(p.nsplit)), kThreads,
           smem, stream>>>(a);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if ((e = cudaGetLastError()) != cudaSuccess || p.nsplit == 1) return e;
  sum_splits_kernel<<<static_cast<unsigned>((nq + 255) / 256), 256, 0, stream>>>(scratch,
                                                                             p.nsplit, nq, w);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError();
}

cudaError_t launch_fp64(const Fp64Plan& p, int mode, const double* tri, int64_t ld, int64_t nf,
                        const double* q, int64_t nq, double* w, double* scratch, int* err,
                        cudaStream_t stream) {
  if (nq <= 0) return cudaSuccess;
  if ((ld & 1) || ld < nf || (p.f_chunk % p.tile_faces) || p.qblocks > 0x7fffffff ||
      p.nsplit > 65535 || (p.nsplit > 1 && scratch == nullptr) ||
      (reinterpret_cast<uintptr_t>(tri) & 15))
    return cudaErrorInvalidValue;
  Fp64Args a{tri, ld, nf, q, nq, p.f_chunk, w, scratch, err};
  cudaError_t e;
  if (p.threads != 128 || p.qpt != 2 || p.tile_faces != 128 || p.stages != 3)
    return cudaErrorInvalidConfiguration;
  if (mode == kFp64Direct)
    e = launch_variant<128, 2, 128, 3, kFp64Direct>(p, a, stream);
  else
    e = launch_variant<128, 2, 128, 3, kFp64ArgProd>(p, a, stream);
  if (e != cudaSuccess || p.nsplit == 1) return e;
  const int threads = 256;
  const int64_t blocks = (nq + threads - 1) / threads;
  sum_splits_kernel<<<static_cast<unsigned>(blocks), threads, 0, stream>>>(scratch, p.nsplit, nq,
                                                                          w);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError();
}

}  // namespace wn
