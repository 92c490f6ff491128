// Data layout of the mixed-precision path (see wn_mixed.cu for the method).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace wn {

constexpr int kTileFaces = 64;  // faces per tile (the angle bound needs <= 64 at kappa >= 3)

// 64-byte tile header, FP64 geometry of the tile.
struct TileHeader {
  double cx, cy, cz;  // centre of the tile's vertex bounding box
  double far_r2;      // (r + kappa*h_tile)^2: queries at least this far need no refinement
  double scale;       // power of two ~ 1/r applied to the FP32 local coordinates
  int32_t n;          // faces in the tile (the last tile may be partial)
  int32_t first;      // reserved
  float r, h;         // tile radius and longest edge (diagnostics)
  int32_t pad[2];
};
static_assert(sizeof(TileHeader) == 64, "tile header is 64 bytes");

// Second 64-byte header: the tile's two 32-face halves (faces [0, 32) and
// [32, 64) of the tile), for kernels that test and sum each half on its own. In
// the tile's scaled FP32 frame: the centre of each half's vertex bounding box
// relative to the tile centre, and (r_half + kappa*h_half)^2 with the radius
// inflated past the frame's FP32 rounding (relative 1e-5 plus 1e-5), so a
// query tested "far" in FP32 has no near pair in that half.
struct HalfHeader {
  float cx[2], cy[2], cz[2];
  float far_r2[2];
  int32_t pad[8];
};
static_assert(sizeof(HalfHeader) == 64, "half header is 64 bytes");

constexpr int kHalfFaces = kTileFaces / 2;
constexpr int kTileHeaderBytes = static_cast<int>(sizeof(TileHeader) + sizeof(HalfHeader));

// 64-byte face record, FP32 tile-local scaled coordinates. With a = A - o the
// pair needs |a|^2, a.e1, a.e2 and a.n only: b = a + e1 and c = a + e2 give
// |b|^2 = |a|^2 + 2 a.e1 + |e1|^2, a.b = |a|^2 + a.e1, b.c = a.b + a.e2 + e1.e2, ...
struct FaceRec {
  float ax, ay, az;     // corner A minus centre, times scale
  float e1x, e1y, e1z;  // B - A (formed in FP64, then rounded)
  float e2x, e2y, e2z;  // C - A
  float nx, ny, nz;     // e1 x e2
  float e11, e22, e12;  // |e1|^2, |e2|^2, e1.e2
  float thr;            // (kappa*h_face*scale)^2; +inf for collapsed faces
};
static_assert(sizeof(FaceRec) == 64, "face record is 64 bytes");

constexpr int kTileBytes = static_cast<int>(kTileHeaderBytes + kTileFaces * sizeof(FaceRec));
static_assert(kTileBytes % 16 == 0, "bulk copies move multiples of 16 bytes");

// A prepared mesh. All pointers are device memory owned by the caller.
struct MixedMesh {
  int64_t nf = 0, ntiles = 0, ld64 = 0;
  double kappa = 4.0;
  unsigned char* tiles = nullptr;  // ntiles * kTileBytes, 16-byte aligned
  double* tri64 = nullptr;         // 9 x ld64 sorted FP64 soup (ld64 = ntiles*kTileFaces)
  uint32_t* face_of = nullptr;     // ld64: sorted slot -> input face (0xffffffff = padding)
  int tile_faces = 64;             // faces per far test and angle product of the mixed
                                   // forward: 64, or 32 (each half tile on its own)
  uint8_t* reuse = nullptr;        // ld64: per corner (2 bits) the previous face's equal corner
                                   // (0..2) or 3 = new; 0xff = padding. May be null.
};

inline int64_t mixed_tiles(int64_t nf) { return nf > 0 ? (nf + kTileFaces - 1) / kTileFaces : 1; }

// Device bytes of the prepared mesh arrays.
inline size_t mixed_tiles_bytes(int64_t nf) {
  return static_cast<size_t>(mixed_tiles(nf)) * kTileBytes;
}
inline size_t mixed_tri64_bytes(int64_t nf) {
  return static_cast<size_t>(mixed_tiles(nf)) * kTileFaces * 9 * sizeof(double);
}
inline size_t mixed_face_of_bytes(int64_t nf) {
  return static_cast<size_t>(mixed_tiles(nf)) * kTileFaces * sizeof(uint32_t);
}
inline size_t mixed_reuse_bytes(int64_t nf) {
  return static_cast<size_t>(mixed_tiles(nf)) * kTileFaces;
}

// Scratch needed by mixed_prepare_mesh (nf faces) and by mixed_forward (nq queries).
size_t mixed_sort_scratch_bytes(int64_t n);

cudaError_t mixed_prepare_mesh(const double* tri, int64_t ld, int64_t nf, double kappa,
                               MixedMesh* m, void* scratch, size_t scratch_bytes,
                               cudaStream_t stream);

// Face-range split of the kernel over grid.y when there are too few queries
// to fill the GPU; partial sums are added per query in split order.
struct MixedSplit {
  int64_t nsplit = 1;
  int64_t tiles_per_split = 0;
  int64_t partial_doubles = 0;  // nsplit * nq when nsplit > 1
};
MixedSplit plan_mixed(int64_t ntiles, int64_t nq, int sms);

// Morton order of the queries: perm[sorted position] = query index.
cudaError_t mixed_sort_queries(const double* q, int64_t nq, uint32_t* perm, void* scratch,
                               size_t scratch_bytes, cudaStream_t stream);

// The kernel on queries already ordered by perm. stats (nullable):
// [0] += pairs refined in FP64, [1] += careful (warp, tile) visits.
cudaError_t mixed_forward_sorted(const MixedMesh& m, const double* q, const uint32_t* perm,
                                 int64_t nq, double* w, const MixedSplit& split, double* partial,
                                 unsigned long long* stats, int* err, cudaStream_t stream);

// Sort + kernel with one scratch block of mixed_forward_scratch_bytes().
size_t mixed_forward_scratch_bytes(int64_t ntiles, int64_t nq, int sms);
cudaError_t mixed_forward(const MixedMesh& m, const double* q, int64_t nq, double* w,
                          void* scratch, size_t scratch_bytes, int sms,
                          unsigned long long* stats, int* err, cudaStream_t stream);

}  // namespace wn
