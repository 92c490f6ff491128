// Host (device="cpu") path of libwn_b200: `mli_winding`, the C-ABI entry the
// reference exports from src/capi.mojo:938-942 (kernel at capi.mojo:205-294).
//
// Same contract as the reference: fill dst[q0:q1) for queries q0..q1-1 of the
// (9, nf) triangle-soup SoA; reentrant over disjoint spans, so the Python shim
// can fan spans out over threads with the GIL released. The pair terms are
// the shared bit-exact ones (wn_pair.cuh; this file is built with
// -ffp-contract=off) and the angles are summed with the argument-of-product
// accumulator, with plain atan2 as the recovery path for a bad accumulator.
// Queries go 8 (AVX-512) or 4 (AVX2) per vector; on meshes the AVX-512 path
// computes each distinct corner position's |v - o| once per block of queries
// (see "corners shared between faces"). Every result is the scalar routine's.
#include <immintrin.h>

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "wn_pair.cuh"

namespace {

double winding_query(const double* tri, int64_t nf, double ox, double oy, double oz) {
  wn::ArgAcc acc;
  wn::argacc_init(acc);
  for (int64_t f = 0; f < nf; ++f) {
    double det, denom;
    wn::pair_terms_exact(ox, oy, oz, tri[f], tri[nf + f], tri[2 * nf + f], tri[3 * nf + f],
                         tri[4 * nf + f], tri[5 * nf + f], tri[6 * nf + f], tri[7 * nf + f],
                         tri[8 * nf + f], det, denom);
    wn::argacc_push(acc, denom, det);
  }
  double angle;
  if (!acc.bad) {
    angle = std::atan2(acc.zi, acc.zr) + static_cast<double>(acc.k) * wn::kTwoPi;
  } else {
    angle = 0.0;
    for (int64_t f = 0; f < nf; ++f) {
      double det, denom;
      wn::pair_terms_exact(ox, oy, oz, tri[f], tri[nf + f], tri[2 * nf + f], tri[3 * nf + f],
                           tri[4 * nf + f], tri[5 * nf + f], tri[6 * nf + f], tri[7 * nf + f],
                           tri[8 * nf + f], det, denom);
      angle += std::atan2(det, denom);
    }
  }
  return angle / wn::kTwoPi;
}

// ---- four queries at a time (AVX2) -----------------------------------------
// The same operations as winding_query, in the same order, on four queries
// (one per 64-bit lane) against each face: IEEE adds, multiplies and square
// roots round the same in a vector lane as in a scalar register, and this file
// is built without FMA contraction, so every lane's pair terms, products,
// turn count and result are the bits winding_query gives for that query.

struct Acc4 {
  __m256d zr, zi;
  __m256i k, bad;
};

inline __m256i bits(__m256d x) { return _mm256_castpd_si256(x); }

// wn::argacc_push on four lanes.
inline void push4(Acc4& s, __m256d d, __m256d t) {
  const __m256i sign = _mm256_set1_epi64x(static_cast<int64_t>(0x8000000000000000ULL));
  const __m256i zero = _mm256_setzero_si256();
  // Both +-0: use (copysign(1, d), t).
  const __m256i both0 =
      _mm256_cmpeq_epi64(_mm256_andnot_si256(sign, _mm256_or_si256(bits(d), bits(t))), zero);
  const __m256d one = _mm256_or_pd(_mm256_castsi256_pd(_mm256_and_si256(bits(d), sign)),
                                   _mm256_set1_pd(1.0));
  d = _mm256_blendv_pd(d, one, _mm256_castsi256_pd(both0));
  const __m256d nr = _mm256_sub_pd(_mm256_mul_pd(s.zr, d), _mm256_mul_pd(s.zi, t));
  const __m256d ni = _mm256_add_pd(_mm256_mul_pd(s.zr, t), _mm256_mul_pd(s.zi, d));
  // Turn count: the imaginary part kept its sign s0 = sign(t) but the product's
  // flipped, so the running argument crossed the negative real axis.
  const __m256i s0 = _mm256_cmpgt_epi64(zero, bits(s.zi));
  const __m256i st = _mm256_cmpgt_epi64(zero, bits(t));
  const __m256i s1 = _mm256_cmpgt_epi64(zero, bits(ni));
  const __m256i cross = _mm256_andnot_si256(_mm256_xor_si256(s0, st), _mm256_xor_si256(s0, s1));
  const __m256i delta = _mm256_or_si256(s0, _mm256_set1_epi64x(1));  // -1 if s0, else +1
  s.k = _mm256_add_epi64(s.k, _mm256_and_si256(cross, delta));
  // Rescale by 2^(1023 - e), e the biased exponent of the larger component.
  const __m256i emask = _mm256_set1_epi64x(0x7ff0000000000000LL);
  const __m256i er = _mm256_and_si256(bits(nr), emask), ei = _mm256_and_si256(bits(ni), emask);
  const __m256i e = _mm256_blendv_epi8(er, ei, _mm256_cmpgt_epi64(ei, er));
  s.bad = _mm256_or_si256(s.bad, _mm256_or_si256(_mm256_cmpeq_epi64(e, zero),
                                                 _mm256_cmpeq_epi64(e, emask)));
  const __m256d scale =
      _mm256_castsi256_pd(_mm256_sub_epi64(_mm256_set1_epi64x(0x7fe0000000000000LL), e));
  s.zr = _mm256_mul_pd(nr, scale);
  s.zi = _mm256_mul_pd(ni, scale);
}

struct Corner4 {
  __m256d x, y, z, l;
};

// wn::corner_exact on four lanes: v - o and its length.
inline Corner4 corner4(__m256d ox, __m256d oy, __m256d oz, double vx, double vy, double vz) {
  Corner4 c;
  c.x = _mm256_sub_pd(_mm256_set1_pd(vx), ox);
  c.y = _mm256_sub_pd(_mm256_set1_pd(vy), oy);
  c.z = _mm256_sub_pd(_mm256_set1_pd(vz), oz);
  c.l = _mm256_sqrt_pd(_mm256_add_pd(_mm256_add_pd(_mm256_mul_pd(c.x, c.x),
                                                   _mm256_mul_pd(c.y, c.y)),
                                     _mm256_mul_pd(c.z, c.z)));
  return c;
}

inline __m256d dot4(const Corner4& a, const Corner4& b) {
  return _mm256_add_pd(_mm256_add_pd(_mm256_mul_pd(a.x, b.x), _mm256_mul_pd(a.y, b.y)),
                       _mm256_mul_pd(a.z, b.z));
}

// wn::face_exact on four lanes.
inline void face4(const Corner4& a, const Corner4& b, const Corner4& c, __m256d& det,
                  __m256d& denom) {
  const __m256d t0 = _mm256_mul_pd(
      a.x, _mm256_sub_pd(_mm256_mul_pd(b.y, c.z), _mm256_mul_pd(b.z, c.y)));
  const __m256d t1 = _mm256_mul_pd(
      a.y, _mm256_sub_pd(_mm256_mul_pd(b.x, c.z), _mm256_mul_pd(b.z, c.x)));
  const __m256d t2 = _mm256_mul_pd(
      a.z, _mm256_sub_pd(_mm256_mul_pd(b.x, c.y), _mm256_mul_pd(b.y, c.x)));
  det = _mm256_add_pd(_mm256_sub_pd(t0, t1), t2);
  __m256d d = _mm256_mul_pd(_mm256_mul_pd(a.l, b.l), c.l);
  d = _mm256_add_pd(d, _mm256_mul_pd(dot4(a, b), c.l));
  d = _mm256_add_pd(d, _mm256_mul_pd(dot4(b, c), a.l));
  d = _mm256_add_pd(d, _mm256_mul_pd(dot4(c, a), b.l));
  denom = d;
}

// W of queries q[0..3] (AoS, 12 doubles) into out[0..3].
void winding_query4(const double* tri, int64_t nf, const double* q, double* out) {
  const __m256d ox = _mm256_set_pd(q[9], q[6], q[3], q[0]);
  const __m256d oy = _mm256_set_pd(q[10], q[7], q[4], q[1]);
  const __m256d oz = _mm256_set_pd(q[11], q[8], q[5], q[2]);
  Acc4 acc{_mm256_set1_pd(1.0), _mm256_setzero_pd(), _mm256_setzero_si256(),
           _mm256_setzero_si256()};
  for (int64_t f = 0; f < nf; ++f) {
    const Corner4 a = corner4(ox, oy, oz, tri[f], tri[nf + f], tri[2 * nf + f]);
    const Corner4 b = corner4(ox, oy, oz, tri[3 * nf + f], tri[4 * nf + f], tri[5 * nf + f]);
    const Corner4 c = corner4(ox, oy, oz, tri[6 * nf + f], tri[7 * nf + f], tri[8 * nf + f]);
    __m256d det, denom;
    face4(a, b, c, det, denom);
    push4(acc, denom, det);
  }
  alignas(32) double zr[4], zi[4];
  alignas(32) int64_t k[4], bad[4];
  _mm256_store_pd(zr, acc.zr);
  _mm256_store_pd(zi, acc.zi);
  _mm256_store_si256(reinterpret_cast<__m256i*>(k), acc.k);
  _mm256_store_si256(reinterpret_cast<__m256i*>(bad), acc.bad);
  for (int j = 0; j < 4; ++j)
    out[j] = bad[j] ? winding_query(tri, nf, q[3 * j], q[3 * j + 1], q[3 * j + 2])
                    : (std::atan2(zi[j], zr[j]) + static_cast<double>(k[j]) * wn::kTwoPi) /
                          wn::kTwoPi;
}

// ---- eight queries at a time (AVX-512, chosen at run time) ------------------
// The same lane-wise operations as winding_query4 on eight lanes.

#define WN_AVX512 __attribute__((target("avx512f,avx512dq")))

struct Acc8 {
  __m512d zr, zi;
  __m512i k;
  __mmask8 bad;
};

WN_AVX512 inline __m512i bits8(__m512d x) { return _mm512_castpd_si512(x); }

WN_AVX512 inline void push8(Acc8& s, __m512d d, __m512d t) {
  const __m512i sign = _mm512_set1_epi64(static_cast<int64_t>(0x8000000000000000ULL));
  const __m512i zero = _mm512_setzero_si512();
  const __mmask8 both0 =
      _mm512_cmpeq_epi64_mask(_mm512_andnot_si512(sign, _mm512_or_si512(bits8(d), bits8(t))), zero);
  const __m512d one = _mm512_castsi512_pd(
      _mm512_or_si512(_mm512_and_si512(bits8(d), sign), bits8(_mm512_set1_pd(1.0))));
  d = _mm512_mask_blend_pd(both0, d, one);
  const __m512d nr = _mm512_sub_pd(_mm512_mul_pd(s.zr, d), _mm512_mul_pd(s.zi, t));
  const __m512d ni = _mm512_add_pd(_mm512_mul_pd(s.zr, t), _mm512_mul_pd(s.zi, d));
  const __mmask8 s0 = _mm512_cmplt_epi64_mask(bits8(s.zi), zero);
  const __mmask8 st = _mm512_cmplt_epi64_mask(bits8(t), zero);
  const __mmask8 s1 = _mm512_cmplt_epi64_mask(bits8(ni), zero);
  const __mmask8 cross = static_cast<__mmask8>(~(s0 ^ st) & (s0 ^ s1));
  const __m512i delta = _mm512_mask_blend_epi64(s0, _mm512_set1_epi64(1), _mm512_set1_epi64(-1));
  s.k = _mm512_mask_add_epi64(s.k, cross, s.k, delta);
  const __m512i emask = _mm512_set1_epi64(0x7ff0000000000000LL);
  const __m512i er = _mm512_and_si512(bits8(nr), emask), ei = _mm512_and_si512(bits8(ni), emask);
  const __m512i e = _mm512_max_epi64(er, ei);
  s.bad = static_cast<__mmask8>(s.bad | _mm512_cmpeq_epi64_mask(e, zero) |
                                _mm512_cmpeq_epi64_mask(e, emask));
  const __m512d scale =
      _mm512_castsi512_pd(_mm512_sub_epi64(_mm512_set1_epi64(0x7fe0000000000000LL), e));
  s.zr = _mm512_mul_pd(nr, scale);
  s.zi = _mm512_mul_pd(ni, scale);
}

struct Corner8 {
  __m512d x, y, z, l;
};

WN_AVX512 inline Corner8 corner8(__m512d ox, __m512d oy, __m512d oz, double vx, double vy,
                                 double vz) {
  Corner8 c;
  c.x = _mm512_sub_pd(_mm512_set1_pd(vx), ox);
  c.y = _mm512_sub_pd(_mm512_set1_pd(vy), oy);
  c.z = _mm512_sub_pd(_mm512_set1_pd(vz), oz);
  c.l = _mm512_sqrt_pd(_mm512_add_pd(_mm512_add_pd(_mm512_mul_pd(c.x, c.x),
                                                   _mm512_mul_pd(c.y, c.y)),
                                     _mm512_mul_pd(c.z, c.z)));
  return c;
}

WN_AVX512 inline __m512d dot8(const Corner8& a, const Corner8& b) {
  return _mm512_add_pd(_mm512_add_pd(_mm512_mul_pd(a.x, b.x), _mm512_mul_pd(a.y, b.y)),
                       _mm512_mul_pd(a.z, b.z));
}

WN_AVX512 inline void face8(const Corner8& a, const Corner8& b, const Corner8& c, __m512d& det,
                            __m512d& denom) {
  const __m512d t0 = _mm512_mul_pd(
      a.x, _mm512_sub_pd(_mm512_mul_pd(b.y, c.z), _mm512_mul_pd(b.z, c.y)));
  const __m512d t1 = _mm512_mul_pd(
      a.y, _mm512_sub_pd(_mm512_mul_pd(b.x, c.z), _mm512_mul_pd(b.z, c.x)));
  const __m512d t2 = _mm512_mul_pd(
      a.z, _mm512_sub_pd(_mm512_mul_pd(b.x, c.y), _mm512_mul_pd(b.y, c.x)));
  det = _mm512_add_pd(_mm512_sub_pd(t0, t1), t2);
  __m512d d = _mm512_mul_pd(_mm512_mul_pd(a.l, b.l), c.l);
  d = _mm512_add_pd(d, _mm512_mul_pd(dot8(a, b), c.l));
  d = _mm512_add_pd(d, _mm512_mul_pd(dot8(b, c), a.l));
  d = _mm512_add_pd(d, _mm512_mul_pd(dot8(c, a), b.l));
  denom = d;
}

// W of queries q[0..7] (AoS, 24 doubles) into out[0..7].
WN_AVX512 void winding_query8(const double* tri, int64_t nf, const double* q, double* out) {
  const __m512i idx = _mm512_set_epi64(21, 18, 15, 12, 9, 6, 3, 0);
  const __m512d ox = _mm512_i64gather_pd(idx, q, 8);
  const __m512d oy = _mm512_i64gather_pd(idx, q + 1, 8);
  const __m512d oz = _mm512_i64gather_pd(idx, q + 2, 8);
  Acc8 acc{_mm512_set1_pd(1.0), _mm512_setzero_pd(), _mm512_setzero_si512(), 0};
  for (int64_t f = 0; f < nf; ++f) {
    const Corner8 a = corner8(ox, oy, oz, tri[f], tri[nf + f], tri[2 * nf + f]);
    const Corner8 b = corner8(ox, oy, oz, tri[3 * nf + f], tri[4 * nf + f], tri[5 * nf + f]);
    const Corner8 c = corner8(ox, oy, oz, tri[6 * nf + f], tri[7 * nf + f], tri[8 * nf + f]);
    __m512d det, denom;
    face8(a, b, c, det, denom);
    push8(acc, denom, det);
  }
  alignas(64) double zr[8], zi[8];
  alignas(64) int64_t k[8];
  _mm512_store_pd(zr, acc.zr);
  _mm512_store_pd(zi, acc.zi);
  _mm512_store_si512(k, acc.k);
  for (int j = 0; j < 8; ++j)
    out[j] = ((acc.bad >> j) & 1)
                 ? winding_query(tri, nf, q[3 * j], q[3 * j + 1], q[3 * j + 2])
                 : (std::atan2(zi[j], zr[j]) + static_cast<double>(k[j]) * wn::kTwoPi) /
                       wn::kTwoPi;
}

// ---- corners shared between faces (AVX-512) ---------------------------------
// A corner's a = v - o and |a| depend only on the vertex position and the
// query, and a mesh gives most positions to several faces (about six in a
// closed triangle mesh), while the soup repeats each position per face. The
// faces are taken in chunks of consecutive faces; each chunk lists its distinct
// corner positions (bitwise-equal coordinates) once, and for every block of
// eight queries the chunk's lengths |a| are computed once per distinct position
// and read back by every face that uses it. They are the same square roots of
// the same sums, and each query still multiplies its faces' factors in face
// order, so every bit of the result is unchanged, with a fraction of the
// square roots (the slowest vector instruction of the pair). A mesh of up to
// kWholeMeshFaces faces with at most kWholeMeshPositions positions is one chunk
// (its lengths, 64 bytes per position, stay in L2); a larger one is cut into
// chunks of kChunkFaces, which shares positions where the face order keeps
// neighbours together (a height field's rows, not every mesh).

constexpr int64_t kChunkFaces = 2048;
constexpr int64_t kWholeMeshFaces = 1 << 16;
constexpr int64_t kWholeMeshPositions = 1 << 14;

// Distinct corner positions of one chunk of faces. Sized once for the largest
// chunk, so listing a chunk allocates nothing.
struct ChunkPositions {
  std::vector<double> pos;   // 3 doubles per distinct position
  std::vector<uint32_t> id;  // corner 3 * (f - f0) + k -> its position's index
  std::vector<uint32_t> stamp, slot_id;
  uint32_t slots = 0, gen = 0;
  int64_t count = 0;

  explicit ChunkPositions(int64_t faces) {
    slots = 64;
    while (slots < 6 * faces) slots *= 2;  // an open-addressing table at most half full
    pos.resize(9 * static_cast<size_t>(faces));
    id.resize(3 * static_cast<size_t>(faces));
    stamp.assign(slots, 0);
    slot_id.resize(slots);
  }
};

inline uint64_t word(double x) {
  uint64_t u;
  std::memcpy(&u, &x, 8);
  return u;
}

// Lists the distinct corner positions of faces [f0, f1) into cp.
void list_chunk(const double* tri, int64_t nf, int64_t f0, int64_t f1, ChunkPositions& cp) {
  const uint32_t gen = ++cp.gen;  // invalidates the previous chunk's table entries
  const uint32_t mask = cp.slots - 1;
  int64_t n = 0;
  for (int64_t f = f0; f < f1; ++f)
    for (int k = 0; k < 3; ++k) {
      const double x = tri[3 * k * nf + f], y = tri[(3 * k + 1) * nf + f],
                   z = tri[(3 * k + 2) * nf + f];
      const uint64_t bx = word(x), by = word(y), bz = word(z);
      uint64_t h = bx * 0x9E3779B97F4A7C15ULL ^ by * 0xC2B2AE3D27D4EB4FULL ^
                   bz * 0x165667B19E3779F9ULL;
      h ^= h >> 29;
      for (uint32_t slot = static_cast<uint32_t>(h) & mask;; slot = (slot + 1) & mask) {
        if (cp.stamp[slot] != gen) {  // a new position of this chunk
          cp.stamp[slot] = gen;
          cp.slot_id[slot] = static_cast<uint32_t>(n);
          cp.pos[3 * n] = x;
          cp.pos[3 * n + 1] = y;
          cp.pos[3 * n + 2] = z;
          cp.id[3 * (f - f0) + k] = static_cast<uint32_t>(n);
          ++n;
          break;
        }
        const double* p = &cp.pos[3 * static_cast<int64_t>(cp.slot_id[slot])];
        if (word(p[0]) == bx && word(p[1]) == by && word(p[2]) == bz) {
          cp.id[3 * (f - f0) + k] = cp.slot_id[slot];
          break;
        }
      }
    }
  cp.count = n;
}

// Chooses the chunks of the shared-corner path: cf faces per chunk, the first
// chunk listed in cp. Shared corners pay when the chunks hold fewer than 1.5
// distinct positions per face, half the corners (measured: at 0.67 per corner,
// with lengths beyond L1, they cost more than they save); false otherwise.
bool plan_shared(const double* tri, int64_t nf, ChunkPositions& cp, int64_t& cf) {
  cf = nf < kChunkFaces ? nf : kChunkFaces;
  cp = ChunkPositions(cf);  // its table sized for the chunk, so that it stays in cache
  list_chunk(tri, nf, 0, cf, cp);
  if (2 * cp.count < 3 * cf) return true;
  if (cf == nf || nf > kWholeMeshFaces) return false;
  cf = nf;
  cp = ChunkPositions(nf);
  list_chunk(tri, nf, 0, nf, cp);
  return cp.count <= kWholeMeshPositions && 2 * cp.count < 3 * nf;
}

// Faces [f0, f1) for the block of eight queries (ox, oy, oz) into acc: the
// chunk's lengths into len (8 doubles per position, 64-byte aligned), then the
// faces with their corners' lengths read back.
WN_AVX512 void chunk8(const double* tri, int64_t nf, int64_t f0, int64_t f1,
                      const ChunkPositions& cp, double* len, __m512d ox, __m512d oy, __m512d oz,
                      Acc8& acc) {
  const double* p = cp.pos.data();
  for (int64_t u = 0; u < cp.count; ++u)
    _mm512_store_pd(len + 8 * u, corner8(ox, oy, oz, p[3 * u], p[3 * u + 1], p[3 * u + 2]).l);
  const uint32_t* id = cp.id.data();
  for (int64_t f = f0; f < f1; ++f) {
    Corner8 v[3];
    for (int k = 0; k < 3; ++k) {
      v[k].x = _mm512_sub_pd(_mm512_set1_pd(tri[3 * k * nf + f]), ox);
      v[k].y = _mm512_sub_pd(_mm512_set1_pd(tri[(3 * k + 1) * nf + f]), oy);
      v[k].z = _mm512_sub_pd(_mm512_set1_pd(tri[(3 * k + 2) * nf + f]), oz);
      v[k].l = _mm512_load_pd(len + 8 * static_cast<int64_t>(id[3 * (f - f0) + k]));
    }
    __m512d det, denom;
    face8(v[0], v[1], v[2], det, denom);
    push8(acc, denom, det);
  }
}

// The blocks of eight queries q[0 .. 24 nb) against every face with shared
// corner lengths, into out[0 .. 8 nb). Chunks outermost, so that each chunk is
// listed once for all blocks. Returns false, having written nothing, when the
// mesh shares too few positions or its buffers cannot be allocated.
WN_AVX512 bool winding_blocks8_shared(const double* tri, int64_t nf, const double* q,
                                      int64_t nb, double* out) {
  const __m512i idx = _mm512_set_epi64(21, 18, 15, 12, 9, 6, 3, 0);
  try {
    ChunkPositions cp(0);
    int64_t cf = 0;
    if (!plan_shared(tri, nf, cp, cf)) return false;
    // Each block's accumulator between chunks: zr, zi, k and the bad mask as 32
    // 8-byte words (a plain aligned buffer: no vector of AVX-512 types in code
    // built for the baseline ISA).
    double* state = static_cast<double*>(std::aligned_alloc(64, 256 * static_cast<size_t>(nb)));
    // Lengths of one chunk's positions: at most three per face, or the whole
    // mesh's count when it is one chunk.
    const size_t npos = cf == nf ? static_cast<size_t>(cp.count) : 3 * static_cast<size_t>(cf);
    double* len = static_cast<double*>(std::aligned_alloc(64, 64 * (npos + 1)));
    if (!state || !len) {
      std::free(state);
      std::free(len);
      return false;
    }
    for (int64_t b = 0; b < nb; ++b) {
      _mm512_store_pd(state + 32 * b, _mm512_set1_pd(1.0));
      _mm512_store_pd(state + 32 * b + 8, _mm512_setzero_pd());
      _mm512_store_si512(state + 32 * b + 16, _mm512_setzero_si512());
      state[32 * b + 24] = 0.0;  // bad mask, as the low byte of the word's bits
    }
    for (int64_t f0 = 0; f0 < nf; f0 += cf) {
      const int64_t f1 = f0 + cf < nf ? f0 + cf : nf;
      if (f0 > 0) list_chunk(tri, nf, f0, f1, cp);
      for (int64_t b = 0; b < nb; ++b) {
        const double* qb = q + 24 * b;
        double* sb = state + 32 * b;
        uint64_t bad_word;
        std::memcpy(&bad_word, sb + 24, 8);
        Acc8 acc{_mm512_load_pd(sb), _mm512_load_pd(sb + 8), _mm512_load_si512(sb + 16),
                 static_cast<__mmask8>(bad_word)};
        chunk8(tri, nf, f0, f1, cp, len, _mm512_i64gather_pd(idx, qb, 8),
               _mm512_i64gather_pd(idx, qb + 1, 8), _mm512_i64gather_pd(idx, qb + 2, 8), acc);
        _mm512_store_pd(sb, acc.zr);
        _mm512_store_pd(sb + 8, acc.zi);
        _mm512_store_si512(sb + 16, acc.k);
        bad_word = acc.bad;
        std::memcpy(sb + 24, &bad_word, 8);
      }
    }
    std::free(len);
    for (int64_t b = 0; b < nb; ++b) {
      const double* qb = q + 24 * b;
      const double* sb = state + 32 * b;
      int64_t k[8];
      uint64_t bad_word;
      std::memcpy(k, sb + 16, 64);
      std::memcpy(&bad_word, sb + 24, 8);
      for (int j = 0; j < 8; ++j)
        out[8 * b + j] =
            ((bad_word >> j) & 1)
                ? winding_query(tri, nf, qb[3 * j], qb[3 * j + 1], qb[3 * j + 2])
                : (std::atan2(sb[8 + j], sb[j]) + static_cast<double>(k[j]) * wn::kTwoPi) /
                      wn::kTwoPi;
    }
    std::free(state);
    return true;
  } catch (const std::bad_alloc&) {
    return false;
  }
}

#undef WN_AVX512

bool has_avx512() {
  static const bool yes = __builtin_cpu_supports("avx512f") && __builtin_cpu_supports("avx512dq");
  return yes;
}

}  // namespace

extern "C" {

// Reference: src/capi.mojo:938-942 `mli_winding(tri, q, dst, nf, nq, q0, q1)`,
// every argument an int64 (pointers as host addresses, python/igl/_lib.py:22).
void mli_winding(int64_t tri, int64_t q, int64_t dst, int64_t nf, int64_t nq, int64_t q0,
                 int64_t q1) {
  (void)nq;
  const double* t = reinterpret_cast<const double*>(tri);
  const double* qq = reinterpret_cast<const double*>(q);
  double* d = reinterpret_cast<double*>(dst);
  int64_t qi = q0;
  if (has_avx512()) {
    const int64_t nb = (q1 - q0) / 8;
    if (nb > 0 && nf > 0 && winding_blocks8_shared(t, nf, qq + 3 * qi, nb, d + qi)) qi += 8 * nb;
    for (; qi + 8 <= q1; qi += 8) winding_query8(t, nf, qq + 3 * qi, d + qi);
  }
  for (; qi + 4 <= q1; qi += 4) winding_query4(t, nf, qq + 3 * qi, d + qi);
  for (; qi < q1; ++qi) d[qi] = winding_query(t, nf, qq[3 * qi], qq[3 * qi + 1], qq[3 * qi + 2]);
}

}  // extern "C"
