// ORACLE — test infrastructure only. Not part of the product library.
//
// CPU restatement of the reference's exact generalized winding number
// (lee101/mojo-libigl, src/capi.mojo:205-294, exported at capi.mojo:938-942).
// Only tests, the smoke check and bench.py's CPU-baseline / reference legs may
// load this library; the product path (libwn_b200.so) never links or calls it.
//
// What is restated, line for line in meaning:
//   * Triangle-soup SoA input `tri[(3*corner+axis)*nf + face]`
//     (python/igl/__init__.py:248-250, capi.mojo:218-226).
//   * Per pair: a,b,c = corner - o; la,lb,lc = |.|; det = a.(b x c) with the
//     reference's operand order; denom = la*lb*lc + (a.b)lc + (b.c)la + (c.a)lb;
//     angle = atan2(det, denom)   (capi.mojo:218-235).
//   * Accumulation structure: 4 partial accumulators x W lanes over the
//     4W-unrolled body, then a W-wide remainder loop into accumulator 0, then
//     ((t0+t1)+(t2+t3)).reduce_add(), then a scalar tail, then / (2*pi)
//     (capi.mojo:207-286). W = simd_width_of[float64] = 8 on AVX-512 hosts.
//   * reduce_add is taken as halving pairwise (lane i + lane i+W/2, repeated).
//   * No floating-point contraction (built with -ffp-contract=off): every
//     product and sum is rounded separately, as plain Mojo `*`/`+` are.
//   * atan2 and sqrt are the C library's (correctly rounded sqrt; glibc atan2).
//
// The closest-point query (`mli_aabb_squared_distance`) lives in
// aabb_oracle.cpp and the vertex normals (`mli_vertex_normals`) in
// normals_oracle.cpp, linked into the same library. The library also exports
// the reference's other nine `mli_*` C-ABI names (capi.mojo:923-1007) as no-ops,
// so the reference's own Python shim
// (python/igl/_lib.py:122-130, which resolves all thirteen names) can load this
// file through MOJO_LIBIGL_LIB and drive `mli_winding` unchanged.
#include <cmath>
#include <cstdint>

namespace {

constexpr int kW = 8;   // simd_width_of[DType.float64]() on AVX-512
constexpr int kL = 4;   // partial accumulators (capi.mojo:207-213)
constexpr double kPi = 3.14159265358979323846264338327950288;  // capi.mojo:14

// One (face, query) term, capi.mojo:218-235 (SIMD body) == 267-284 (tail).
inline void pair_terms(const double* tri, int64_t nf, int64_t fi, double ox, double oy,
                       double oz, double* det_out, double* denom_out) {
  const double ax = tri[fi] - ox;
  const double ay = tri[nf + fi] - oy;
  const double az = tri[2 * nf + fi] - oz;
  const double bx = tri[3 * nf + fi] - ox;
  const double by = tri[4 * nf + fi] - oy;
  const double bz = tri[5 * nf + fi] - oz;
  const double cx = tri[6 * nf + fi] - ox;
  const double cy = tri[7 * nf + fi] - oy;
  const double cz = tri[8 * nf + fi] - oz;
  const double la = std::sqrt(ax * ax + ay * ay + az * az);
  const double lb = std::sqrt(bx * bx + by * by + bz * bz);
  const double lc = std::sqrt(cx * cx + cy * cy + cz * cz);
  const double det =
      ax * (by * cz - bz * cy) - ay * (bx * cz - bz * cx) + az * (bx * cy - by * cx);
  double denom = la * lb * lc;
  denom += (ax * bx + ay * by + az * bz) * lc;
  denom += (bx * cx + by * cy + bz * cz) * la;
  denom += (cx * ax + cy * ay + cz * az) * lb;
  *det_out = det;
  *denom_out = denom;
}

inline double pair_angle(const double* tri, int64_t nf, int64_t fi, double ox, double oy,
                         double oz) {
  double det, denom;
  pair_terms(tri, nf, fi, ox, oy, oz, &det, &denom);
  return std::atan2(det, denom);
}

// capi.mojo:205-286. Each W-wide group's (det, denom) terms are formed first and
// their atan2 taken after, lane by lane: the same separately rounded operations as
// one pair at a time, so every angle is the same, while the term loop can run as W
// vector lanes. Multiversioned: the AVX-512 clone (W = 8 doubles per vector, the
// reference's simd_width_of[float64] there) runs on hosts that have it, the build's
// AVX2 baseline elsewhere; oracle_isa() says which one runs.
__attribute__((target_clones("avx512f", "default")))
double winding_one(const double* tri, double ox, double oy, double oz, int64_t nf) {
  double t[kL][kW];
  for (int l = 0; l < kL; ++l)
    for (int w = 0; w < kW; ++w) t[l][w] = 0.0;
  double det[kW], den[kW];
  auto group = [&](int64_t at, double* acc) {
    for (int w = 0; w < kW; ++w) pair_terms(tri, nf, at + w, ox, oy, oz, &det[w], &den[w]);
    for (int w = 0; w < kW; ++w) acc[w] += std::atan2(det[w], den[w]);
  };
  int64_t fi = 0;
  while (fi + kL * kW <= nf) {  // capi.mojo:215-244
    for (int l = 0; l < kL; ++l) group(fi + l * kW, t[l]);
    fi += kL * kW;
  }
  while (fi + kW <= nf) {  // capi.mojo:245-264
    group(fi, t[0]);
    fi += kW;
  }
  // capi.mojo:265: ((totals + totals1) + (totals2 + totals3)).reduce_add()
  double s[kW];
  for (int w = 0; w < kW; ++w) s[w] = (t[0][w] + t[1][w]) + (t[2][w] + t[3][w]);
  for (int width = kW / 2; width >= 1; width /= 2)
    for (int w = 0; w < width; ++w) s[w] = s[w] + s[w + width];
  double total = s[0];
  while (fi < nf) {  // capi.mojo:266-285
    total += pair_angle(tri, nf, fi, ox, oy, oz);
    fi += 1;
  }
  return total / (2.0 * kPi);  // capi.mojo:286
}

}  // namespace

extern "C" {

// capi.mojo:289-294 (`winding`) behind capi.mojo:938-942 (`mli_winding`).
void mli_winding(int64_t tri, int64_t q, int64_t dst, int64_t nf, int64_t nq, int64_t q0,
                 int64_t q1) {
  (void)nq;
  const double* t = reinterpret_cast<const double*>(tri);
  const double* qq = reinterpret_cast<const double*>(q);
  double* d = reinterpret_cast<double*>(dst);
  for (int64_t qi = q0; qi < q1; ++qi)
    d[qi] = winding_one(t, qq[qi * 3], qq[qi * 3 + 1], qq[qi * 3 + 2], nf);
}

// The oracle has no GPU: report failure exactly as capi.mojo:397-398 does.
int64_t mli_winding_gpu(int64_t, int64_t, int64_t, int64_t, int64_t) { return 0; }

// The remaining reference exports (capi.mojo:923-932, 962-1007): out of scope,
// present only so the reference shim's loader finds every name.
void mli_cot_entries(int64_t, int64_t, int64_t, int64_t, int64_t) {}
void mli_mass_contributions(int64_t, int64_t, int64_t, int64_t, int64_t, int64_t) {}
void mli_heat_vector_divergence(int64_t, int64_t, int64_t, int64_t, int64_t, int64_t) {}
void mli_heat_precompute(int64_t, int64_t, int64_t, int64_t) {}
void mli_arap_covariance(int64_t, int64_t, int64_t, int64_t, int64_t, int64_t, int64_t,
                         int64_t) {}
void mli_arap_rhs(int64_t, int64_t, int64_t, int64_t, int64_t, int64_t, int64_t, int64_t) {}
void mli_arap_covariance_rims(int64_t, int64_t, int64_t, int64_t, int64_t, int64_t, int64_t,
                              int64_t) {}
void mli_arap_rhs_rims(int64_t, int64_t, int64_t, int64_t, int64_t, int64_t, int64_t,
                       int64_t) {}
void mli_arap_rotations(int64_t, int64_t, int64_t, int64_t, int64_t, int64_t) {}

// Which clone of winding_one this host runs: 512 (AVX-512) or 256 (AVX2 baseline).
int oracle_isa(void) {
  __builtin_cpu_init();
  return __builtin_cpu_supports("avx512f") ? 512 : 256;
}

// Oracle extras (no reference counterpart): per-pair term, exposed so tests can
// compare single (det, denom, angle) triples bit-for-bit with the GPU kernel.
void oracle_pair_terms(const double* tri, int64_t nf, int64_t fi, const double* o,
                       double* det_denom_angle) {
  pair_terms(tri, nf, fi, o[0], o[1], o[2], &det_denom_angle[0], &det_denom_angle[1]);
  det_denom_angle[2] = std::atan2(det_denom_angle[0], det_denom_angle[1]);
}

}  // extern "C"
