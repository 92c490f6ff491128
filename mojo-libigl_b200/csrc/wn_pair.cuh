// Per-pair arithmetic of the exact generalized winding number, shared by the
// CUDA kernels and the host (device="cpu") path of libwn_b200.
//
// For one query o and one triangle (A, B, C) the reference evaluates
// (lee101/mojo-libigl, src/capi.mojo:218-235):
//   a = A - o, b = B - o, c = C - o, la = |a|, lb = |b|, lc = |c|
//   det   = ax*(by*cz - bz*cy) - ay*(bx*cz - bz*cx) + az*(bx*cy - by*cx)
//   denom = la*lb*lc + (a.b)*lc + (b.c)*la + (c.a)*lb
//   angle = atan2(det, denom)           W(o) = sum(angle) / (2*pi)
// `pair_terms_exact` reproduces det and denom bit for bit: the same operand
// order, every product/sum rounded on its own (no FMA contraction: the
// __d*_rn intrinsics on the device; the host file is built with
// -ffp-contract=off), and a correctly rounded sqrt.
//
// `ArgAcc` sums the angles without one atan2 per pair. The angles of the
// complex numbers z_i = denom_i + i*det_i add under multiplication, so
//   sum_i atan2(det_i, denom_i) = arg(prod_i z_i) + 2*pi*K,
// where K counts how often the running product crosses the negative real axis.
// With "upper" meaning sign bit of the imaginary part clear (argument in
// [+0, pi]) and "lower" meaning it set (argument in [-pi, -0]), a crossing can
// only happen when the running product and the new factor lie in the same half
// plane and the product lands in the other one: K += 1 (both upper) or K -= 1
// (both lower). This uses the signed-zero convention of atan2 itself, so
// det = +-0 with denom < 0 contributes +-pi exactly as atan2 does, and
// z_i = (+-0, +-0) is replaced by the unit vector (copysign(1, denom), det),
// whose argument is atan2's value for that pair. After every factor the
// product is rescaled by an exact power of two (no rounding), keeping it in
// [1, 2); a factor that drives it to zero, subnormal, inf or NaN marks the
// accumulator bad and the caller recomputes that query with plain atan2.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

#if defined(__CUDACC__)
#define WN_HD __host__ __device__ __forceinline__
#else
#define WN_HD inline
#endif

namespace wn {

constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr double kTwoPi = 2.0 * kPi;

#if defined(__CUDA_ARCH__)
WN_HD double dmul(double a, double b) { return __dmul_rn(a, b); }
WN_HD double dadd(double a, double b) { return __dadd_rn(a, b); }
WN_HD double dsub(double a, double b) { return __dsub_rn(a, b); }
WN_HD double dsqrt(double a) { return __dsqrt_rn(a); }
WN_HD int32_t hi_word(double x) { return __double2hiint(x); }
WN_HD uint32_t lo_word(double x) { return static_cast<uint32_t>(__double2loint(x)); }
WN_HD double from_words(int32_t hi, uint32_t lo) {
  return __hiloint2double(hi, static_cast<int32_t>(lo));
}
#else
WN_HD double dmul(double a, double b) { return a * b; }
WN_HD double dadd(double a, double b) { return a + b; }
WN_HD double dsub(double a, double b) { return a - b; }
WN_HD double dsqrt(double a) { return std::sqrt(a); }
WN_HD int32_t hi_word(double x) {
  uint64_t u;
  std::memcpy(&u, &x, 8);
  return static_cast<int32_t>(u >> 32);
}
WN_HD uint32_t lo_word(double x) {
  uint64_t u;
  std::memcpy(&u, &x, 8);
  return static_cast<uint32_t>(u);
}
WN_HD double from_words(int32_t hi, uint32_t lo) {
  const uint64_t u = (static_cast<uint64_t>(static_cast<uint32_t>(hi)) << 32) | lo;
  double x;
  std::memcpy(&x, &u, 8);
  return x;
}
#endif

// One corner of a pair: a = V - o and la = |a|, bit-identical to capi.mojo:218-229.
// These depend only on the vertex and the query, so a corner shared by consecutive
// faces can be reused without changing any bit of the result.
struct Corner {
  double x, y, z, l;
};

WN_HD Corner corner_exact(double ox, double oy, double oz, double Vx, double Vy, double Vz) {
  Corner c;
  c.x = dsub(Vx, ox);
  c.y = dsub(Vy, oy);
  c.z = dsub(Vz, oz);
  c.l = dsqrt(dadd(dadd(dmul(c.x, c.x), dmul(c.y, c.y)), dmul(c.z, c.z)));
  return c;
}

// det and denom of a pair from its three corners, bit-identical to capi.mojo:230-234.
WN_HD void face_exact(const Corner& a, const Corner& b, const Corner& c, double& det,
                      double& denom) {
  const double t0 = dmul(a.x, dsub(dmul(b.y, c.z), dmul(b.z, c.y)));
  const double t1 = dmul(a.y, dsub(dmul(b.x, c.z), dmul(b.z, c.x)));
  const double t2 = dmul(a.z, dsub(dmul(b.x, c.y), dmul(b.y, c.x)));
  det = dadd(dsub(t0, t1), t2);
  double d = dmul(dmul(a.l, b.l), c.l);
  d = dadd(d, dmul(dadd(dadd(dmul(a.x, b.x), dmul(a.y, b.y)), dmul(a.z, b.z)), c.l));
  d = dadd(d, dmul(dadd(dadd(dmul(b.x, c.x), dmul(b.y, c.y)), dmul(b.z, c.z)), a.l));
  d = dadd(d, dmul(dadd(dadd(dmul(c.x, a.x), dmul(c.y, a.y)), dmul(c.z, a.z)), b.l));
  denom = d;
}

// det and denom of one (triangle, query) pair, bit-identical to capi.mojo:218-235.
WN_HD void pair_terms_exact(double ox, double oy, double oz, double Ax, double Ay, double Az,
                            double Bx, double By, double Bz, double Cx, double Cy, double Cz,
                            double& det, double& denom) {
  face_exact(corner_exact(ox, oy, oz, Ax, Ay, Az), corner_exact(ox, oy, oz, Bx, By, Bz),
             corner_exact(ox, oy, oz, Cx, Cy, Cz), det, denom);
}

// Running product of z_i = denom_i + i*det_i (see the file comment).
struct ArgAcc {
  double zr, zi;
  int k;
  int bad;
};

WN_HD void argacc_init(ArgAcc& s) {
  s.zr = 1.0;
  s.zi = 0.0;
  s.k = 0;
  s.bad = 0;
}

WN_HD void argacc_push(ArgAcc& s, double d, double t) {
  const int32_t hd = hi_word(d), ht = hi_word(t);
  // Both +-0: use (copysign(1, d), t), which has argument atan2(t, d).
  const bool zero = ((static_cast<uint32_t>(hd | ht) << 1) | lo_word(d) | lo_word(t)) == 0u;
  if (zero) d = from_words((hd & static_cast<int32_t>(0x80000000u)) | 0x3ff00000, 0u);
  const double nr = s.zr * d - s.zi * t;
  const double ni = s.zr * t + s.zi * d;
  const bool s0 = hi_word(s.zi) < 0, st = ht < 0, s1 = hi_word(ni) < 0;
  s.k += (s0 == st && s0 != s1) ? (s0 ? -1 : 1) : 0;
  // Rescale by 2^(1023 - e), e the biased exponent of the larger component.
  const int32_t er = hi_word(nr) & 0x7ff00000, ei = hi_word(ni) & 0x7ff00000;
  const int32_t e = er > ei ? er : ei;
  s.bad |= (e == 0) | (e == 0x7ff00000);
  const double scale = from_words(0x7fe00000 - e, 0u);
  s.zr = nr * scale;
  s.zi = ni * scale;
}

}  // namespace wn
