// Host (device="cpu") path of libwn_b200: `mli_winding`, the C-ABI entry the
// reference exports from src/capi.mojo:938-942 (kernel at capi.mojo:205-294).
//
// Same contract as the reference: fill dst[q0:q1) for queries q0..q1-1 of the
// (9, nf) triangle-soup SoA; reentrant over disjoint spans, so the Python shim
// can fan spans out over threads with the GIL released. The pair terms are
// the shared bit-exact ones (wn_pair.cuh; this file is built with
// -ffp-contract=off) and the angles are summed with the argument-of-product
// accumulator, with plain atan2 as the recovery path for a bad accumulator.
#include <cmath>
#include <cstdint>

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
  for (int64_t qi = q0; qi < q1; ++qi)
    d[qi] = winding_query(t, nf, qq[3 * qi], qq[3 * qi + 1], qq[3 * qi + 2]);
}

}  // extern "C"
