// Host (device="cpu") path of the per-vertex normals: `mli_vertex_normals`,
// the reference's C-ABI export (src/capi.mojo:933-935, kernel capi.mojo:146-202),
// on the shared arithmetic of wn_normals.cuh (built with -ffp-contract=off).
#include <cstdint>

#include "wn_normals.cuh"

extern "C" {

// Every argument an int64 (host addresses, python/igl/_lib.py:21); weighting
// 0 uniform, 1 area, 2 angle, 3 default (= area).
void mli_vertex_normals(int64_t v_addr, int64_t f_addr, int64_t dst_addr, int64_t nv, int64_t nf,
                        int64_t weighting) {
  const double* v = reinterpret_cast<const double*>(v_addr);
  const int64_t* f = reinterpret_cast<const int64_t*>(f_addr);
  double* dst = reinterpret_cast<double*>(dst_addr);
  for (int64_t i = 0; i < 3 * nv; ++i) dst[i] = 0.0;
  const int mode = weighting == 3 ? wn::kNormalsArea : static_cast<int>(weighting);
  for (int64_t fi = 0; fi < nf; ++fi) {
    const double* P[3] = {v + 3 * f[3 * fi], v + 3 * f[3 * fi + 1], v + 3 * f[3 * fi + 2]};
    double u[3], norm;
    if (!wn::face_unit_normal(P[0], P[1], P[2], u, &norm)) continue;
    for (int corner = 0; corner < 3; ++corner) {
      const double w = wn::corner_weight(P, corner, mode, norm);
      double* d = dst + 3 * f[3 * fi + corner];
      for (int k = 0; k < 3; ++k) d[k] = wn::dadd(d[k], wn::dmul(u[k], w));
    }
  }
  for (int64_t i = 0; i < nv; ++i) wn::normal_finish(dst + 3 * i);
}

}  // extern "C"
