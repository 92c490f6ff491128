// ORACLE — test infrastructure only. Not part of the product library.
//
// CPU restatement of the reference's per-vertex normals (lee101/mojo-libigl,
// src/capi.mojo:146-202, exported as `mli_vertex_normals` at capi.mojo:933-935,
// driven by python/igl/__init__.py:195-211). Linked into liboracle_wn.so; only
// tests, the smoke check and bench.py's CPU-baseline / reference legs load it.
//
// Restated step for step: clear the output; weighting 3 (the default) means
// area; for every face in order: n = (B - A) x (C - A) with the reference's
// component formulas, |n| = sqrt(nx*nx + ny*ny + nz*nz), faces with
// |n| <= 1e-30 skipped, u = n / |n|; for each corner in order the weight is 1
// (uniform), |n| (area) or acos(clamp((e1.e2) / (|e1| |e2|), -1, 1)) with e1,
// e2 the corner's two outgoing edges (angle); the vertex's sum gets u * weight
// added component by component. Then every vertex with |sum| > 1e-30 is
// divided by |sum|. Every product and sum is rounded on its own
// (-ffp-contract=off); acos is the C library's.
#include <cmath>
#include <cstdint>

extern "C" {

void mli_vertex_normals(int64_t v_addr, int64_t f_addr, int64_t dst_addr, int64_t nv, int64_t nf,
                        int64_t weighting) {
  const double* v = reinterpret_cast<const double*>(v_addr);
  const int64_t* f = reinterpret_cast<const int64_t*>(f_addr);
  double* dst = reinterpret_cast<double*>(dst_addr);
  for (int64_t i = 0; i < nv * 3; ++i) dst[i] = 0.0;
  const int64_t mode = weighting == 3 ? 1 : weighting;
  for (int64_t fi = 0; fi < nf; ++fi) {
    const double* A = v + 3 * f[3 * fi];
    const double* B = v + 3 * f[3 * fi + 1];
    const double* C = v + 3 * f[3 * fi + 2];
    const double abx = B[0] - A[0], aby = B[1] - A[1], abz = B[2] - A[2];
    const double acx = C[0] - A[0], acy = C[1] - A[1], acz = C[2] - A[2];
    const double nx = aby * acz - abz * acy;
    const double ny = abz * acx - abx * acz;
    const double nz = abx * acy - aby * acx;
    const double norm = std::sqrt(nx * nx + ny * ny + nz * nz);
    if (norm <= 1.0e-30) continue;
    const double ux = nx / norm, uy = ny / norm, uz = nz / norm;
    for (int corner = 0; corner < 3; ++corner) {
      const int64_t vi = f[3 * fi + corner];
      double weight = mode == 1 ? norm : 1.0;
      if (mode == 2) {
        const int64_t vj = f[3 * fi + (corner + 1) % 3], vk = f[3 * fi + (corner + 2) % 3];
        const double e1x = v[3 * vj] - v[3 * vi], e1y = v[3 * vj + 1] - v[3 * vi + 1],
                     e1z = v[3 * vj + 2] - v[3 * vi + 2];
        const double e2x = v[3 * vk] - v[3 * vi], e2y = v[3 * vk + 1] - v[3 * vi + 1],
                     e2z = v[3 * vk + 2] - v[3 * vi + 2];
        const double l1 = std::sqrt(e1x * e1x + e1y * e1y + e1z * e1z);
        const double l2 = std::sqrt(e2x * e2x + e2y * e2y + e2z * e2z);
        double cosine = (e1x * e2x + e1y * e2y + e1z * e2z) / (l1 * l2);
        cosine = std::fmax(-1.0, std::fmin(1.0, cosine));
        weight = std::acos(cosine);
      }
      dst[3 * vi] += ux * weight;
      dst[3 * vi + 1] += uy * weight;
      dst[3 * vi + 2] += uz * weight;
    }
  }
  for (int64_t i = 0; i < nv; ++i) {
    const double x = dst[3 * i], y = dst[3 * i + 1], z = dst[3 * i + 2];
    const double norm = std::sqrt(x * x + y * y + z * z);
    if (norm > 1.0e-30) {
      dst[3 * i] = x / norm;
      dst[3 * i + 1] = y / norm;
      dst[3 * i + 2] = z / norm;
    }
  }
}

}  // extern "C"
