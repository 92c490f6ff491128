// Per-vertex normals on the GPU (internal interface between wn_normals.cu and
// the C ABI). The topology (faces) is prepared once: faces as int32, the visit
// order of the vertices (by first incident face) and the list of (face, corner)
// incidences of every vertex in face order, stored in visit order: list t
// belongs to vertex order[t] (CSR: indptr nv + 1, entries 3 nf = 3 * face +
// corner; built by two stable radix sorts, vertices by first face, then
// incidences by their vertex's rank). A normals call then runs two passes: one
// thread per face writes its contribution u * weight (per face for the uniform
// and area weights, whose three corners share it; per corner for the angle
// weight; a NaN marks a face the reference skips), then thread t adds list t's
// contributions in order and normalises vertex order[t] (a face's three readers
// come close together in time, and the lists are read contiguously). The
// additions are the reference's, operand for operand and in its order
// (wn_normals.cuh), so positions can change between calls at no set-up cost.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace wn {

// Doubles per contribution record (a face's for the uniform and area weights, a
// corner's for the angle weight).
constexpr int kContribRecord = 3;

// Doubles of contribution records for nf faces under weighting `mode`.
inline int64_t normals_contrib_doubles(int64_t nf, int mode) {
  return (mode == 2 ? 3 : 1) * kContribRecord * nf;
}

struct NormalsTopology {
  int32_t* F = nullptr;        // 3 nf, 16-byte aligned (read with 16-byte loads)
  int32_t* indptr = nullptr;   // nv + 1, by visit slot
  int32_t* entries = nullptr;  // 3 nf, lists in visit order
  int32_t* order = nullptr;    // nv: vertices by first incident face (the gather's visit order)
  double* contrib = nullptr;   // normals_contrib_doubles(nf, mode), grown on demand
  int64_t contrib_doubles = 0;
  int64_t nf = 0, nv = 0;
};

// Device bytes of scratch for preparing nf faces over nv vertices.
size_t normals_scratch_bytes(int64_t nf, int64_t nv);

// Prepares t.F, the incidence lists and the vertex visit order from F64 (device,
// 3 nf int64). Indices outside [0, nv) are counted in *bad (device int, zeroed
// here) and kept out of the lists; the caller checks *bad after the stream drains.
cudaError_t normals_build(NormalsTopology& t, const int64_t* F64, int* bad, void* scratch,
                          size_t scratch_bytes, cudaStream_t stream);

// N (nv x 3) from V (nv x 3) with weighting 0 uniform, 1 area, 2 angle; t.contrib
// must hold 9 nf doubles for the angle weight, 3 nf otherwise.
cudaError_t normals_eval(const NormalsTopology& t, const double* V, int mode, double* N,
                         cudaStream_t stream);

}  // namespace wn
