// Per-vertex normals on the GPU (internal interface between wn_normals.cu and
// the C ABI). The topology (faces) is prepared once: faces as int32 and the
// list of (face, corner) incidences of every vertex in face order, built by a
// stable radix sort of the flattened face array (CSR: indptr nv + 1, entries
// 3 nf = 3 * face + corner). A normals call then runs two coalesced passes:
// one thread per face writes its contribution u * weight (per face for the
// uniform and area weights, whose three corners share it; per corner for the
// angle weight; a NaN marks a face the reference skips), then one thread per
// vertex adds its incidences' contributions in CSR order and normalises (the
// vertices are visited by first incident face, an order set up with the lists,
// so that a face's three readers come close together in time). The
// additions are the reference's, operand for operand and in its order
// (wn_normals.cuh), so positions can change between calls at no set-up cost.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace wn {

struct NormalsTopology {
  int32_t* F = nullptr;        // 3 nf
  int32_t* indptr = nullptr;   // nv + 1
  int32_t* entries = nullptr;  // 3 nf
  int32_t* order = nullptr;    // nv: vertices by first incident face (the gather's visit order)
  double* contrib = nullptr;   // 9 nf (angle) or 3 nf doubles, grown on demand
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
