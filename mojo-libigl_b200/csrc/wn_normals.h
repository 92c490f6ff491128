// Per-vertex normals on the GPU (internal interface between wn_normals.cu and
// the C ABI). The topology (faces) is prepared once: faces as int32 and the
// list of (face, corner) incidences of every vertex in face order, built by a
// stable radix sort of the flattened face array (CSR: indptr nv + 1, entries
// 3 nf = 3 * face + corner). A normals call then runs one thread per vertex
// over its incidences (wn_normals.cuh), so every vertex sums in the reference's
// order and positions can change between calls at no extra set-up cost.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace wn {

struct NormalsTopology {
  int32_t* F = nullptr;        // 3 nf
  int32_t* indptr = nullptr;   // nv + 1
  int32_t* entries = nullptr;  // 3 nf
  int64_t nf = 0, nv = 0;
};

// Device bytes of sort scratch for 3 nf incidences.
size_t normals_scratch_bytes(int64_t nf);

// Builds the incidence lists from F (device, 3 nf int32, every index in
// [0, nv)); `t` holds device arrays of the sizes above; scratch has
// normals_scratch_bytes(nf) bytes.
cudaError_t normals_build(NormalsTopology& t, void* scratch, size_t scratch_bytes,
                          cudaStream_t stream);

// N (nv x 3) from V (nv x 3) with weighting 0 uniform, 1 area, 2 angle.
cudaError_t normals_eval(const NormalsTopology& t, const double* V, int mode, double* N,
                         cudaStream_t stream);

}  // namespace wn
