// Adjoint (backward) of the winding number: interfaces (see wn_adjoint.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace wn {

struct AdjointPlan {
  int64_t nranges = 1, blocks_per_range = 1;   // face ranges (grid.x) of 256-face blocks
  int64_t ngroups = 1, queries_per_group = 1;  // query groups (grid.y)
};

AdjointPlan plan_adjoint(int64_t nf, int64_t nq, int sms);

// Scratch for the partial sums: nranges*nq*3 + ngroups*9*ld doubles.
size_t adjoint_scratch_bytes(const AdjointPlan& p, int64_t ld, int64_t nq);

// FP64 adjoint: gw (nq) = dL/dW; outputs dq (nq x 3) = dL/do and dtri (9 x ld) = dL/d(corner).
cudaError_t adjoint_fp64(const AdjointPlan& p, const double* tri, int64_t ld, int64_t nf,
                         const double* q, int64_t nq, const double* gw, double* dq, double* dtri,
                         void* scratch, size_t scratch_bytes, cudaStream_t stream);

// Mixed-precision adjoint over a prepared mesh (wn_mixed.h) with Morton-ordered queries
// (perm from mixed_sort_queries). Same outputs as adjoint_fp64, in input order; dtri has
// row stride ld >= nf. Scratch: adjoint_scratch_bytes(p, m.ld64, nq).
AdjointPlan plan_adjoint_mixed(int64_t ntiles, int64_t nq, int sms);
struct MixedMesh;
cudaError_t adjoint_mixed(const AdjointPlan& p, const MixedMesh& m, const double* q,
                          const uint32_t* perm, int64_t nq, const double* gw, double* dq,
                          double* dtri, int64_t ld, void* scratch, size_t scratch_bytes,
                          cudaStream_t stream);

// Boundary-edge adjoint (indexed meshes): edges 7 x le (P, Q, net multiplicity m), outputs
// dq (nq x 3) and dedge (6 x le: dL/dP, dL/dQ).
AdjointPlan plan_adjoint_edges(int64_t ne, int64_t nq, int sms);
size_t adjoint_edges_scratch_bytes(const AdjointPlan& p, int64_t le, int64_t nq);
cudaError_t adjoint_edges(const AdjointPlan& p, const double* edges, int64_t le, int64_t ne,
                          const double* q, int64_t nq, const double* gw, double* dq,
                          double* dedge, void* scratch, size_t scratch_bytes,
                          cudaStream_t stream);

// Mixed-precision boundary-edge adjoint: the same inputs and outputs as
// adjoint_edges, FP32 far pairs in Morton-ordered 64-edge tiles and FP64 pairs
// with an endpoint within kappa |e| of the query (kappa >= 3). The edge and query
// orders are built inside the call from `scratch`. With `unit` the per-endpoint sums
// are unweighted and the multiplicity weights dL/do only (edges welded by position:
// each edge stands for the soup's directed sides on it, signed per side afterwards).
// With `unit`, dq may be null: dL/do is not computed (no_dq in the plan; every m is 0
// when the soup is a closed surface, so dL/do is exactly 0 there).
AdjointPlan plan_adjoint_edges_mixed(int64_t ne, int64_t nq, int sms, bool no_dq = false);
size_t adjoint_edges_mixed_scratch_bytes(const AdjointPlan& p, int64_t ne, int64_t nq);
cudaError_t adjoint_edges_mixed(const AdjointPlan& p, const double* edges, int64_t le, int64_t ne,
                                const double* q, int64_t nq, const double* gw, double kappa,
                                bool unit, double* dq, double* dedge, void* scratch,
                                size_t scratch_bytes, cudaStream_t stream);

// dV (nv x 3) from per-element corner gradients (rows 3*corner+axis, stride ld) through the
// vertex -> (corners*element + corner) list (CSR indptr, entries); corners = 3 (faces) or 2
// (edges).
cudaError_t gather_vertex_grad(const double* dtri, int64_t ld, int corners,
                               const int64_t* indptr, const int64_t* entries, int64_t nv,
                               double* dV, cudaStream_t stream);

}  // namespace wn
