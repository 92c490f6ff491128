// Batched meshes: many meshes and query sets of uneven sizes evaluated by one
// persistent launch (see wn_mixed.cu, "batched meshes").
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

#include "wn_mixed.h"

namespace wn {

// One unit of persistent work: up to THREADS*QPT Morton-ordered queries of one mesh
// against a contiguous range of that mesh's tiles; its per-query angle sums go to
// partial[p_base + (s - q_begin)].
struct BatchItem {
  int64_t q_begin;  // first sorted query position (over the whole batch)
  int64_t t_begin;  // first tile (over the whole batch)
  int64_t p_base;   // partial-sum index of q_begin
  int32_t q_count, t_count;
};

// Per-mesh offsets used by the finishing kernels.
struct BatchMeshInfo {
  int64_t q_off, nq, p_off, nchunk;
};

struct BatchPlan {
  int qpt = 2;
  int64_t target_pairs = int64_t(1) << 23;  // pairs per work item
  int ctas_per_sm = 0;                      // 0 = as many as fit
  double kappa = 4.0;
  int tile_faces = 64;                      // 64, or 32: far test and angle per half tile
};

struct BatchDevice;  // device buffers of the forward, defined in wn_mixed.cu
struct BatchEdges;   // boundary edges and buffers of the adjoint, defined in wn_adjoint.cu

struct BatchState {
  int device = -1;
  int sms = 0;
  BatchPlan plan;
  int64_t nmesh = 0, total_nv = 0, total_nf = 0, total_nq = 0, total_tiles = 0;
  int64_t n_items = 0, total_partials = 0, ldt = 0;
  int grid = 0;
  int mesh_bits = 1;
  std::vector<int64_t> v_off, nv, f_off, nf, q_off, nq, t_off, ntile;
  BatchDevice* dev = nullptr;
  BatchEdges* edges = nullptr;
};

// Host-side layout + device allocation. F: total_nf x 3, vertex indices local to
// each mesh. Returns a CUDA error (allocation) or cudaSuccess.
cudaError_t batch_create(BatchState* b, int64_t nmesh, const int64_t* nv, const int64_t* nf,
                         const int64_t* nq, const int64_t* F, const BatchPlan& plan, int sms);
void batch_destroy(BatchState* b);

// Forward of every mesh: V (total_nv x 3), q (total_nq x 3) -> w (total_nq).
// Allocation-free and free of host synchronisation (capturable in a graph).
cudaError_t batch_forward(BatchState* b, const double* V, const double* q, double* w,
                          unsigned long long* stats, int* err, cudaStream_t stream);

// Boundary-edge adjoint of every mesh (FP64, persistent, deterministic):
// set up from the faces (host, local indices) once, then per call
// gw (total_nq) -> dq (total_nq x 3), dV (total_nv x 3).
cudaError_t batch_edges_create(BatchState* b, const int64_t* F);
void batch_edges_destroy(BatchState* b);
int64_t batch_boundary_edges(const BatchState* b);
int64_t batch_edge_items(const BatchState* b);
cudaError_t batch_backward(BatchState* b, const double* V, const double* q, const double* gw,
                           double* dq, double* dV, cudaStream_t stream);

// The adjoint's precision: mixed (FP32 edge pairs in per-mesh Morton-ordered 64-edge
// tiles, FP64 near pairs; the default, as the forward) or FP64. Both paths' buffers
// are allocated by batch_edges_create, so switching allocates nothing.
void batch_set_adjoint_fp64(BatchState* b, bool fp64);
bool batch_adjoint_fp64(const BatchState* b);

// Morton order of n points (x, y, z rows) inside each mesh: keys mesh << 30 | the
// 30-bit code against the mesh's own box (the single-mesh code for the same points),
// one radix sort; perm[s] = the point at sorted position s, meshes in order. Buffers:
// box nmesh x 6, keys and values n each, temp batch_morton_temp_bytes(n, mesh_bits).
size_t batch_morton_temp_bytes(int64_t n, int mesh_bits);
cudaError_t batch_morton_order(const double* pts, int64_t n, const int32_t* mesh_of,
                               int64_t nmesh, int mesh_bits, unsigned long long* box,
                               uint64_t* keys_in, uint64_t* keys_out, uint32_t* vals_in,
                               uint32_t* perm, void* temp, size_t temp_bytes,
                               cudaStream_t stream);

}  // namespace wn
