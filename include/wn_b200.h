/* libwn_b200 — C ABI of the B200 (sm_100a) exact generalized winding number.
 *
 * Drop-in for the winding-number entry points of lee101/mojo-libigl's
 * `libmojo-libigl.so` (exported from src/capi.mojo:923-1007, bound by
 * python/igl/_lib.py:18-32 with every argument an int64). Plain C types only:
 * pointers, int64_t sizes and int status codes; no torch or CUDA types.
 *
 * Conventions
 *   tri   triangle soup, structure of arrays: 9 rows of nf doubles, row
 *         3*corner+axis (corner a,b,c; axis x,y,z), i.e. tri[(3c+x)*nf + f].
 *         This is python/igl/__init__.py:248-250's
 *         `vertices[faces].transpose(1, 2, 0).reshape(9, nf)`.
 *   q     queries, nq x 3 row-major doubles.
 *   w     nq doubles, W(q) = sum_f atan2(det_f, denom_f) / (2*pi).
 *   "host" entry points take host pointers, copy in, compute, copy out and
 *   synchronise. "device" entry points take device pointers and a cudaStream_t
 *   passed as void*; they are asynchronous: call wn_stream_check() to
 *   synchronise and collect device-side errors.
 *   Return value: 0 = success, otherwise a WN_E* code; wn_last_error() gives
 *   the message (per calling thread). The mli_* names keep the reference's
 *   own return conventions.
 */
#ifndef WN_B200_H
#define WN_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  WN_OK = 0,
  WN_EINVAL = 1,   /* bad sizes, pointers or alignment */
  WN_ENODEV = 2,   /* no CUDA device / driver */
  WN_ECUDA = 3,    /* a CUDA runtime call failed */
  WN_EDEVICE = 4,  /* a kernel reported an error (e.g. a bounded wait ran out) */
  WN_ENOMEM = 5    /* device allocation failed */
};

/* Fault kinds of wn_inject_fault. */
enum { WN_FAULT_NONE = 0, WN_FAULT_ALLOC = 1 };

/* FP64 accumulation modes of the plain kernel. */
enum {
  WN_FP64_ARGPROD = 0, /* bit-exact pair terms, argument-of-product sum */
  WN_FP64_DIRECT = 1,  /* bit-exact pair terms, one atan2 per pair */
  WN_FP64_TILED = 2    /* WN_FP64_ARGPROD over a prepared mesh (Morton tiles, faces in
                          strips) that reuses repeated corners; host entry only */
};

/* ---- reference-compatible entry points --------------------------------- */

/* Replaces src/capi.mojo:938-942 `mli_winding(tri, q, dst, nf, nq, q0, q1)`:
 * CPU evaluation of queries [q0, q1) into dst[q0:q1). Reentrant over disjoint
 * spans (python/igl/_lib.py:72-95 fans spans out over threads). */
void mli_winding(int64_t tri, int64_t q, int64_t dst, int64_t nf, int64_t nq, int64_t q0,
                 int64_t q1);

/* Replaces src/capi.mojo:945-947 `mli_winding_gpu(tri, q, dst, nf, nq) -> Int`
 * (host addresses; 1 = success, 0 = failure, python/igl/__init__.py:253-263).
 * Runs the plain FP64 kernel on the current CUDA device. */
int64_t mli_winding_gpu(int64_t tri, int64_t q, int64_t dst, int64_t nf, int64_t nq);

/* Replaces src/capi.mojo:950-959 `mli_aabb_squared_distance(p, v, f, boxes,
 * nodes, order, sqrd, indices, closest, stack, np, nnodes, q0, q1)` (every
 * argument an int64 host address or size, python/igl/_lib.py:23): CPU closest
 * point of queries [q0, q1) over the tree arrays of python/igl/__init__.py:
 * 286-319 (boxes nnodes x 6, nodes nnodes x 4, order nf), writing sqrd[qi],
 * indices[qi] and closest[3*qi..3*qi+2]; `stack` holds at least depth + 1
 * int64. Reentrant over disjoint spans, each with its own stack. */
void mli_aabb_squared_distance(int64_t p, int64_t v, int64_t f, int64_t boxes, int64_t nodes,
                               int64_t order, int64_t sqrd, int64_t indices, int64_t closest,
                               int64_t stack, int64_t np, int64_t nnodes, int64_t q0,
                               int64_t q1);

/* Replaces src/capi.mojo:933-935 `mli_vertex_normals(v, f, dst, nv, nf,
 * weighting)` (int64 host addresses and sizes, python/igl/_lib.py:21): CPU
 * per-vertex normals into dst (nv x 3), weighting 0 uniform, 1 area, 2 angle,
 * 3 default (= area), bit-identical to the reference's loop for 0, 1 and 3. */
void mli_vertex_normals(int64_t v, int64_t f, int64_t dst, int64_t nv, int64_t nf,
                        int64_t weighting);

/* The reference's other nine exports (src/capi.mojo:923-932, 962-1007) are
 * exported under the same names so the reference shim's loader
 * (python/igl/_lib.py:122-130) resolves every symbol; they are outside this
 * library's scope and abort the process with a message if called. */

/* ---- runtime ------------------------------------------------------------ */

int wn_version(void);                 /* 100 * major + minor */
const char* wn_last_error(void);      /* message of this thread's last failure */
int wn_device_count(void);            /* CUDA devices visible (0 if none) */
int wn_device_memory(int64_t* free_bytes, int64_t* total_bytes); /* current device */
/* Synchronise `stream` and report (then clear) device-side errors raised by
 * device entry points launched on it since the last check. */
int wn_stream_check(void* stream);
/* Failure-detection self-test: a kernel waits on a phase that nothing completes,
 * gives up after `polls` bounded polls (1..2^24), reports it through the device
 * error word, and returns. Expected result: WN_EDEVICE, with the context still
 * usable. No fault, no trap, no hang. */
int wn_selftest_bounded_wait(int64_t polls);
/* Number of kernels this library has launched since it was loaded. */
int64_t wn_launch_count(void);
/* Host-side fault injection, for tests of the out-of-memory paths on a real
 * device: kind WN_FAULT_ALLOC makes the (after+1)-th device allocation of the
 * library from now on report failure (WN_ENOMEM from the entry point) without
 * allocating; WN_FAULT_NONE disarms. One-shot. Every entry point returns
 * before launching work that needs the failed allocation, so nothing on the
 * device runs differently. WN_INJECT_FAULT=alloc:N in the environment arms it
 * when the library is loaded. */
int wn_inject_fault(int kind, int64_t after);
/* 1 while an injected fault is armed and has not fired, else 0. */
int wn_fault_armed(void);
/* Measured FMA-pipe peak of the current device in TFLOP/s (FMA = 2 flops),
 * bits = 64 or 32: the roofline denominator of these FP64/FP32-bound kernels. */
int wn_probe_fma_tflops(int bits, double* tflops);

/* ---- plain FP64 forward (no reference counterpart beyond mli_winding_gpu) */

/* Host pointers; mode = WN_FP64_ARGPROD, WN_FP64_DIRECT or WN_FP64_TILED. */
int wn_forward_fp64_host(const double* tri, const double* q, double* w, int64_t nf, int64_t nq,
                         int mode);

/* Device pointers. tri: 9 rows with row stride ld doubles (ld even, ld >= nf),
 * 16-byte aligned. Scratch (for face splits when nq is small) comes from the
 * library's per-device workspace. */
int wn_forward_fp64_device(const double* tri, int64_t ld, const double* q, double* w, int64_t nf,
                           int64_t nq, int mode, void* stream);

/* No counterpart in the reference: the plain FP64 forward for callers that
 * must not allocate GPU memory, such as host applications and plugins that own
 * all device memory through their own pool or a fixed budget and forbid
 * libraries from calling cudaMalloc. Same arguments and results as
 * wn_forward_fp64_device, but its face-split scratch is a fixed 4 MiB array
 * inside the library (held on every GPU that loads it until exit) instead of an
 * allocation. Limit: nq <= 524288 (2^19) queries, else WN_EINVAL. The first call
 * on each device looks up the array's device address and should come before
 * any stream capture. The stream must belong to the current device (else
 * WN_EINVAL). All calls share the array: within one process a mutex held until
 * the caller's stream has finished the work keeps calls from overlapping; calls
 * that did overlap on the GPU would race. Returns after the caller's stream has
 * finished the work, so a stream that is being captured is refused (WN_EINVAL)
 * and left untouched. */
int wn_forward_fp64_device_noalloc(const double* tri, int64_t ld, const double* q, double* w,
                                   int64_t nf, int64_t nq, int mode, void* stream);

/* ---- mixed precision forward (no reference counterpart) ----------------
 * FP32 pair terms, FP32 two-sum accumulation across 64-face tiles, FP64
 * refinement (bit-exact pair terms + atan2) of every pair with a vertex closer
 * than kappa * (the face's longest edge). kappa in [3, 1e6]; 4 is the default
 * of the Python API. Results agree with the FP64 kernel to ~1e-7 (the tests
 * and bench report max / p99 absolute error). */

/* Host pointers: prepares the mesh, sorts the queries and evaluates. */
int wn_forward_mixed_host(const double* tri, const double* q, double* w, int64_t nf, int64_t nq,
                          double kappa);

/* Device path: prepare a mesh once (tri: device SoA, row stride ld, even,
 * 16-byte aligned), evaluate query batches against it, destroy it. */
int wn_mixed_mesh_create(const double* tri, int64_t ld, int64_t nf, double kappa, void* stream,
                         void** mesh_out);
int wn_mixed_mesh_destroy(void* mesh);
/* The plain FP64 forward over a prepared mesh (WN_FP64_TILED): same bit-exact
 * pair terms, corners shared by consecutive faces evaluated once. */
int wn_forward_fp64_mesh_device(void* mesh, const double* q, int64_t nq, double* w,
                                void* stream);
int wn_forward_mixed_device(void* mesh, const double* q, int64_t nq, double* w, void* stream);
/* Re-prepare an existing mesh in place from new vertex positions (same face
 * count), e.g. once per step of a shape optimisation. */
int wn_mixed_mesh_update(void* mesh, const double* tri, int64_t ld, void* stream);
/* Faces per far test and angle product of the mixed forward on this mesh: 64
 * (the default) or 32 (each half of a 64-face tile tested against its own ball
 * and summed with its own product); same error bound either way. */
int wn_mixed_mesh_set_tile_faces(void* mesh, int tile_faces);
/* The two halves of wn_forward_mixed_device: Morton-order the queries into
 * perm (nq uint32, device), then evaluate the queries in that order. */
int wn_mixed_sort_queries(const double* q, int64_t nq, uint32_t* perm, void* stream);
int wn_forward_mixed_sorted_device(void* mesh, const double* q, const uint32_t* perm, int64_t nq,
                                   double* w, void* stream);

/* Counters of the mixed path on the current device since the last reset:
 * pairs refined in FP64, and (warp, tile) visits that ran the near test. */
int wn_mixed_stats(int64_t* refined_pairs, int64_t* careful_visits, int reset);

/* ---- batched meshes (no reference counterpart) ---------------------------
 * Many indexed meshes with their own query sets, of uneven sizes, evaluated by
 * one persistent launch (mixed precision). Create once per set of sizes and
 * faces; forward is asynchronous, allocation-free and synchronisation-free, so
 * a sequence of forwards can be captured in a CUDA graph.
 *   nv/nf/nq: host arrays of nmesh sizes; faces: host, total_nf x 3 int64,
 *   vertex indices local to each mesh (meshes concatenated in order).
 *   qpt: queries per thread (1, 2 or 4); target_pairs: pairs per work item;
 *   ctas_per_sm: persistent CTAs per SM (0 = as many as fit); tile_faces: faces
 *   per far test and angle product, 64 or 32 (each half of a 64-face tile on its
 *   own).
 *   V (total_nv x 3), q (total_nq x 3), w (total_nq): device, concatenated. */
int wn_batch_create(int64_t nmesh, const int64_t* nv, const int64_t* nf, const int64_t* nq,
                    const int64_t* faces, double kappa, int qpt, int64_t target_pairs,
                    int ctas_per_sm, int tile_faces, void** batch_out);
int wn_batch_forward(void* batch, const double* V, const double* q, double* w, void* stream);
/* Adjoint of every mesh through its net boundary edges (deterministic): gw
 * (total_nq) -> dq (total_nq x 3), dV (total_nv x 3). Same launch properties as
 * wn_batch_forward. Mixed precision by default, as the forward (each mesh's edges
 * in their own Morton order, 64-edge tiles, FP32 pairs with FP64 pairs near an
 * edge, as wn_backward_edges_mixed_device); FP64 after
 * wn_batch_set_adjoint_fp64(batch, 1). Both paths' buffers come from
 * wn_batch_create: switching allocates nothing. */
int wn_batch_backward(void* batch, const double* V, const double* q, const double* gw,
                      double* dq, double* dV, void* stream);
int wn_batch_set_adjoint_fp64(void* batch, int fp64);
/* out[0..n): nmesh, total_nv, total_nf, total_nq, total_tiles, work items,
 * persistent grid, partial sums, qpt, target_pairs, boundary edges, adjoint
 * work items (of the selected precision), tile_faces, adjoint in FP64 (0/1). */
int wn_batch_info(void* batch, int64_t* out, int64_t n);
int wn_batch_destroy(void* batch);

/* ---- adjoint (no reference counterpart) ---------------------------------
 * gw: dL/dW per query (nq). Outputs dq (nq x 3) = dL/do and dtri (9 rows of
 * stride ld, the soup's layout) = dL/d(corner) per face; every pair term is
 * recomputed (nothing nf x nq is stored) and the reductions over faces and
 * over queries are deterministic (fixed order, no floating-point atomics).
 * Pairs with the query on a vertex or on a side contribute zero. */
int wn_backward_fp64_device(const double* tri, int64_t ld, int64_t nf, const double* q,
                            int64_t nq, const double* gw, double* dq, double* dtri, void* stream);

/* Mixed-precision adjoint over a mesh prepared by wn_mixed_mesh_create: FP32
 * pair terms for pairs with every vertex at least kappa * (longest edge) away,
 * FP64 for the others, FP64 sums across query chunks and over faces. dtri has
 * row stride ld (even, >= nf) and is indexed by the input face order. */
int wn_backward_mixed_device(void* mesh, const double* q, int64_t nq, const double* gw,
                             double* dq, double* dtri, int64_t ld, void* stream);

/* Boundary-edge adjoint for indexed meshes (mathematically equal to the per-face
 * adjoint summed at the vertices: the terms of a directed side and its reverse
 * cancel, so only edges with nonzero net multiplicity m = #(u->v) - #(v->u)
 * remain). edges: 7 rows of stride le (Px, Py, Pz, Qx, Qy, Qz, m); outputs dq
 * (nq x 3) and dedge (6 rows of stride le: dL/dP, dL/dQ). FP64, deterministic. */
int wn_backward_edges_device(const double* edges, int64_t le, int64_t ne, const double* q,
                             int64_t nq, const double* gw, double* dq, double* dedge,
                             void* stream);
/* The boundary-edge adjoint in mixed precision: the same arguments and outputs,
 * plus kappa (>= 3). Edges are Morton-ordered into 64-edge tiles inside the call;
 * pairs with both endpoints at least kappa * |edge| from the query run in FP32 in
 * the tile's scaled frame, the others in FP64; FP64 sums across query chunks and
 * over edges. Deterministic. unit_weights = 0: the per-endpoint sums are weighted
 * by m, as wn_backward_edges_device's. unit_weights = 1 (edges welded by position
 * from a triangle soup, m = the net count of the soup's directed sides on the
 * edge): dedge holds the unweighted sums -dL/dW dOmega/dP and -dL/dW dOmega/dQ of
 * one side P -> Q, to be signed per soup side, while dq still uses m; there dq
 * may be NULL, and dL/do is then not computed (a soup that is a closed surface has
 * every m = 0, so its dL/do is exactly 0), which takes a leaner kernel. */
int wn_backward_edges_mixed_device(const double* edges, int64_t le, int64_t ne, const double* q,
                                   int64_t nq, const double* gw, double kappa, int unit_weights,
                                   double* dq, double* dedge, void* stream);

/* dV (nv x 3) = sum of per-element corner gradients over each vertex's uses.
 * grad: rows 3*corner+axis with stride ld; corners = 3 (faces, dtri) or 2 (edges,
 * dedge); indptr (nv+1) and entries (corners*element + corner, grouped by
 * vertex) form a CSR list summed in list order (deterministic). */
int wn_gather_vertex_grad_device(const double* grad, int64_t ld, int corners,
                                 const int64_t* indptr, const int64_t* entries, int64_t nv,
                                 double* dV, void* stream);

/* ---- closest points over the median-split hierarchy ---------------------
 * V: nv x 3 doubles; F: nf x 3 int64; P: np x 3 doubles. Tree arrays as the
 * reference's python/igl/__init__.py:286-319 `_build_aabb` returns them:
 * boxes nnodes x 6 (lo xyz, hi xyz), nodes nnodes x 4 (left, right, start,
 * count; count > 0 marks a leaf of order[start:start+count]), order nf, nodes
 * in preorder. Results per point: sqrd (squared distance), index (face) and
 * closest (3 doubles), bit-identical to mli_aabb_squared_distance; with no
 * faces, 1e300, -1 and (0, 0, 0). */

/* Nodes of the tree over nf faces with at most leaf_size faces per leaf (the
 * reference uses 8); 0 for nf = 0. No reference counterpart. */
int64_t wn_aabb_node_count(int64_t nf, int64_t leaf_size);

/* Replaces python/igl/__init__.py:286-319 `_build_aabb(vertices, faces,
 * leaf_size)`: fills boxes (wn_aabb_node_count x 6), nodes (x 4) and order
 * (nf) with the same tree, and *stack_size with depth + 1 (0 for nf = 0).
 * Host memory; builds subtrees on up to `threads` threads (<= 0: all cores). */
int wn_aabb_build(const double* V, int64_t nv, const int64_t* F, int64_t nf, int64_t leaf_size,
                  double* boxes, int64_t* nodes, int64_t* order, int64_t* stack_size,
                  int threads);

/* Uploads a tree (host arrays above) to the current device: *tree receives a
 * handle. The arrays are validated (children after their parent and inside
 * the tree, leaf ranges inside order, order a list of faces, depth + 1 <= 64).
 * No reference counterpart (the reference has no device tree). */
int wn_aabb_create(const double* V, int64_t nv, const int64_t* F, int64_t nf,
                   const double* boxes, const int64_t* nodes, const int64_t* order,
                   int64_t nnodes, void** tree);
int wn_aabb_destroy(void* tree);

/* Closest points of np device-resident points (device outputs). Asynchronous
 * on `stream`. No reference counterpart. */
int wn_aabb_squared_distance_device(void* tree, const double* P, int64_t np, double* sqrd,
                                    int64_t* index, double* closest, void* stream);

/* Same with host buffers: copy in, traverse, copy out, synchronise. The GPU
 * counterpart of mli_aabb_squared_distance over all points. */
int wn_aabb_squared_distance_host(void* tree, const double* P, int64_t np, double* sqrd,
                                  int64_t* index, double* closest);

/* The same with the fast winding number (wn_fast_create over the same faces,
 * evaluated at `beta`) for the sign: the sign can differ from the exact one only
 * where |W| lies within the approximation's error of 1/2 (points essentially
 * on the surface of a closed mesh, or near the boundary of an open one). The
 * closest-point and winding-number walks run side by side, the second on a
 * stream of the library's own that is forked from `stream` and joined back to
 * it by events, so all results are ordered on `stream` as usual. */
int wn_signed_distance_fast_device(void* tree, void* fast, double beta, const double* P,
                                   int64_t np, double* s, int64_t* index, double* closest,
                                   double* w, void* stream);

/* Diagnostic: closest point on one triangle (tri9 = A, B, C) from p on the
 * host; out4 = (squared distance, x, y, z), by the arithmetic the host
 * traversal and the GPU kernel share, bit-identical to src/capi.mojo:401-495.
 * Returns 0, or 1 for a null argument. No reference counterpart. */
int wn_closest_point(const double* p, const double* tri9, double* out4);

/* Diagnostic: the eight-lane form of wn_closest_point that the host traversal
 * uses for a leaf's faces (AVX-512), on eight triangles at once: tri72 = rows
 * Ax, Ay, Az, Bx, By, Bz, Cx, Cy, Cz of eight doubles (one triangle per
 * column); out32 = rows squared distance, x, y, z of eight. Every lane is the
 * scalar function's bits. Returns 0, 1 for a null argument, 2 when the CPU has
 * no AVX-512. No reference counterpart. */
int wn_closest_point8(const double* p, const double* tri72, double* out32);

/* Signed distance by the winding-number sign (no reference counterpart):
 * s[i] = -sqrt(sqrd) where |W(P_i)| > 1/2, else +sqrt(sqrd); W comes from the
 * winding-number mesh `mesh` (wn_mixed_mesh_create over the same faces) with
 * precision 0 = FP64 (wn_forward_fp64_mesh_device) or 1 = mixed
 * (wn_forward_mixed_device) and is written to w (np doubles). index and
 * closest as for wn_aabb_squared_distance_device. Device buffers, async. */
int wn_signed_distance_device(void* tree, void* mesh, int precision, const double* P,
                              int64_t np, double* s, int64_t* index, double* closest, double* w,
                              void* stream);

/* ---- per-vertex normals on the GPU --------------------------------------
 * The reference computes them only on the CPU (src/capi.mojo:146-202). Here the
 * topology F (nf x 3 int64, indices in [0, nv)) is prepared once per mesh (a
 * vertex -> (face, corner) list in face order, built on the device) and
 * wn_vertex_normals_device then evaluates N (nv x 3) from V (nv x 3, device
 * doubles, any 8-byte-aligned address) in two launches (one thread per face
 * writes its contribution, one thread per vertex adds its list), summing in the
 * reference's order: uniform and area normals bit-identical to
 * mli_vertex_normals, angle normals through CUDA's acos (within 1e-14). */
int wn_normals_create(const int64_t* F, int64_t nf, int64_t nv, void* stream, void** handle);
int wn_normals_destroy(void* handle);
int wn_vertex_normals_device(void* handle, const double* V, int weighting, double* N,
                             void* stream);
/* One-shot GPU normals with host buffers (prepare, copy in, evaluate, copy out). */
int wn_vertex_normals_host(const double* V, int64_t nv, const int64_t* F, int64_t nf,
                           int weighting, double* N);

/* ---- fast approximate winding numbers (no reference counterpart) --------
 * The hierarchical evaluation of Barill et al., "Fast Winding Numbers for
 * Soups and Clouds" (2018), which the reference lists as not covered
 * (README.md:29): the faces are grouped by the median-split tree, a node whose
 * centre p is farther than beta * r from the query (r: the radius about p
 * holding its vertices) adds its second-order dipole expansion, nearer leaves
 * add their faces' exact solid angles. Larger beta: more exact work, smaller
 * error (beta >= 1; 2 is the published default). Each query sums in a fixed
 * order, so results repeat bit for bit. */

/* Builds the tree and moments on the host (no device work): *handle. */
int wn_fast_create(const double* V, int64_t nv, const int64_t* F, int64_t nf, void** handle);
int wn_fast_destroy(void* handle);
/* out[0..n): faces, nodes, depth. */
int wn_fast_info(void* handle, int64_t* out, int64_t n);
/* Host evaluation of queries [q0, q1) of q (nq x 3) into w; reentrant over disjoint spans. */
int wn_fast_eval_cpu(void* handle, const double* q, int64_t nq, double beta, double* w,
                     int64_t q0, int64_t q1);
/* GPU evaluation of device queries into device w, asynchronous on `stream`. The
 * first GPU call uploads the tree to the current device; the handle then stays
 * on that device. */
int wn_fast_eval_device(void* handle, const double* q, int64_t nq, double beta, double* w,
                        void* stream);
/* Same with host buffers: copy in, evaluate, copy out, synchronise. */
int wn_fast_eval_host(void* handle, const double* q, int64_t nq, double beta, double* w);

#ifdef __cplusplus
}
#endif

#endif /* WN_B200_H */
