// C ABI of libwn_b200 (declared in include/wn_b200.h) and its small runtime:
// one context per CUDA device (stream, SM count, device error word) and a
// grow-only workspace for the host-pointer entry points, all behind one mutex
// so the library is safe to call from the reference shim's worker threads.
//
// The reference creates a DeviceContext, four allocations and a synchronise on
// every call (src/capi.mojo:366-398); here the context and buffers persist and
// only grow. Every device allocation goes through dev_malloc/dev_malloc_async
// (host-side fault injection for the out-of-memory tests), every GPU entry point
// opens an NVTX range, and handles refuse use on another device than their own.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <algorithm>
#include <cstdlib>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/wn_b200.h"
#include "wn_aabb.h"
#include "wn_adjoint.h"
#include "wn_fwn.h"
#include "wn_normals.h"
#include "wn_batch.h"
#include "wn_internal.h"
#include "wn_mixed.h"

namespace wn {

std::atomic<int64_t> g_launches{0};

namespace {

std::atomic<int> g_fault_kind{WN_FAULT_NONE};  // armed kind
std::atomic<int64_t> g_fault_left{0};          // matching events to let through first

// One-shot: true for the armed event that the countdown reaches.
bool fault_fires(int kind) {
  if (g_fault_kind.load(std::memory_order_acquire) != kind) return false;
  if (g_fault_left.fetch_sub(1, std::memory_order_acq_rel) != 0) return false;
  int armed = kind;
  return g_fault_kind.compare_exchange_strong(armed, WN_FAULT_NONE);
}

// WN_INJECT_FAULT=alloc:N arms an allocation fault when the library is loaded.
struct FaultFromEnv {
  FaultFromEnv() {
    const char* s = std::getenv("WN_INJECT_FAULT");
    long long n = -1;
    if (s && std::sscanf(s, "alloc:%lld", &n) == 1 && n >= 0) {
      g_fault_left.store(n);
      g_fault_kind.store(WN_FAULT_ALLOC);
    }
  }
} g_fault_from_env;

}  // namespace

cudaError_t dev_malloc(void** p, size_t bytes) {
  if (fault_fires(WN_FAULT_ALLOC)) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc(p, bytes);
}

cudaError_t dev_malloc_async(void** p, size_t bytes, cudaStream_t stream) {
  if (fault_fires(WN_FAULT_ALLOC)) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMallocAsync(p, bytes, stream);
}

namespace {

constexpr int kMaxDevices = 64;

thread_local std::string t_last_error;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  t_last_error = buf;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  return fail(e == cudaErrorMemoryAllocation ? WN_ENOMEM : WN_ECUDA, "%s: %s (%s)", what,
              cudaGetErrorString(e), cudaGetErrorName(e));
}

// A handle's device memory belongs to the device it was made on: a call made
// while another device is current would launch kernels on memory that device
// cannot address, so it is refused.
int check_device(int handle_device, const char* what) {
  int dev = -1;
  const cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev != handle_device)
    return fail(WN_EINVAL, "%s lives on device %d, but device %d is current", what,
                handle_device, dev);
  return WN_OK;
}

struct Buffer {
  void* ptr = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t need) {
    if (need <= bytes) return cudaSuccess;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
    size_t grow = need + need / 4;
    cudaError_t e = dev_malloc(&ptr, grow);
    if (e != cudaSuccess) {
      ptr = nullptr;
      return e;
    }
    bytes = grow;
    return cudaSuccess;
  }
};

struct DeviceCtx {
  bool ready = false;
  int sms = 0;
  cudaStream_t stream = nullptr;
  int* err = nullptr;  // device error word
  unsigned long long* stats = nullptr;  // mixed-path counters (refined pairs, careful visits)
  Buffer tri, q, w, scratch;
  Buffer mesh_tiles, mesh_tri64, mesh_face_of, mesh_reuse;  // prepared mesh (host entry points)
  Buffer nrm_f, nrm_indptr, nrm_entries, nrm_order, nrm_contrib;  // one-shot vertex normals
  // Second stream and fork/join events for entry points that run two
  // independent kernels side by side (created on first use).
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};

std::mutex g_mutex;
DeviceCtx g_ctx[kMaxDevices];

// Returns the current device's context (initialising it), or null with the
// error recorded.
DeviceCtx* context(int* code) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    *code = fail(WN_ENODEV, "no usable CUDA device: %s", cudaGetErrorString(e));
    return nullptr;
  }
  DeviceCtx& c = g_ctx[dev];
  if (c.ready) return &c;
  if ((e = cudaDeviceGetAttribute(&c.sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess ||
      (!c.stream &&
       (e = cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking)) != cudaSuccess) ||
      (!c.err && (e = dev_malloc(&c.err, sizeof(int))) != cudaSuccess) ||
      (e = cudaMemset(c.err, 0, sizeof(int))) != cudaSuccess ||
      (!c.stats && (e = dev_malloc(&c.stats, 2 * sizeof(unsigned long long))) != cudaSuccess) ||
      (e = cudaMemset(c.stats, 0, 2 * sizeof(unsigned long long))) != cudaSuccess) {
    *code = cuda_fail(e, "device context setup");
    return nullptr;
  }
  // Keep memory freed by cudaFreeAsync in the device's pool across synchronisations
  // (the default threshold of 0 hands it back to the driver at every sync, and the
  // next stream-ordered allocation of the same scratch maps it again).
  cudaMemPool_t pool = nullptr;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  cudaGetLastError();
  c.ready = true;
  return &c;
}

// Reads and clears the device error word after `stream` has drained.
int collect_device_error(DeviceCtx* c, cudaStream_t stream) {
  int h = 0;
  cudaError_t e = cudaMemcpyAsync(&h, c->err, sizeof(int), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return cuda_fail(e, "kernel execution");
  if (h != 0) {
    cudaMemsetAsync(c->err, 0, sizeof(int), stream);
    cudaStreamSynchronize(stream);
    return fail(WN_EDEVICE, "device error word 0x%x (1 = bounded wait ran out, 2 = bad launch)",
                h);
  }
  return WN_OK;
}

int64_t even_ld(int64_t nf) { return ((nf > 0 ? nf : 1) + 1) & ~int64_t(1); }

int forward_fp64_host(const double* tri, const double* q, double* w, int64_t nf, int64_t nq,
                      int mode) {
  if (nf < 0 || nq < 0) return fail(WN_EINVAL, "negative size (nf=%lld, nq=%lld)",
                                    (long long)nf, (long long)nq);
  if (mode != kFp64ArgProd && mode != kFp64Direct && mode != kFp64Tiled)
    return fail(WN_EINVAL, "bad mode %d", mode);
  if (mode == kFp64Tiled && nf > 0x7fffffffLL) return fail(WN_EINVAL, "more than 2^31-1 faces");
  if (nq == 0) return WN_OK;
  if ((nf > 0 && !tri) || !q || !w) return fail(WN_EINVAL, "null pointer");
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  DeviceCtx* c = context(&code);
  if (!c) return code;
  const int64_t ld = even_ld(nf);
  const Fp64Plan plan = plan_fp64(nf, nq, c->sms);
  const Fp64TiledPlan tplan = plan_fp64_tiled(mixed_tiles(nf), nq, c->sms);
  size_t scratch = sizeof(double) * (plan.scratch_doubles + 1);
  if (mode == kFp64Tiled)
    scratch = std::max(mixed_sort_scratch_bytes(nf), sizeof(double) * (tplan.scratch_doubles + 1));
  cudaError_t e;
  if ((e = c->tri.ensure(sizeof(double) * 9 * ld)) != cudaSuccess ||
      (e = c->q.ensure(sizeof(double) * 3 * nq)) != cudaSuccess ||
      (e = c->w.ensure(sizeof(double) * nq)) != cudaSuccess ||
      (e = c->scratch.ensure(scratch)) != cudaSuccess)
    return cuda_fail(e, "device allocation");
  if (mode == kFp64Tiled &&
      ((e = c->mesh_tiles.ensure(mixed_tiles_bytes(nf))) != cudaSuccess ||
       (e = c->mesh_tri64.ensure(mixed_tri64_bytes(nf))) != cudaSuccess ||
       (e = c->mesh_face_of.ensure(mixed_face_of_bytes(nf))) != cudaSuccess ||
       (e = c->mesh_reuse.ensure(mixed_reuse_bytes(nf))) != cudaSuccess))
    return cuda_fail(e, "device allocation");
  double* tri_d = static_cast<double*>(c->tri.ptr);
  double* q_d = static_cast<double*>(c->q.ptr);
  double* w_d = static_cast<double*>(c->w.ptr);
  if (nf > 0 && (e = cudaMemcpy2DAsync(tri_d, sizeof(double) * ld, tri, sizeof(double) * nf,
                                       sizeof(double) * nf, 9, cudaMemcpyHostToDevice,
                                       c->stream)) != cudaSuccess)
    return cuda_fail(e, "copy of the triangle soup");
  if ((e = cudaMemcpyAsync(q_d, q, sizeof(double) * 3 * nq, cudaMemcpyHostToDevice, c->stream)) !=
      cudaSuccess)
    return cuda_fail(e, "copy of the queries");
  if (mode == kFp64Tiled) {
    MixedMesh m;
    m.tiles = static_cast<unsigned char*>(c->mesh_tiles.ptr);
    m.tri64 = static_cast<double*>(c->mesh_tri64.ptr);
    m.face_of = static_cast<uint32_t*>(c->mesh_face_of.ptr);
    m.reuse = static_cast<uint8_t*>(c->mesh_reuse.ptr);
    if ((e = mixed_prepare_mesh(tri_d, ld, nf, 4.0, &m, c->scratch.ptr, c->scratch.bytes,
                                c->stream)) != cudaSuccess)
      return cuda_fail(e, "mesh preparation");
    if ((e = launch_fp64_tiled(tplan, m, q_d, nq, w_d, static_cast<double*>(c->scratch.ptr),
                               c->err, c->stream)) != cudaSuccess)
      return cuda_fail(e, "FP64 winding-number launch");
  } else if ((e = launch_fp64(plan, mode, tri_d, ld, nf, q_d, nq, w_d,
                              static_cast<double*>(c->scratch.ptr), c->err, c->stream)) !=
             cudaSuccess) {
    return cuda_fail(e, "FP64 winding-number launch");
  }
  if ((e = cudaMemcpyAsync(w, w_d, sizeof(double) * nq, cudaMemcpyDeviceToHost, c->stream)) !=
      cudaSuccess)
    return cuda_fail(e, "copy of the result");
  return collect_device_error(c, c->stream);
}

constexpr double kMinKappa = 3.0;  // the 64-face tile angle bound needs kappa >= 3

struct MeshHandle {
  MixedMesh m;
  int device = -1;
};

int check_kappa(double kappa) {
  if (!(kappa >= kMinKappa) || !(kappa <= 1e6))
    return fail(WN_EINVAL, "kappa must lie in [3, 1e6] (got %g)", kappa);
  return WN_OK;
}

int forward_mixed_host(const double* tri, const double* q, double* w, int64_t nf, int64_t nq,
                       double kappa) {
  if (nf < 0 || nq < 0)
    return fail(WN_EINVAL, "negative size (nf=%lld, nq=%lld)", (long long)nf, (long long)nq);
  if (nf > 0x7fffffffLL || nq > 0x7fffffffLL) return fail(WN_EINVAL, "more than 2^31-1 items");
  if (int code = check_kappa(kappa)) return code;
  if (nq == 0) return WN_OK;
  if ((nf > 0 && !tri) || !q || !w) return fail(WN_EINVAL, "null pointer");
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  DeviceCtx* c = context(&code);
  if (!c) return code;
  const int64_t ld = even_ld(nf);
  const size_t scratch = std::max(mixed_sort_scratch_bytes(nf),
                                  mixed_forward_scratch_bytes(mixed_tiles(nf), nq, c->sms));
  cudaError_t e;
  if ((e = c->tri.ensure(sizeof(double) * 9 * ld)) != cudaSuccess ||
      (e = c->q.ensure(sizeof(double) * 3 * nq)) != cudaSuccess ||
      (e = c->w.ensure(sizeof(double) * nq)) != cudaSuccess ||
      (e = c->scratch.ensure(scratch)) != cudaSuccess ||
      (e = c->mesh_tiles.ensure(mixed_tiles_bytes(nf))) != cudaSuccess ||
      (e = c->mesh_tri64.ensure(mixed_tri64_bytes(nf))) != cudaSuccess ||
      (e = c->mesh_face_of.ensure(mixed_face_of_bytes(nf))) != cudaSuccess ||
      (e = c->mesh_reuse.ensure(mixed_reuse_bytes(nf))) != cudaSuccess)
    return cuda_fail(e, "device allocation");
  double* tri_d = static_cast<double*>(c->tri.ptr);
  if (nf > 0 && (e = cudaMemcpy2DAsync(tri_d, sizeof(double) * ld, tri, sizeof(double) * nf,
                                       sizeof(double) * nf, 9, cudaMemcpyHostToDevice,
                                       c->stream)) != cudaSuccess)
    return cuda_fail(e, "copy of the triangle soup");
  if ((e = cudaMemcpyAsync(c->q.ptr, q, sizeof(double) * 3 * nq, cudaMemcpyHostToDevice,
                           c->stream)) != cudaSuccess)
    return cuda_fail(e, "copy of the queries");
  MixedMesh m;
  m.tiles = static_cast<unsigned char*>(c->mesh_tiles.ptr);
  m.tri64 = static_cast<double*>(c->mesh_tri64.ptr);
  m.face_of = static_cast<uint32_t*>(c->mesh_face_of.ptr);
  m.reuse = static_cast<uint8_t*>(c->mesh_reuse.ptr);
  if ((e = mixed_prepare_mesh(tri_d, ld, nf, kappa, &m, c->scratch.ptr, c->scratch.bytes,
                              c->stream)) != cudaSuccess)
    return cuda_fail(e, "mesh preparation");
  if ((e = mixed_forward(m, static_cast<const double*>(c->q.ptr), nq,
                         static_cast<double*>(c->w.ptr), c->scratch.ptr, c->scratch.bytes,
                         c->sms, c->stats, c->err, c->stream)) != cudaSuccess)
    return cuda_fail(e, "mixed winding-number launch");
  if ((e = cudaMemcpyAsync(w, c->w.ptr, sizeof(double) * nq, cudaMemcpyDeviceToHost,
                           c->stream)) != cudaSuccess)
    return cuda_fail(e, "copy of the result");
  return collect_device_error(c, c->stream);
}

[[noreturn]] void out_of_scope(const char* name) {
  std::fprintf(stderr,
               "libwn_b200: %s is not provided: this library implements only the "
               "winding-number, closest-point and vertex-normal paths (mli_winding, "
               "mli_winding_gpu, mli_aabb_squared_distance, mli_vertex_normals)\n",
               name);
  std::abort();
}

}  // namespace

void record_error(const char* message) { t_last_error = message; }

}  // namespace wn

using namespace wn;

extern "C" {

int wn_version(void) { return 100; }

int64_t wn_launch_count(void) { return g_launches.load(); }

int wn_inject_fault(int kind, int64_t after) {
  if (kind != WN_FAULT_NONE && kind != WN_FAULT_ALLOC)
    return fail(WN_EINVAL, "unknown fault kind %d", kind);
  if (after < 0) return fail(WN_EINVAL, "negative countdown");
  g_fault_kind.store(WN_FAULT_NONE);
  g_fault_left.store(after);
  g_fault_kind.store(kind);
  return WN_OK;
}

int wn_fault_armed(void) { return g_fault_kind.load() != WN_FAULT_NONE ? 1 : 0; }

int wn_probe_fma_tflops(int bits, double* tflops) {
  WN_NVTX_RANGE();
  if ((bits != 32 && bits != 64) || !tflops) return fail(WN_EINVAL, "bits must be 32 or 64");
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  DeviceCtx* c = context(&code);
  if (!c) return code;
  cudaError_t e = probe_fma_tflops(bits, c->sms, c->stream, tflops);
  return e == cudaSuccess ? WN_OK : cuda_fail(e, "FMA probe");
}

const char* wn_last_error(void) { return t_last_error.c_str(); }

int wn_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

int wn_device_memory(int64_t* free_bytes, int64_t* total_bytes) {
  size_t f = 0, t = 0;
  cudaError_t e = cudaMemGetInfo(&f, &t);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(WN_ENODEV, "cudaMemGetInfo: %s", cudaGetErrorString(e));
  }
  if (free_bytes) *free_bytes = static_cast<int64_t>(f);
  if (total_bytes) *total_bytes = static_cast<int64_t>(t);
  return WN_OK;
}

int wn_selftest_bounded_wait(int64_t polls) {
  WN_NVTX_RANGE();
  if (polls < 1 || polls > (int64_t(1) << 24)) return fail(WN_EINVAL, "polls must be in [1, 2^24]");
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  DeviceCtx* c = context(&code);
  if (!c) return code;
  cudaError_t e = launch_wait_selftest(static_cast<uint32_t>(polls), c->err, c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "wait self-test launch");
  return collect_device_error(c, c->stream);
}

int wn_stream_check(void* stream) {
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  DeviceCtx* c = context(&code);
  if (!c) return code;
  return collect_device_error(c, static_cast<cudaStream_t>(stream));
}

int wn_forward_fp64_host(const double* tri, const double* q, double* w, int64_t nf, int64_t nq,
                         int mode) {
  WN_NVTX_RANGE();
  return forward_fp64_host(tri, q, w, nf, nq, mode);
}

int wn_forward_fp64_device(const double* tri, int64_t ld, const double* q, double* w, int64_t nf,
                           int64_t nq, int mode, void* stream) {
  WN_NVTX_RANGE();
  if (nf < 0 || nq < 0 || (ld & 1) || ld < nf)
    return fail(WN_EINVAL, "bad sizes (nf=%lld, nq=%lld, ld=%lld; ld must be even and >= nf)",
                (long long)nf, (long long)nq, (long long)ld);
  if (reinterpret_cast<uintptr_t>(tri) & 15) return fail(WN_EINVAL, "tri must be 16-byte aligned");
  if (mode != kFp64ArgProd && mode != kFp64Direct)
    return fail(WN_EINVAL, "bad mode %d (the prepared-mesh mode has its own entry point)", mode);
  if (nq == 0) return WN_OK;
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  DeviceCtx* c = context(&code);
  if (!c) return code;
  const Fp64Plan plan = plan_fp64(nf, nq, c->sms);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // Stream-ordered scratch: calls on different streams never share it.
  double* scratch = nullptr;
  cudaError_t e = cudaSuccess;
  if (plan.scratch_doubles > 0 &&
      (e = dev_malloc_async(reinterpret_cast<void**>(&scratch),
                           sizeof(double) * plan.scratch_doubles, st)) != cudaSuccess)
    return cuda_fail(e, "device allocation");
  e = launch_fp64(plan, mode, tri, ld, nf, q, nq, w, scratch, c->err, st);
  if (scratch) cudaFreeAsync(scratch, st);
  return e == cudaSuccess ? WN_OK : cuda_fail(e, "FP64 winding-number launch");
}

int wn_forward_mixed_host(const double* tri, const double* q, double* w, int64_t nf, int64_t nq,
                          double kappa) {
  WN_NVTX_RANGE();
  return forward_mixed_host(tri, q, w, nf, nq, kappa);
}

int wn_mixed_mesh_create(const double* tri, int64_t ld, int64_t nf, double kappa, void* stream,
                         void** mesh_out) {
  WN_NVTX_RANGE();
  if (!mesh_out) return fail(WN_EINVAL, "null mesh_out");
  *mesh_out = nullptr;
  if (nf < 0 || nf > 0x7fffffffLL || (ld & 1) || ld < nf)
    return fail(WN_EINVAL, "bad sizes (nf=%lld, ld=%lld; ld must be even and >= nf)",
                (long long)nf, (long long)ld);
  if (int code = check_kappa(kappa)) return code;
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  DeviceCtx* c = context(&code);
  if (!c) return code;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  MeshHandle* h = new MeshHandle();
  cudaGetDevice(&h->device);
  cudaError_t e;
  void* scratch = nullptr;
  const size_t sb = mixed_sort_scratch_bytes(nf);
  if ((e = dev_malloc(reinterpret_cast<void**>(&h->m.tiles), mixed_tiles_bytes(nf))) !=
          cudaSuccess ||
      (e = dev_malloc(reinterpret_cast<void**>(&h->m.tri64), mixed_tri64_bytes(nf))) !=
          cudaSuccess ||
      (e = dev_malloc(reinterpret_cast<void**>(&h->m.face_of), mixed_face_of_bytes(nf))) !=
          cudaSuccess ||
      (e = dev_malloc(reinterpret_cast<void**>(&h->m.reuse), mixed_reuse_bytes(nf))) !=
          cudaSuccess ||
      (e = dev_malloc_async(&scratch, sb, st)) != cudaSuccess) {
    cudaFree(h->m.tiles);
    cudaFree(h->m.tri64);
    cudaFree(h->m.face_of);
    cudaFree(h->m.reuse);
    delete h;
    return cuda_fail(e, "device allocation");
  }
  e = mixed_prepare_mesh(tri, ld, nf, kappa, &h->m, scratch, sb, st);
  cudaFreeAsync(scratch, st);
  if (e != cudaSuccess) {
    cudaStreamSynchronize(st);
    cudaFree(h->m.tiles);
    cudaFree(h->m.tri64);
    cudaFree(h->m.face_of);
    cudaFree(h->m.reuse);
    delete h;
    return cuda_fail(e, "mesh preparation");
  }
  *mesh_out = h;
  return WN_OK;
}

int wn_mixed_mesh_destroy(void* mesh) {
  if (!mesh) return WN_OK;
  MeshHandle* h = static_cast<MeshHandle*>(mesh);
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(h->device);
  cudaDeviceSynchronize();
  cudaFree(h->m.tiles);
  cudaFree(h->m.tri64);
  cudaFree(h->m.face_of);
  cudaFree(h->m.reuse);
  cudaSetDevice(prev);
  delete h;
  return WN_OK;
}

int wn_forward_mixed_device(void* mesh, const double* q, int64_t nq, double* w, void* stream) {
  WN_NVTX_RANGE();
  if (!mesh) return fail(WN_EINVAL, "null mesh");
  if (nq < 0 || nq > 0x7fffffffLL) return fail(WN_EINVAL, "bad nq=%lld", (long long)nq);
  if (nq == 0) return WN_OK;
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  DeviceCtx* c = context(&code);
  if (!c) return code;
  const MeshHandle* h = static_cast<const MeshHandle*>(mesh);
  if ((code = check_device(h->device, "mesh")) != WN_OK) return code;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t sb = mixed_forward_scratch_bytes(h->m.ntiles, nq, c->sms);
  void* scratch = nullptr;
  cudaError_t e = dev_malloc_async(&scratch, sb, st);
  if (e != cudaSuccess) return cuda_fail(e, "device allocation");
  e = mixed_forward(h->m, q, nq, w, scratch, sb, c->sms, c->stats, c->err, st);
  cudaFreeAsync(scratch, st);
  return e == cudaSuccess ? WN_OK : cuda_fail(e, "mixed winding-number launch");
}

int wn_forward_fp64_mesh_device(void* mesh, const double* q, int64_t nq, double* w,
                                void* stream) {
  WN_NVTX_RANGE();
  if (!mesh) return fail(WN_EINVAL, "null mesh");
  if (nq < 0 || nq > 0x7fffffffLL) return fail(WN_EINVAL, "bad nq=%lld", (long long)nq);
  if (nq == 0) return WN_OK;
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  DeviceCtx* c = context(&code);
  if (!c) return code;
  const MeshHandle* h = static_cast<const MeshHandle*>(mesh);
  if ((code = check_device(h->device, "mesh")) != WN_OK) return code;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const Fp64TiledPlan p = plan_fp64_tiled(h->m.ntiles, nq, c->sms);
  double* scratch = nullptr;
  cudaError_t e = cudaSuccess;
  if (p.scratch_doubles > 0 &&
      (e = dev_malloc_async(reinterpret_cast<void**>(&scratch), sizeof(double) * p.scratch_doubles,
                           st)) != cudaSuccess)
    return cuda_fail(e, "device allocation");
  e = launch_fp64_tiled(p, h->m, q, nq, w, scratch, c->err, st);
  if (scratch) cudaFreeAsync(scratch, st);
  return e == cudaSuccess ? WN_OK : cuda_fail(e, "FP64 winding-number launch");
}

int wn_mixed_sort_queries(const double* q, int64_t nq, uint32_t* perm, void* stream) {
  WN_NVTX_RANGE();
  if (nq < 0 || nq > 0x7fffffffLL) return fail(WN_EINVAL, "bad nq=%lld", (long long)nq);
  if (nq == 0) return WN_OK;
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  if (!context(&code)) return code;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t sb = mixed_sort_scratch_bytes(nq);
  void* scratch = nullptr;
  cudaError_t e = dev_malloc_async(&scratch, sb, st);
  if (e != cudaSuccess) return cuda_fail(e, "device allocation");
  e = mixed_sort_queries(q, nq, perm, scratch, sb, st);
  cudaFreeAsync(scratch, st);
  return e == cudaSuccess ? WN_OK : cuda_fail(e, "query sort");
}

int wn_forward_mixed_sorted_device(void* mesh, const double* q, const uint32_t* perm, int64_t nq,
                                   double* w, void* stream) {
  WN_NVTX_RANGE();
  if (!mesh) return fail(WN_EINVAL, "null mesh");
  if (nq < 0 || nq > 0x7fffffffLL) return fail(WN_EINVAL, "bad nq=%lld", (long long)nq);
  if (nq == 0) return WN_OK;
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  DeviceCtx* c = context(&code);
  if (!c) return code;
  const MeshHandle* h = static_cast<const MeshHandle*>(mesh);
  if ((code = check_device(h->device, "mesh")) != WN_OK) return code;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const MixedSplit p = plan_mixed(h->m.ntiles, nq, c->sms);
  double* partial = nullptr;
  cudaError_t e = cudaSuccess;
  if (p.partial_doubles > 0 &&
      (e = dev_malloc_async(reinterpret_cast<void**>(&partial), sizeof(double) * p.partial_doubles,
                           st)) != cudaSuccess)
    return cuda_fail(e, "device allocation");
  e = mixed_forward_sorted(h->m, q, perm, nq, w, p, partial, c->stats, c->err, st);
  if (partial) cudaFreeAsync(partial, st);
  return e == cudaSuccess ? WN_OK : cuda_fail(e, "mixed winding-number launch");
}

int wn_mixed_mesh_update(void* mesh, const double* tri, int64_t ld, void* stream) {
  WN_NVTX_RANGE();
  if (!mesh) return fail(WN_EINVAL, "null mesh");
  MeshHandle* h = static_cast<MeshHandle*>(mesh);
  if ((ld & 1) || ld < h->m.nf)
    return fail(WN_EINVAL, "bad ld=%lld for a mesh of %lld faces", (long long)ld,
                (long long)h->m.nf);
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  if (!context(&code)) return code;
  if ((code = check_device(h->device, "mesh")) != WN_OK) return code;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t sb = mixed_sort_scratch_bytes(h->m.nf);
  void* scratch = nullptr;
  cudaError_t e = dev_malloc_async(&scratch, sb, st);
  if (e != cudaSuccess) return cuda_fail(e, "device allocation");
  e = mixed_prepare_mesh(tri, ld, h->m.nf, h->m.kappa, &h->m, scratch, sb, st);
  cudaFreeAsync(scratch, st);
  return e == cudaSuccess ? WN_OK : cuda_fail(e, "mesh preparation");
}

int wn_mixed_mesh_set_tile_faces(void* mesh, int tile_faces) {
  if (!mesh) return fail(WN_EINVAL, "null mesh");
  if (tile_faces != kTileFaces && tile_faces != kHalfFaces)
    return fail(WN_EINVAL, "tile_faces must be 64 or 32");
  std::lock_guard<std::mutex> lock(g_mutex);
  static_cast<MeshHandle*>(mesh)->m.tile_faces = tile_faces;
  return WN_OK;
}

int wn_mixed_stats(int64_t* refined_pairs, int64_t* careful_visits, int reset) {
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  DeviceCtx* c = context(&code);
  if (!c) return code;
  unsigned long long h[2] = {0, 0};
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(h, c->stats, sizeof(h), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && reset) e = cudaMemset(c->stats, 0, sizeof(h));
  if (e != cudaSuccess) return cuda_fail(e, "reading mixed-path counters");
  if (refined_pairs) *refined_pairs = static_cast<int64_t>(h[0]);
  if (careful_visits) *careful_visits = static_cast<int64_t>(h[1]);
  return WN_OK;
}

int wn_backward_fp64_device(const double* tri, int64_t ld, int64_t nf, const double* q,
                            int64_t nq, const double* gw, double* dq, double* dtri, void* stream) {
  WN_NVTX_RANGE();
  if (nf < 0 || nq < 0 || (ld & 1) || ld < nf)
    return fail(WN_EINVAL, "bad sizes (nf=%lld, nq=%lld, ld=%lld; ld must be even and >= nf)",
                (long long)nf, (long long)nq, (long long)ld);
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  DeviceCtx* c = context(&code);
  if (!c) return code;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const AdjointPlan p = plan_adjoint(nf, nq, c->sms);
  const size_t sb = adjoint_scratch_bytes(p, ld, nq);
  void* scratch = nullptr;
  cudaError_t e = dev_malloc_async(&scratch, sb, st);
  if (e != cudaSuccess) return cuda_fail(e, "device allocation");
  e = adjoint_fp64(p, tri, ld, nf, q, nq, gw, dq, dtri, scratch, sb, st);
  cudaFreeAsync(scratch, st);
  return e == cudaSuccess ? WN_OK : cuda_fail(e, "FP64 adjoint launch");
}

int wn_backward_mixed_device(void* mesh, const double* q, int64_t nq, const double* gw,
                             double* dq, double* dtri, int64_t ld, void* stream) {
  WN_NVTX_RANGE();
  if (!mesh) return fail(WN_EINVAL, "null mesh");
  const MeshHandle* h = static_cast<const MeshHandle*>(mesh);
  if (nq < 0 || nq > 0x7fffffffLL || (ld & 1) || ld < h->m.nf)
    return fail(WN_EINVAL, "bad sizes (nq=%lld, ld=%lld for %lld faces)", (long long)nq,
                (long long)ld, (long long)h->m.nf);
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  DeviceCtx* c = context(&code);
  if (!c) return code;
  if ((code = check_device(h->device, "mesh")) != WN_OK) return code;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const AdjointPlan p = plan_adjoint_mixed(h->m.ntiles, nq, c->sms);
  const size_t perm_bytes = ((static_cast<size_t>(std::max<int64_t>(nq, 1)) * 4 + 255) / 256) * 256;
  const size_t sort_bytes = mixed_sort_scratch_bytes(nq);
  const size_t adj_bytes = adjoint_scratch_bytes(p, h->m.ld64, nq);
  unsigned char* scratch = nullptr;
  cudaError_t e = dev_malloc_async(reinterpret_cast<void**>(&scratch),
                                  perm_bytes + std::max(sort_bytes, adj_bytes), st);
  if (e != cudaSuccess) return cuda_fail(e, "device allocation");
  uint32_t* perm = reinterpret_cast<uint32_t*>(scratch);
  e = mixed_sort_queries(q, nq, perm, scratch + perm_bytes, sort_bytes, st);
  if (e == cudaSuccess)
    e = adjoint_mixed(p, h->m, q, perm, nq, gw, dq, dtri, ld, scratch + perm_bytes, adj_bytes,
                      st);
  cudaFreeAsync(scratch, st);
  return e == cudaSuccess ? WN_OK : cuda_fail(e, "mixed adjoint launch");
}

int wn_backward_edges_device(const double* edges, int64_t le, int64_t ne, const double* q,
                             int64_t nq, const double* gw, double* dq, double* dedge,
                             void* stream) {
  WN_NVTX_RANGE();
  if (ne < 0 || nq < 0 || le < ne)
    return fail(WN_EINVAL, "bad sizes (ne=%lld, nq=%lld, le=%lld)", (long long)ne,
                (long long)nq, (long long)le);
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  DeviceCtx* c = context(&code);
  if (!c) return code;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const AdjointPlan p = plan_adjoint_edges(ne, nq, c->sms);
  const size_t sb = adjoint_edges_scratch_bytes(p, le, nq);
  void* scratch = nullptr;
  cudaError_t e = dev_malloc_async(&scratch, sb, st);
  if (e != cudaSuccess) return cuda_fail(e, "device allocation");
  e = adjoint_edges(p, edges, le, ne, q, nq, gw, dq, dedge, scratch, sb, st);
  cudaFreeAsync(scratch, st);
  return e == cudaSuccess ? WN_OK : cuda_fail(e, "boundary-edge adjoint launch");
}

int wn_backward_edges_mixed_device(const double* edges, int64_t le, int64_t ne, const double* q,
                                   int64_t nq, const double* gw, double kappa, int unit_weights,
                                   double* dq, double* dedge, void* stream) {
  WN_NVTX_RANGE();
  if (ne < 0 || nq < 0 || le < ne || nq > 0x7fffffffLL || ne > 0x7fffffffLL)
    return fail(WN_EINVAL, "bad sizes (ne=%lld, nq=%lld, le=%lld)", (long long)ne,
                (long long)nq, (long long)le);
  if (int code = check_kappa(kappa)) return code;
  if (!dq && !unit_weights) return fail(WN_EINVAL, "dq is required unless unit_weights = 1");
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  DeviceCtx* c = context(&code);
  if (!c) return code;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const AdjointPlan p = plan_adjoint_edges_mixed(ne, nq, c->sms, dq == nullptr);
  const size_t sb = adjoint_edges_mixed_scratch_bytes(p, ne, nq);
  void* scratch = nullptr;
  cudaError_t e = dev_malloc_async(&scratch, sb, st);
  if (e != cudaSuccess) return cuda_fail(e, "device allocation");
  e = adjoint_edges_mixed(p, edges, le, ne, q, nq, gw, kappa, unit_weights != 0, dq, dedge,
                          scratch, sb, st);
  cudaFreeAsync(scratch, st);
  return e == cudaSuccess ? WN_OK : cuda_fail(e, "mixed boundary-edge adjoint launch");
}

int wn_gather_vertex_grad_device(const double* dtri, int64_t ld, int corners,
                                 const int64_t* indptr, const int64_t* entries, int64_t nv,
                                 double* dV, void* stream) {
  WN_NVTX_RANGE();
  if (nv < 0 || (corners != 2 && corners != 3))
    return fail(WN_EINVAL, "bad nv=%lld or corners=%d", (long long)nv, corners);
  cudaError_t e = gather_vertex_grad(dtri, ld, corners, indptr, entries, nv, dV,
                                     static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? WN_OK : cuda_fail(e, "vertex gradient gather");
}

int wn_batch_create(int64_t nmesh, const int64_t* nv, const int64_t* nf, const int64_t* nq,
                    const int64_t* faces, double kappa, int qpt, int64_t target_pairs,
                    int ctas_per_sm, int tile_faces, void** batch_out) {
  WN_NVTX_RANGE();
  if (!batch_out) return fail(WN_EINVAL, "null batch_out");
  *batch_out = nullptr;
  if (nmesh <= 0 || nmesh > (1 << 20) || !nv || !nf || !nq)
    return fail(WN_EINVAL, "bad mesh count %lld or null size arrays", (long long)nmesh);
  int64_t tf = 0, tq = 0, tv = 0;
  for (int64_t m = 0; m < nmesh; ++m) {
    if (nv[m] < 0 || nf[m] < 0 || nq[m] < 0) return fail(WN_EINVAL, "negative size in mesh %lld",
                                                         (long long)m);
    tv += nv[m];
    tf += nf[m];
    tq += nq[m];
  }
  if (tf > 0x7fffffffLL || tq > 0x7fffffffLL) return fail(WN_EINVAL, "more than 2^31-1 items");
  if (tf > 0 && !faces) return fail(WN_EINVAL, "null faces");
  for (int64_t m = 0, f0 = 0; m < nmesh; f0 += nf[m], ++m)
    for (int64_t i = 3 * f0; i < 3 * (f0 + nf[m]); ++i)
      if (faces[i] < 0 || faces[i] >= nv[m])
        return fail(WN_EINVAL, "face index %lld outside mesh %lld's %lld vertices",
                    (long long)faces[i], (long long)m, (long long)nv[m]);
  if (int code = check_kappa(kappa)) return code;
  if (qpt != 1 && qpt != 2 && qpt != 4) return fail(WN_EINVAL, "qpt must be 1, 2 or 4");
  if (target_pairs < 1) return fail(WN_EINVAL, "target_pairs must be positive");
  if (tile_faces != kTileFaces && tile_faces != kHalfFaces)
    return fail(WN_EINVAL, "tile_faces must be 64 or 32");
  if (ctas_per_sm < 0) return fail(WN_EINVAL, "ctas_per_sm must be >= 0");
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  DeviceCtx* c = context(&code);
  if (!c) return code;
  BatchPlan plan;
  plan.tile_faces = tile_faces;
  plan.qpt = qpt;
  plan.kappa = kappa;
  plan.target_pairs = target_pairs;
  plan.ctas_per_sm = ctas_per_sm;
  BatchState* b = new BatchState();
  cudaError_t e = batch_create(b, nmesh, nv, nf, nq, faces, plan, c->sms);
  if (e == cudaSuccess) e = batch_edges_create(b, faces);
  if (e != cudaSuccess) {
    batch_edges_destroy(b);
    batch_destroy(b);
    delete b;
    return cuda_fail(e, "batch setup");
  }
  *batch_out = b;
  return WN_OK;
}

int wn_batch_forward(void* batch, const double* V, const double* q, double* w, void* stream) {
  WN_NVTX_RANGE();
  if (!batch) return fail(WN_EINVAL, "null batch");
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  DeviceCtx* c = context(&code);
  if (!c) return code;
  if ((code = check_device(static_cast<const BatchState*>(batch)->device, "batch")) != WN_OK)
    return code;
  cudaError_t e = batch_forward(static_cast<BatchState*>(batch), V, q, w, c->stats, c->err,
                                static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? WN_OK : cuda_fail(e, "batched forward launch");
}

int wn_batch_backward(void* batch, const double* V, const double* q, const double* gw,
                      double* dq, double* dV, void* stream) {
  WN_NVTX_RANGE();
  if (!batch) return fail(WN_EINVAL, "null batch");
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  if (!context(&code)) return code;
  if ((code = check_device(static_cast<const BatchState*>(batch)->device, "batch")) != WN_OK)
    return code;
  cudaError_t e = batch_backward(static_cast<BatchState*>(batch), V, q, gw, dq, dV,
                                 static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? WN_OK : cuda_fail(e, "batched adjoint launch");
}

int wn_batch_set_adjoint_fp64(void* batch, int fp64) {
  if (!batch) return fail(WN_EINVAL, "null batch");
  if (fp64 != 0 && fp64 != 1) return fail(WN_EINVAL, "fp64 must be 0 or 1, got %d", fp64);
  std::lock_guard<std::mutex> lock(g_mutex);
  batch_set_adjoint_fp64(static_cast<BatchState*>(batch), fp64 != 0);
  return WN_OK;
}

int wn_batch_info(void* batch, int64_t* out, int64_t n) {
  if (!batch || !out) return fail(WN_EINVAL, "null argument");
  const BatchState* b = static_cast<const BatchState*>(batch);
  const int64_t vals[] = {b->nmesh,       b->total_nv,    b->total_nf, b->total_nq,
                          b->total_tiles, b->n_items,     b->grid,     b->total_partials,
                          b->plan.qpt,    b->plan.target_pairs,
                          batch_boundary_edges(b), batch_edge_items(b), b->plan.tile_faces,
                          batch_adjoint_fp64(b) ? 1 : 0};
  for (int64_t i = 0; i < n && i < static_cast<int64_t>(sizeof(vals) / sizeof(vals[0])); ++i)
    out[i] = vals[i];
  return WN_OK;
}

int wn_batch_destroy(void* batch) {
  if (!batch) return WN_OK;
  BatchState* b = static_cast<BatchState*>(batch);
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(b->device);
  cudaDeviceSynchronize();
  batch_edges_destroy(b);
  batch_destroy(b);
  cudaSetDevice(prev);
  delete b;
  return WN_OK;
}

// ---- closest points -------------------------------------------------------
namespace {

struct AabbHandle {
  AabbDeviceTree t;
  int device = -1;
};

size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

// Bytes of the Morton permutation + its sort scratch for np points (0 below
// the sorting threshold).
size_t aabb_sort_bytes(int64_t np) {
  return np >= kAabbSortMin ? align256(sizeof(uint32_t) * np) + mixed_sort_scratch_bytes(np) : 0;
}

// Sorts (when np is large enough) and traverses; scratch holds aabb_sort_bytes(np).
cudaError_t aabb_run(const AabbHandle* h, const double* P, int64_t np, double* sqrd,
                     int64_t* index, double* closest, void* scratch, int* err, cudaStream_t st) {
  uint32_t* perm = nullptr;
  cudaError_t e = cudaSuccess;
  if (np >= kAabbSortMin) {
    perm = static_cast<uint32_t*>(scratch);
    unsigned char* rest = static_cast<unsigned char*>(scratch) + align256(sizeof(uint32_t) * np);
    if ((e = mixed_sort_queries(P, np, perm, rest, mixed_sort_scratch_bytes(np), st)) !=
        cudaSuccess)
      return e;
  }
  return aabb_query(h->t, P, np, perm, sqrd, index, closest, err, st);
}

int check_points(const void* tree, int64_t np) {
  if (!tree) return fail(WN_EINVAL, "null tree");
  if (np < 0 || np > 0x7fffffffLL) return fail(WN_EINVAL, "bad np=%lld", (long long)np);
  return WN_OK;
}

}  // namespace

int64_t wn_aabb_node_count(int64_t nf, int64_t leaf_size) {
  return leaf_size < 1 ? -1 : aabb_node_count(nf, leaf_size);
}

int wn_aabb_build(const double* V, int64_t nv, const int64_t* F, int64_t nf, int64_t leaf_size,
                  double* boxes, int64_t* nodes, int64_t* order, int64_t* stack_size,
                  int threads) {
  if (!stack_size) return fail(WN_EINVAL, "null stack_size");
  const char* why = "";
  const int64_t s = aabb_build(V, nv, F, nf, leaf_size, boxes, nodes, order, threads, &why);
  if (s < 0) return fail(WN_EINVAL, "cannot build the tree: %s", why);
  *stack_size = s;
  return WN_OK;
}

int wn_aabb_create(const double* V, int64_t nv, const int64_t* F, int64_t nf,
                   const double* boxes, const int64_t* nodes, const int64_t* order,
                   int64_t nnodes, void** tree) {
  WN_NVTX_RANGE();
  if (!tree) return fail(WN_EINVAL, "null output handle");
  *tree = nullptr;
  if (nv < 0 || nf < 0 || nnodes < 0) return fail(WN_EINVAL, "negative size");
  if (nnodes > 0 && (!V || !F || !boxes || !nodes || !order))
    return fail(WN_EINVAL, "null pointer");
  std::vector<AabbNodeRec> nrec(static_cast<size_t>(nnodes));
  std::vector<AabbTriRec> trec(static_cast<size_t>(nnodes > 0 ? nf : 0));
  const char* why = "";
  double scale = 0.0;
  const int64_t depth = aabb_pack(V, nv, F, nf, boxes, nodes, order, nnodes, nrec.data(),
                                  trec.data(), &scale, &why);
  if (depth < 0) return fail(WN_EINVAL, "invalid tree: %s", why);
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  if (!context(&code)) return code;
  AabbHandle* h = new AabbHandle();
  cudaGetDevice(&h->device);
  h->t.nnodes = nnodes;
  h->t.nleaf_faces = static_cast<int64_t>(trec.size());
  h->t.depth = static_cast<int>(depth);
  h->t.scale = scale;
  if (nnodes > 0) {
    for (int k = 0; k < 6; ++k) h->t.root[k] = boxes[k];
    cudaError_t e;
    if ((e = dev_malloc(&h->t.nodes, sizeof(AabbNodeRec) * nrec.size())) != cudaSuccess ||
        (e = dev_malloc(&h->t.tris, sizeof(AabbTriRec) * trec.size())) != cudaSuccess ||
        (e = cudaMemcpy(h->t.nodes, nrec.data(), sizeof(AabbNodeRec) * nrec.size(),
                        cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(h->t.tris, trec.data(), sizeof(AabbTriRec) * trec.size(),
                        cudaMemcpyHostToDevice)) != cudaSuccess) {
      cudaFree(h->t.nodes);
      cudaFree(h->t.tris);
      delete h;
      return cuda_fail(e, "device tree upload");
    }
  }
  *tree = h;
  return WN_OK;
}

int wn_aabb_destroy(void* tree) {
  if (!tree) return WN_OK;
  AabbHandle* h = static_cast<AabbHandle*>(tree);
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(h->device);
  cudaDeviceSynchronize();
  cudaFree(h->t.nodes);
  cudaFree(h->t.tris);
  cudaSetDevice(prev);
  delete h;
  return WN_OK;
}

int wn_aabb_squared_distance_device(void* tree, const double* P, int64_t np, double* sqrd,
                                    int64_t* index, double* closest, void* stream) {
  WN_NVTX_RANGE();
  if (int code = check_points(tree, np)) return code;
  if (np == 0) return WN_OK;
  if (!P || !sqrd || !index || !closest) return fail(WN_EINVAL, "null pointer");
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  DeviceCtx* c = context(&code);
  if (!c) return code;
  if ((code = check_device(static_cast<const AabbHandle*>(tree)->device, "tree")) != WN_OK)
    return code;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t sb = aabb_sort_bytes(np);
  void* scratch = nullptr;
  cudaError_t e = cudaSuccess;
  if (sb && (e = dev_malloc_async(&scratch, sb, st)) != cudaSuccess)
    return cuda_fail(e, "device allocation");
  e = aabb_run(static_cast<const AabbHandle*>(tree), P, np, sqrd, index, closest, scratch, c->err,
               st);
  if (scratch) cudaFreeAsync(scratch, st);
  return e == cudaSuccess ? WN_OK : cuda_fail(e, "closest-point launch");
}

int wn_aabb_squared_distance_host(void* tree, const double* P, int64_t np, double* sqrd,
                                  int64_t* index, double* closest) {
  WN_NVTX_RANGE();
  if (int code = check_points(tree, np)) return code;
  if (np == 0) return WN_OK;
  if (!P || !sqrd || !index || !closest) return fail(WN_EINVAL, "null pointer");
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  DeviceCtx* c = context(&code);
  if (!c) return code;
  if ((code = check_device(static_cast<const AabbHandle*>(tree)->device, "tree")) != WN_OK)
    return code;
  const size_t out_bytes = align256(sizeof(int64_t) * np) + align256(sizeof(double) * 3 * np);
  cudaError_t e;
  if ((e = c->q.ensure(sizeof(double) * 3 * np)) != cudaSuccess ||
      (e = c->w.ensure(sizeof(double) * np)) != cudaSuccess ||
      (e = c->scratch.ensure(out_bytes + aabb_sort_bytes(np))) != cudaSuccess)
    return cuda_fail(e, "device allocation");
  unsigned char* s = static_cast<unsigned char*>(c->scratch.ptr);
  int64_t* index_d = reinterpret_cast<int64_t*>(s);
  double* closest_d = reinterpret_cast<double*>(s + align256(sizeof(int64_t) * np));
  double* P_d = static_cast<double*>(c->q.ptr);
  double* sqrd_d = static_cast<double*>(c->w.ptr);
  if ((e = cudaMemcpyAsync(P_d, P, sizeof(double) * 3 * np, cudaMemcpyHostToDevice,
                           c->stream)) != cudaSuccess)
    return cuda_fail(e, "copy of the points");
  if ((e = aabb_run(static_cast<const AabbHandle*>(tree), P_d, np, sqrd_d, index_d, closest_d,
                    s + out_bytes, c->err, c->stream)) != cudaSuccess)
    return cuda_fail(e, "closest-point launch");
  if ((e = cudaMemcpyAsync(sqrd, sqrd_d, sizeof(double) * np, cudaMemcpyDeviceToHost,
                           c->stream)) != cudaSuccess ||
      (e = cudaMemcpyAsync(index, index_d, sizeof(int64_t) * np, cudaMemcpyDeviceToHost,
                           c->stream)) != cudaSuccess ||
      (e = cudaMemcpyAsync(closest, closest_d, sizeof(double) * 3 * np, cudaMemcpyDeviceToHost,
                           c->stream)) != cudaSuccess)
    return cuda_fail(e, "copy of the results");
  return collect_device_error(c, c->stream);
}

int wn_signed_distance_device(void* tree, void* mesh, int precision, const double* P,
                              int64_t np, double* s, int64_t* index, double* closest, double* w,
                              void* stream) {
  WN_NVTX_RANGE();
  if (int code = check_points(tree, np)) return code;
  if (!mesh) return fail(WN_EINVAL, "null mesh");
  if (precision != 0 && precision != 1) return fail(WN_EINVAL, "bad precision %d", precision);
  if (np == 0) return WN_OK;
  if (!w) return fail(WN_EINVAL, "null pointer");
  if (int code = wn_aabb_squared_distance_device(tree, P, np, s, index, closest, stream))
    return code;
  if (int code = precision == 0 ? wn_forward_fp64_mesh_device(mesh, P, np, w, stream)
                                : wn_forward_mixed_device(mesh, P, np, w, stream))
    return code;
  std::lock_guard<std::mutex> lock(g_mutex);
  const cudaError_t e = signed_from_winding(w, s, np, static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? WN_OK : cuda_fail(e, "signed-distance launch");
}

// ---- fast (hierarchical) winding numbers ----------------------------------
namespace {

struct FwnHandle {
  FwnHostTree host;
  FwnDeviceTree dev;
  int device = -1;  // device holding `dev` (-1: not uploaded yet)
};

int check_beta(double beta) {
  if (!(beta >= 1.0) || !(beta <= 1e12))
    return fail(WN_EINVAL, "beta must lie in [1, 1e12] (got %g)", beta);
  return WN_OK;
}

// Uploads the tree to the current device on first use; the handle then stays
// bound to that device.
int fwn_upload(FwnHandle* h) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (h->device >= 0) {
    if (h->device != dev)
      return fail(WN_EINVAL, "fast winding-number handle lives on device %d, not %d",
                  h->device, dev);
    return WN_OK;
  }
  FwnDeviceTree& d = h->dev;
  d.nnodes = h->host.nnodes;
  d.depth = h->host.depth;
  if (d.nnodes > 0) {
    cudaError_t e;
    if ((e = dev_malloc(&d.nodes, sizeof(FwnNode) * d.nnodes)) != cudaSuccess ||
        (e = dev_malloc(&d.moments, sizeof(FwnMoments) * d.nnodes)) != cudaSuccess ||
        (e = dev_malloc(&d.tris, sizeof(AabbTriRec) * h->host.nf)) != cudaSuccess ||
        (e = cudaMemcpy(d.nodes, h->host.nodes, sizeof(FwnNode) * d.nnodes,
                        cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(d.moments, h->host.moments, sizeof(FwnMoments) * d.nnodes,
                        cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(d.tris, h->host.tris, sizeof(AabbTriRec) * h->host.nf,
                        cudaMemcpyHostToDevice)) != cudaSuccess) {
      cudaFree(d.nodes);
      cudaFree(d.moments);
      cudaFree(d.tris);
      d = FwnDeviceTree{};
      return cuda_fail(e, "fast winding-number tree upload");
    }
  }
  h->device = dev;
  return WN_OK;
}

cudaError_t fwn_run(const FwnHandle* h, const double* q, int64_t nq, double beta, double* w,
                    void* scratch, int* err, cudaStream_t st) {
  uint32_t* perm = nullptr;
  if (nq >= kAabbSortMin) {
    perm = static_cast<uint32_t*>(scratch);
    unsigned char* rest = static_cast<unsigned char*>(scratch) + align256(sizeof(uint32_t) * nq);
    cudaError_t e = mixed_sort_queries(q, nq, perm, rest, mixed_sort_scratch_bytes(nq), st);
    if (e != cudaSuccess) return e;
  }
  return fwn_eval_device(h->dev, q, nq, perm, beta, w, err, st);
}

}  // namespace

int wn_fast_create(const double* V, int64_t nv, const int64_t* F, int64_t nf, void** out) {
  if (!out) return fail(WN_EINVAL, "null output handle");
  *out = nullptr;
  if (nf > 0 && (!V || !F)) return fail(WN_EINVAL, "null pointer");
  FwnHandle* h = new FwnHandle();
  const char* why = "";
  if (fwn_build(V, nv, F, nf, 0, &h->host, &why) != 0) {
    delete h;
    return fail(WN_EINVAL, "cannot build the fast winding-number tree: %s", why);
  }
  *out = h;
  return WN_OK;
}

int wn_fast_destroy(void* handle) {
  if (!handle) return WN_OK;
  FwnHandle* h = static_cast<FwnHandle*>(handle);
  if (h->device >= 0) {
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(h->device);
    cudaDeviceSynchronize();
    cudaFree(h->dev.nodes);
    cudaFree(h->dev.moments);
    cudaFree(h->dev.tris);
    cudaSetDevice(prev);
  }
  fwn_free(&h->host);
  delete h;
  return WN_OK;
}

int wn_fast_info(void* handle, int64_t* out, int64_t n) {
  if (!handle || !out) return fail(WN_EINVAL, "null argument");
  const FwnHandle* h = static_cast<const FwnHandle*>(handle);
  const int64_t vals[] = {h->host.nf, h->host.nnodes, h->host.depth};
  for (int64_t i = 0; i < n && i < 3; ++i) out[i] = vals[i];
  return WN_OK;
}

int wn_fast_eval_cpu(void* handle, const double* q, int64_t nq, double beta, double* w,
                     int64_t q0, int64_t q1) {
  if (!handle) return fail(WN_EINVAL, "null handle");
  if (int code = check_beta(beta)) return code;
  if (nq < 0 || q0 < 0 || q1 > nq || q0 > q1) return fail(WN_EINVAL, "bad query range");
  if (q1 == q0) return WN_OK;
  if (!q || !w) return fail(WN_EINVAL, "null pointer");
  fwn_eval_host(static_cast<const FwnHandle*>(handle)->host, q, q0, q1, beta, w);
  return WN_OK;
}

int wn_fast_eval_device(void* handle, const double* q, int64_t nq, double beta, double* w,
                        void* stream) {
  WN_NVTX_RANGE();
  if (!handle) return fail(WN_EINVAL, "null handle");
  if (int code = check_beta(beta)) return code;
  if (nq < 0 || nq > 0x7fffffffLL) return fail(WN_EINVAL, "bad nq=%lld", (long long)nq);
  if (nq == 0) return WN_OK;
  if (!q || !w) return fail(WN_EINVAL, "null pointer");
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  DeviceCtx* c = context(&code);
  if (!c) return code;
  FwnHandle* h = static_cast<FwnHandle*>(handle);
  if ((code = fwn_upload(h)) != WN_OK) return code;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t sb = aabb_sort_bytes(nq);
  void* scratch = nullptr;
  cudaError_t e = cudaSuccess;
  if (sb && (e = dev_malloc_async(&scratch, sb, st)) != cudaSuccess)
    return cuda_fail(e, "device allocation");
  e = fwn_run(h, q, nq, beta, w, scratch, c->err, st);
  if (scratch) cudaFreeAsync(scratch, st);
  return e == cudaSuccess ? WN_OK : cuda_fail(e, "fast winding-number launch");
}

int wn_fast_eval_host(void* handle, const double* q, int64_t nq, double beta, double* w) {
  WN_NVTX_RANGE();
  if (!handle) return fail(WN_EINVAL, "null handle");
  if (int code = check_beta(beta)) return code;
  if (nq < 0 || nq > 0x7fffffffLL) return fail(WN_EINVAL, "bad nq=%lld", (long long)nq);
  if (nq == 0) return WN_OK;
  if (!q || !w) return fail(WN_EINVAL, "null pointer");
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  DeviceCtx* c = context(&code);
  if (!c) return code;
  FwnHandle* h = static_cast<FwnHandle*>(handle);
  if ((code = fwn_upload(h)) != WN_OK) return code;
  cudaError_t e;
  if ((e = c->q.ensure(sizeof(double) * 3 * nq)) != cudaSuccess ||
      (e = c->w.ensure(sizeof(double) * nq)) != cudaSuccess ||
      (e = c->scratch.ensure(aabb_sort_bytes(nq) + 256)) != cudaSuccess)
    return cuda_fail(e, "device allocation");
  if ((e = cudaMemcpyAsync(c->q.ptr, q, sizeof(double) * 3 * nq, cudaMemcpyHostToDevice,
                           c->stream)) != cudaSuccess)
    return cuda_fail(e, "copy of the queries");
  if ((e = fwn_run(h, static_cast<const double*>(c->q.ptr), nq, beta,
                   static_cast<double*>(c->w.ptr), c->scratch.ptr, c->err, c->stream)) !=
      cudaSuccess)
    return cuda_fail(e, "fast winding-number launch");
  if ((e = cudaMemcpyAsync(w, c->w.ptr, sizeof(double) * nq, cudaMemcpyDeviceToHost,
                           c->stream)) != cudaSuccess)
    return cuda_fail(e, "copy of the result");
  return collect_device_error(c, c->stream);
}

// ---- per-vertex normals ----------------------------------------------------
namespace {

struct NormalsHandle {
  NormalsTopology t;
  int device = -1;
};

void normals_release(NormalsHandle* h) {
  cudaFree(h->t.F);
  cudaFree(h->t.indptr);
  cudaFree(h->t.entries);
  cudaFree(h->t.order);
  cudaFree(h->t.contrib);
  h->t = NormalsTopology{};
}

int check_weighting(int weighting) {
  if (weighting < 0 || weighting > 3)
    return fail(WN_EINVAL, "weighting must be 0 (uniform), 1 (area), 2 (angle) or 3 (default)");
  return WN_OK;
}

int normals_check_sizes(const int64_t* F, int64_t nf, int64_t nv) {
  if (nf < 0 || nv < 0) return fail(WN_EINVAL, "negative size");
  if (nv > 0x7fffffffLL || 3 * nf > 0x7fffffffLL)
    return fail(WN_EINVAL, "more than 2^31-1 vertices or incidences");
  if (nf > 0 && !F) return fail(WN_EINVAL, "null pointer");
  return WN_OK;
}

// Own device arrays of a handle's topology.
int normals_alloc(NormalsHandle* h, int64_t nf, int64_t nv) {
  h->t.nf = nf;
  h->t.nv = nv;
  cudaGetDevice(&h->device);
  cudaError_t e;
  if ((e = dev_malloc(&h->t.F, sizeof(int32_t) * (3 * nf + 1))) != cudaSuccess ||
      (e = dev_malloc(&h->t.indptr, sizeof(int32_t) * (nv + 1))) != cudaSuccess ||
      (e = dev_malloc(&h->t.entries, sizeof(int32_t) * (3 * nf + 1))) != cudaSuccess ||
      (e = dev_malloc(&h->t.order, sizeof(int32_t) * (nv + 1))) != cudaSuccess) {
    normals_release(h);
    return cuda_fail(e, "device allocation");
  }
  return WN_OK;
}

// Uploads F (host, nf x 3 int64), checks and converts it on the device and
// builds the incidence lists into h->t's arrays on `st`; returns after `st`
// drains (caller holds g_mutex and a context).
int normals_prepare(const int64_t* F, int64_t nf, cudaStream_t st, NormalsHandle* h) {
  cudaError_t e = cudaSuccess;
  const size_t f64_bytes = ((sizeof(int64_t) * 3 * nf + 255) / 256) * 256;
  const size_t sb = f64_bytes + 256 + normals_scratch_bytes(nf, h->t.nv);
  unsigned char* scratch = nullptr;
  if ((e = dev_malloc_async(reinterpret_cast<void**>(&scratch), sb, st)) != cudaSuccess)
    return cuda_fail(e, "device allocation");
  int64_t* F64 = reinterpret_cast<int64_t*>(scratch);
  int* bad = reinterpret_cast<int*>(scratch + f64_bytes);
  if (nf > 0)
    e = cudaMemcpyAsync(F64, F, sizeof(int64_t) * 3 * nf, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = normals_build(h->t, F64, bad, scratch + f64_bytes + 256, normals_scratch_bytes(nf, h->t.nv),
                      st);
  int bad_h = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&bad_h, bad, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(scratch, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "incidence list build");
  if (bad_h != 0) return fail(WN_EINVAL, "%d face indices outside V", bad_h);
  return WN_OK;
}

// Grows the per-face contribution buffer for `mode` (uniform/area: 3 doubles
// per face, angle: 9).
int normals_contrib(NormalsHandle* h, int mode) {
  const int64_t need = normals_contrib_doubles(h->t.nf, mode);
  if (need <= h->t.contrib_doubles) return WN_OK;
  cudaFree(h->t.contrib);
  h->t.contrib = nullptr;
  h->t.contrib_doubles = 0;
  const cudaError_t e = dev_malloc(&h->t.contrib, sizeof(double) * (need > 0 ? need : 1));
  if (e != cudaSuccess) return cuda_fail(e, "device allocation");
  h->t.contrib_doubles = need;
  return WN_OK;
}

}  // namespace

int wn_normals_create(const int64_t* F, int64_t nf, int64_t nv, void* stream, void** out) {
  WN_NVTX_RANGE();
  if (!out) return fail(WN_EINVAL, "null output handle");
  *out = nullptr;
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  if (!context(&code)) return code;
  if ((code = normals_check_sizes(F, nf, nv)) != WN_OK) return code;
  NormalsHandle* h = new NormalsHandle();
  if ((code = normals_alloc(h, nf, nv)) != WN_OK ||
      (code = normals_prepare(F, nf, static_cast<cudaStream_t>(stream), h)) != WN_OK) {
    normals_release(h);
    delete h;
    return code;
  }
  *out = h;
  return WN_OK;
}

int wn_normals_destroy(void* handle) {
  if (!handle) return WN_OK;
  NormalsHandle* h = static_cast<NormalsHandle*>(handle);
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(h->device);
  cudaDeviceSynchronize();
  normals_release(h);
  cudaSetDevice(prev);
  delete h;
  return WN_OK;
}

int wn_vertex_normals_device(void* handle, const double* V, int weighting, double* N,
                             void* stream) {
  WN_NVTX_RANGE();
  if (!handle) return fail(WN_EINVAL, "null handle");
  if (int code = check_weighting(weighting)) return code;
  NormalsHandle* h = static_cast<NormalsHandle*>(handle);
  if (h->t.nv == 0) return WN_OK;
  if (!V || !N) return fail(WN_EINVAL, "null pointer");
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  if (!context(&code)) return code;
  if ((code = check_device(h->device, "normals topology")) != WN_OK) return code;
  const int mode = weighting == 3 ? 1 : weighting;
  if ((code = normals_contrib(h, mode)) != WN_OK) return code;
  const cudaError_t e = normals_eval(h->t, V, mode, N, static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? WN_OK : cuda_fail(e, "vertex-normal launch");
}

int wn_vertex_normals_host(const double* V, int64_t nv, const int64_t* F, int64_t nf,
                           int weighting, double* N) {
  WN_NVTX_RANGE();
  if (int code = check_weighting(weighting)) return code;
  if (nv < 0 || nf < 0) return fail(WN_EINVAL, "negative size");
  if (nv == 0) return WN_OK;
  if (!V || !N) return fail(WN_EINVAL, "null pointer");
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  DeviceCtx* c = context(&code);
  if (!c) return code;
  if ((code = normals_check_sizes(F, nf, nv)) != WN_OK) return code;
  // The context's grow-only buffers hold the topology: no allocation per call
  // once they are large enough.
  const int mode = weighting == 3 ? 1 : weighting;
  const int64_t ncontrib = normals_contrib_doubles(nf, mode);
  cudaError_t e;
  if ((e = c->nrm_f.ensure(sizeof(int32_t) * (3 * nf + 1))) != cudaSuccess ||
      (e = c->nrm_indptr.ensure(sizeof(int32_t) * (nv + 1))) != cudaSuccess ||
      (e = c->nrm_entries.ensure(sizeof(int32_t) * (3 * nf + 1))) != cudaSuccess ||
      (e = c->nrm_order.ensure(sizeof(int32_t) * (nv + 1))) != cudaSuccess ||
      (e = c->nrm_contrib.ensure(sizeof(double) * (ncontrib + 1))) != cudaSuccess ||
      (e = c->q.ensure(sizeof(double) * 3 * nv)) != cudaSuccess ||
      (e = c->w.ensure(sizeof(double) * 3 * nv)) != cudaSuccess)
    return cuda_fail(e, "device allocation");
  NormalsHandle h;
  h.t.F = static_cast<int32_t*>(c->nrm_f.ptr);
  h.t.indptr = static_cast<int32_t*>(c->nrm_indptr.ptr);
  h.t.entries = static_cast<int32_t*>(c->nrm_entries.ptr);
  h.t.order = static_cast<int32_t*>(c->nrm_order.ptr);
  h.t.contrib = static_cast<double*>(c->nrm_contrib.ptr);
  h.t.contrib_doubles = ncontrib;
  h.t.nf = nf;
  h.t.nv = nv;
  if ((code = normals_prepare(F, nf, c->stream, &h)) != WN_OK) return code;
  if ((e = cudaMemcpyAsync(c->q.ptr, V, sizeof(double) * 3 * nv, cudaMemcpyHostToDevice,
                           c->stream)) != cudaSuccess ||
      (e = normals_eval(h.t, static_cast<const double*>(c->q.ptr), mode,
                        static_cast<double*>(c->w.ptr), c->stream)) != cudaSuccess ||
      (e = cudaMemcpyAsync(N, c->w.ptr, sizeof(double) * 3 * nv, cudaMemcpyDeviceToHost,
                           c->stream)) != cudaSuccess) {
    cudaStreamSynchronize(c->stream);
    return cuda_fail(e, "vertex normals");
  }
  return collect_device_error(c, c->stream);
}

// The closest-point walk and the fast winding-number walk read only the points
// and are both latency bound at low occupancy, so they run side by side: the
// points are Morton-sorted once on the caller's stream, the closest-point
// kernel follows there and the winding-number kernel runs on the context's
// second stream (fork/join by events), then the sign is taken on the caller's
// stream. Same results as running the two entry points one after the other.
int wn_signed_distance_fast_device(void* tree, void* fast, double beta, const double* P,
                                   int64_t np, double* s, int64_t* index, double* closest,
                                   double* w, void* stream) {
  WN_NVTX_RANGE();
  if (int code = check_points(tree, np)) return code;
  if (!fast) return fail(WN_EINVAL, "null fast winding-number handle");
  if (int code = check_beta(beta)) return code;
  if (np == 0) return WN_OK;
  if (!P || !s || !index || !closest || !w) return fail(WN_EINVAL, "null pointer");
  std::lock_guard<std::mutex> lock(g_mutex);
  int code = WN_OK;
  DeviceCtx* c = context(&code);
  if (!c) return code;
  const AabbHandle* ah = static_cast<const AabbHandle*>(tree);
  if ((code = check_device(ah->device, "tree")) != WN_OK) return code;
  FwnHandle* fh = static_cast<FwnHandle*>(fast);
  if ((code = fwn_upload(fh)) != WN_OK) return code;
  cudaError_t e = cudaSuccess;
  if ((!c->side && (e = cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking)) !=
                       cudaSuccess) ||
      (!c->fork && (e = cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming)) !=
                       cudaSuccess) ||
      (!c->join && (e = cudaEventCreateWithFlags(&c->join, cudaEventDisableTiming)) !=
                       cudaSuccess))
    return cuda_fail(e, "second stream set-up");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t sb = aabb_sort_bytes(np);
  void* scratch = nullptr;
  if (sb && (e = dev_malloc_async(&scratch, sb, st)) != cudaSuccess)
    return cuda_fail(e, "device allocation");
  uint32_t* perm = nullptr;
  if (np >= kAabbSortMin) {
    perm = static_cast<uint32_t*>(scratch);
    unsigned char* rest = static_cast<unsigned char*>(scratch) + align256(sizeof(uint32_t) * np);
    e = mixed_sort_queries(P, np, perm, rest, mixed_sort_scratch_bytes(np), st);
  }
  bool forked = false;
  if (e == cudaSuccess && (e = cudaEventRecord(c->fork, st)) == cudaSuccess &&
      (e = cudaStreamWaitEvent(c->side, c->fork, 0)) == cudaSuccess) {
    forked = true;
    e = aabb_query(ah->t, P, np, perm, s, index, closest, c->err, st);
    const cudaError_t e2 = fwn_eval_device(fh->dev, P, np, perm, beta, w, c->err, c->side);
    if (e == cudaSuccess) e = e2;
  }
  // Join whatever was forked before anything else touches the scratch.
  if (forked) {
    const cudaError_t ej = cudaEventRecord(c->join, c->side) == cudaSuccess
                               ? cudaStreamWaitEvent(st, c->join, 0)
                               : cudaStreamSynchronize(c->side);
    if (e == cudaSuccess) e = ej;
  }
  if (e == cudaSuccess) e = signed_from_winding(w, s, np, st);
  if (scratch) cudaFreeAsync(scratch, st);
  return e == cudaSuccess ? WN_OK : cuda_fail(e, "signed-distance launch");
}

// src/capi.mojo:945-947: 1 on success, 0 on failure (the shim raises). Large
// problems go through the prepared-mesh FP64 kernel (its ~2 ms preparation is
// repaid above ~1e9 pairs), small ones through the streaming FP64 kernel; both
// give pair terms bit-identical to the reference.
int64_t mli_winding_gpu(int64_t tri, int64_t q, int64_t dst, int64_t nf, int64_t nq) {
  WN_NVTX_RANGE();
  const bool large = nf >= 4096 && static_cast<double>(nf) * static_cast<double>(nq) >= 1e9 &&
                     nf <= 0x7fffffffLL;
  return forward_fp64_host(reinterpret_cast<const double*>(tri),
                           reinterpret_cast<const double*>(q), reinterpret_cast<double*>(dst), nf,
                           nq, large ? kFp64Tiled : kFp64ArgProd) == WN_OK
             ? 1
             : 0;
}

// Out-of-scope reference exports (src/capi.mojo:923-932, 962-1007).
void mli_cot_entries(int64_t, int64_t, int64_t, int64_t, int64_t) {
  out_of_scope("mli_cot_entries");
}
void mli_mass_contributions(int64_t, int64_t, int64_t, int64_t, int64_t, int64_t) {
  out_of_scope("mli_mass_contributions");
}
void mli_heat_vector_divergence(int64_t, int64_t, int64_t, int64_t, int64_t, int64_t) {
  out_of_scope("mli_heat_vector_divergence");
}
void mli_heat_precompute(int64_t, int64_t, int64_t, int64_t) {
  out_of_scope("mli_heat_precompute");
}
void mli_arap_covariance(int64_t, int64_t, int64_t, int64_t, int64_t, int64_t, int64_t,
                         int64_t) {
  out_of_scope("mli_arap_covariance");
}
void mli_arap_rhs(int64_t, int64_t, int64_t, int64_t, int64_t, int64_t, int64_t, int64_t) {
  out_of_scope("mli_arap_rhs");
}
void mli_arap_covariance_rims(int64_t, int64_t, int64_t, int64_t, int64_t, int64_t, int64_t,
                              int64_t) {
  out_of_scope("mli_arap_covariance_rims");
}
void mli_arap_rhs_rims(int64_t, int64_t, int64_t, int64_t, int64_t, int64_t, int64_t, int64_t) {
  out_of_scope("mli_arap_rhs_rims");
}
void mli_arap_rotations(int64_t, int64_t, int64_t, int64_t, int64_t, int64_t) {
  out_of_scope("mli_arap_rotations");
}

}  // extern "C"
