// Internal (non-exported) interfaces between the kernel files and the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <atomic>
#include <cstdint>

namespace wn {

// Stores `message` as the calling thread's wn_last_error().
void record_error(const char* message);

// An NVTX range named after a C-ABI entry point, so a profiler's timeline (and
// `ncu --nvtx --nvtx-include`) shows which call launched what. Without a tool
// attached it costs a branch.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};
#define WN_NVTX_RANGE() const ::wn::NvtxRange wn_nvtx_range_(__func__)

// Kernels launched by this library since load (wn_launch_count()).
extern std::atomic<int64_t> g_launches;

// Every device allocation of the library goes through these two. They behave
// as cudaMalloc / cudaMallocAsync, except that an allocation fault armed by
// wn_inject_fault (or WN_INJECT_FAULT=alloc:N in the environment) makes the
// chosen allocation report cudaErrorMemoryAllocation without allocating, so
// the tests can walk every out-of-memory path on a real device.
cudaError_t dev_malloc(void** p, size_t bytes);
cudaError_t dev_malloc_async(void** p, size_t bytes, cudaStream_t stream);
template <class T>
cudaError_t dev_malloc(T** p, size_t bytes) {
  return dev_malloc(reinterpret_cast<void**>(p), bytes);
}
template <class T>
cudaError_t dev_malloc_async(T** p, size_t bytes, cudaStream_t stream) {
  return dev_malloc_async(reinterpret_cast<void**>(p), bytes, stream);
}

// Failure-path self-test (wn_probe.cu): one CTA waits on an mbarrier phase that no
// copy will complete, with a `polls` limit; the wait runs out, the kernel sets the
// timeout bit of `err` and returns.
cudaError_t launch_wait_selftest(uint32_t polls, int* err, cudaStream_t stream);

// FMA-pipe peak probe (wn_probe.cu): TFLOP/s for bits = 64 or 32.
cudaError_t probe_fma_tflops(int bits, int sms, cudaStream_t stream, double* tflops);

// ---- plain FP64 forward (wn_fp64.cu) ---------------------------------------
enum Fp64Mode : int {
  kFp64ArgProd = 0,  // bit-exact pair terms, argument-of-product accumulation
  kFp64Direct = 1,   // bit-exact pair terms, one atan2 per pair
  kFp64Tiled = 2,    // kFp64ArgProd over a prepared mesh, repeated corners reused
};

struct Fp64Plan {
  int threads = 128;      // threads per CTA
  int qpt = 2;            // queries held per thread
  int tile_faces = 128;   // faces per shared-memory tile
  int stages = 3;         // bulk-copy ring depth
  int64_t nsplit = 1;     // face-range splits (grid.y)
  int64_t f_chunk = 0;    // faces per split (multiple of tile_faces)
  int64_t qblocks = 0;    // grid.x
  int64_t scratch_doubles = 0;  // nsplit * nq when nsplit > 1
};

// Chooses the launch shape for nf faces x nq queries on a device with `sms` SMs.
// force_nsplit > 0 pins the number of face splits (tests use it).
Fp64Plan plan_fp64(int64_t nf, int64_t nq, int sms, int force_nsplit = 0);

// Plan of wn_forward_fp64_device_noalloc: plan_fp64 with the face splits capped
// so that its nsplit * nq partial sums fit the fixed array of
// kNoAllocScratchDoubles doubles (4 MiB) compiled into the library.
constexpr int64_t kNoAllocScratchDoubles = int64_t(1) << 19;
Fp64Plan noalloc_plan(int64_t nf, int64_t nq, int sms);

// tri: 9 rows of `ld` doubles (row 3*corner+axis, ld even, ld >= nf), 16-byte
// aligned; q: nq x 3; w: nq outputs (W, already divided by 2*pi); scratch:
// plan.scratch_doubles doubles or null when that is 0; err: device error word.
cudaError_t launch_fp64(const Fp64Plan& plan, int mode, const double* tri, int64_t ld, int64_t nf,
                        const double* q, int64_t nq, double* w, double* scratch, int* err,
                        cudaStream_t stream);

// ---- plain FP64 over a prepared mesh, with corner reuse (wn_fp64.cu) -------
struct MixedMesh;
struct Fp64TiledPlan {
  int64_t qblocks = 1, nsplit = 1, tiles_per_split = 1, scratch_doubles = 0;
};
Fp64TiledPlan plan_fp64_tiled(int64_t ntiles, int64_t nq, int sms);
cudaError_t launch_fp64_tiled(const Fp64TiledPlan& p, const MixedMesh& m, const double* q,
                              int64_t nq, double* w, double* scratch, int* err,
                              cudaStream_t stream);

}  // namespace wn
