// wn_forward_fp64_device_noalloc: the plain FP64 forward for callers that
// must not allocate GPU memory.
//
// Who needs it: host applications and plugins that own every byte of device
// memory through their own pool or a fixed budget (a renderer, a simulation
// or game engine, an embedded/real-time service), and that forbid a library
// from calling cudaMalloc/cudaMallocAsync behind their back, because such a
// call can fail at an arbitrary moment, fragment their pool or exceed the
// budget they planned for. wn_forward_fp64_device draws its face-split
// scratch from the stream-ordered allocator; this entry point draws it from a
// fixed array compiled into the library instead.
//
// The scratch array is g_noalloc_partial below: kNoAllocScratchDoubles
// doubles (4 MiB), resident on every GPU that loads this library until the
// process exits. It holds the per-split partial angle sums of a face-split
// launch, nsplit x nq doubles. The entry point accepts at most
// kNoAllocMaxQueries queries and caps the number of face splits so that
// nsplit * nq fits the array (noalloc_plan); larger query counts are rejected
// with WN_EINVAL.
//
// Host code must not pass the array's name to a kernel: in host code the name
// denotes a host-side stand-in, not a device address. On the first call on each
// device (with that device current) the entry point asks the runtime for the
// array's device address with cudaGetSymbolAddress, checks the result, and
// caches it per device; that first call on a device should come before any
// stream capture. Later calls reuse the cached address. The stream must belong
// to the current device: the address is looked up for the current device, so a
// stream of another device is refused with WN_EINVAL.
//
// Every call shares the one array and the one error word, and the array keeps
// the last call's contents. Each call overwrites every partial sum it later
// reads (one CTA writes each (split, query) entry before the summing kernel
// reads it) and clears the error word, so nothing stale is read. Within one
// process calls do not overlap: each holds a mutex until its stream has
// finished the work. That guarantee rests on those two alone; calls that did
// overlap on the GPU would race on the array and give wrong results.
//
// The call is ordered on the caller's stream and returns after that stream has
// finished the work, so that a kernel-reported error (a bounded wait that ran
// out) can be returned. Waiting for a stream that is being captured would end
// the caller's capture with an error, so such a stream is refused up front
// (WN_EINVAL) and left untouched. The call makes no cudaMalloc, cudaFree or
// any allocating library routine.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <mutex>

#include "../../include/wn_b200.h"
#include "wn_internal.h"

namespace wn {
namespace {

constexpr int64_t kNoAllocMaxQueries = kNoAllocScratchDoubles;
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_partial[kNoAllocScratchDoubles];
static __device__ __align__(256) int g_noalloc_err;

struct NoAllocDevice {
  bool ready = false;
  int sms = 0;
  double* partial = nullptr;  // device address of g_noalloc_partial
  int* err = nullptr;         // device address of g_noalloc_err
};

std::mutex g_noalloc_mutex;
NoAllocDevice g_noalloc_dev[kNoAllocMaxDevices];

// Failure: the message goes to wn_last_error() of the calling thread.
int noalloc_fail(int code, const char* msg, cudaError_t e = cudaSuccess) {
  char buf[320];
  if (e != cudaSuccess)
    std::snprintf(buf, sizeof(buf), "%s: %s", msg, cudaGetErrorString(e));
  else
    std::snprintf(buf, sizeof(buf), "%s", msg);
  record_error(buf);
  return code;
}

}  // namespace

Fp64Plan noalloc_plan(int64_t nf, int64_t nq, int sms) {
  // wn_forward_fp64_device's plan, with the face splits capped so that the
  // nsplit * nq partial sums fit the fixed array.
  Fp64Plan plan = plan_fp64(nf, nq, sms);
  const int64_t max_split = kNoAllocScratchDoubles / std::max<int64_t>(nq, 1);
  if (plan.nsplit > max_split) plan = plan_fp64(nf, nq, sms, static_cast<int>(max_split));
  return plan;
}

}  // namespace wn

using namespace wn;

extern "C" {

int wn_forward_fp64_device_noalloc(const double* tri, int64_t ld, const double* q, double* w,
                                   int64_t nf, int64_t nq, int mode, void* stream) {
  WN_NVTX_RANGE();
  if (nf < 0 || nq < 0 || (ld & 1) || ld < nf)
    return noalloc_fail(WN_EINVAL, "bad sizes: need nf >= 0, nq >= 0, ld even and ld >= nf");
  if (nq > kNoAllocMaxQueries)
    return noalloc_fail(WN_EINVAL,
                        "nq exceeds the no-allocation limit of 524288 queries "
                        "(use wn_forward_fp64_device)");
  if (reinterpret_cast<uintptr_t>(tri) & 15)
    return noalloc_fail(WN_EINVAL, "tri must be 16-byte aligned");
  if (mode != kFp64ArgProd && mode != kFp64Direct) return noalloc_fail(WN_EINVAL, "bad mode");
  if (nq == 0) return WN_OK;

  // The capture state is asked first, before any other runtime call touches the
  // stream: a refused call must leave the caller's capture intact.
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  cudaError_t e = cudaStreamIsCapturing(st, &capture);
  if (e != cudaSuccess)
    return noalloc_fail(WN_EINVAL, "cudaStreamIsCapturing on the given stream", e);
  if (capture != cudaStreamCaptureStatusNone)
    return noalloc_fail(WN_EINVAL,
                        "the stream is being captured: this call waits for its stream before "
                        "it returns, which would end the capture");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  int dev = 0;
  e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices)
    return noalloc_fail(WN_ENODEV, "no usable CUDA device", e);
  int stream_dev = dev;
  if ((e = cudaStreamGetDevice(st, &stream_dev)) != cudaSuccess)
    return noalloc_fail(WN_EINVAL, "cudaStreamGetDevice on the given stream", e);
  if (stream_dev != dev)
    return noalloc_fail(WN_EINVAL,
                        "the stream belongs to another device than the current one: make the "
                        "stream's device current before the call");
  NoAllocDevice& d = g_noalloc_dev[dev];
  if (!d.ready) {
    // Once per device, with that device current: device addresses of the
    // file-scope arrays (their host-side names are not device addresses).
    if ((e = cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev)) !=
        cudaSuccess)
      return noalloc_fail(WN_ECUDA, "cudaDeviceGetAttribute", e);
    if ((e = cudaGetSymbolAddress(reinterpret_cast<void**>(&d.partial), g_noalloc_partial)) !=
        cudaSuccess)
      return noalloc_fail(WN_ECUDA, "cudaGetSymbolAddress(g_noalloc_partial)", e);
    if ((e = cudaGetSymbolAddress(reinterpret_cast<void**>(&d.err), g_noalloc_err)) !=
        cudaSuccess)
      return noalloc_fail(WN_ECUDA, "cudaGetSymbolAddress(g_noalloc_err)", e);
    d.ready = true;
  }

  const Fp64Plan plan = noalloc_plan(nf, nq, d.sms);
  if (plan.scratch_doubles > kNoAllocScratchDoubles)
    return noalloc_fail(WN_EINVAL, "face split does not fit the fixed scratch array");

  if ((e = cudaMemsetAsync(d.err, 0, sizeof(int), st)) != cudaSuccess)
    return noalloc_fail(WN_ECUDA, "clearing the error word", e);
  if ((e = launch_fp64(plan, mode, tri, ld, nf, q, nq, w, d.partial, d.err, st)) != cudaSuccess)
    return noalloc_fail(WN_ECUDA, "FP64 winding-number launch", e);
  int herr = 0;
  if ((e = cudaMemcpyAsync(&herr, d.err, sizeof(int), cudaMemcpyDeviceToHost, st)) !=
          cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess)
    return noalloc_fail(WN_ECUDA, "kernel execution", e);
  if (herr != 0) return noalloc_fail(WN_EDEVICE, "a kernel reported a bounded-wait timeout");
  return WN_OK;
}

}  // extern "C"
