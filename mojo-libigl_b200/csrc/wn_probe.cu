// Issue-rate probes for the roofline denominators of this compute-bound path.
//
// The pair kernels are bound by the FP64 pipe (plain form) or the FP32 and
// MUFU pipes (mixed form), not by HBM or tensor cores, so bench.py measures
// those pipes' peaks live on the same GPU with these kernels: many independent
// FMA chains per thread, full occupancy, timed with CUDA events.
#include <cuda_runtime.h>

#include <cstdint>

#include "wn_common.cuh"
#include "wn_internal.h"

namespace wn {
namespace {

constexpr int kChains = 8;

template <typename T>
__global__ void __launch_bounds__(256) fma_probe_kernel(T a, T b, int iters, T* sink) {
  T x[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) x[c] = static_cast<T>(threadIdx.x + c);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = x[c] * a + b;  // one FMA each
  }
  T s = 0;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += x[c];
  if (s == static_cast<T>(-12345.678)) *sink = s;  // keeps the chains live
}

template <typename T>
cudaError_t run_probe(int sms, int iters, cudaStream_t stream, float* ms) {
  T* sink = nullptr;
  cudaError_t e = dev_malloc_async(reinterpret_cast<void**>(&sink), sizeof(T), stream);
  if (e != cudaSuccess) return e;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = sms * 8;
  fma_probe_kernel<T><<<blocks, 256, 0, stream>>>(static_cast<T>(0.999), static_cast<T>(0.001),
                                                  iters, sink);  // warm-up
  cudaEventRecord(e0, stream);
  fma_probe_kernel<T><<<blocks, 256, 0, stream>>>(static_cast<T>(0.999), static_cast<T>(0.001),
                                                  iters, sink);
  cudaEventRecord(e1, stream);
  e = cudaEventSynchronize(e1);
  if (e == cudaSuccess) e = cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFreeAsync(sink, stream);
  cudaStreamSynchronize(stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  return e;
}

// The mbarrier expects one arrival plus 16 transaction bytes; the thread arrives
// and announces the bytes but no copy ever delivers them, so the phase never
// completes and the bounded wait gives up after `polls` polls.
__global__ void wait_selftest_kernel(uint32_t polls, int* err) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x != 0) return;
  mbar_init(&bar, 1);
  fence_barrier_init();
  mbar_arrive_expect_tx(&bar, 16);
  for (uint32_t i = 0; i < polls; ++i)
    if (mbar_try_wait(&bar, 0)) return;  // cannot happen: nothing completes the bytes
  atomicOr(err, kErrWaitTimeout);
}

}  // namespace

cudaError_t launch_wait_selftest(uint32_t polls, int* err, cudaStream_t stream) {
  wait_selftest_kernel<<<1, 32, 0, stream>>>(polls, err);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError();
}

// FMA throughput in TFLOP/s (FMA = 2 flops) for precision 64 or 32.
cudaError_t probe_fma_tflops(int bits, int sms, cudaStream_t stream, double* tflops) {
  const int iters = bits == 64 ? 4096 : 16384;
  float ms = 0.f;
  cudaError_t e = bits == 64 ? run_probe<double>(sms, iters, stream, &ms)
                             : run_probe<float>(sms, iters, stream, &ms);
  if (e != cudaSuccess) return e;
  const double flops = 2.0 * kChains * static_cast<double>(iters) * sms * 8 * 256;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return cudaSuccess;
}

}  // namespace wn
