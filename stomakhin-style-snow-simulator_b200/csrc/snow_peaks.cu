// Measured arithmetic peaks of the GPU the library runs on: FP64 and FP32
// fused multiply-add throughput, the compute roofs beside HBM bandwidth that
// the particle kernels are judged against (they do 3x3 algebra and stencil
// sums in double or float, never a dense contraction).
//
// Each thread runs kChains independent FMA chains (a <- a * b + c) for `iters`
// iterations: enough independent work per warp to cover the pipe latency at
// full occupancy, so the pipe, not the scheduler, sets the rate.  The result is
// written only when it equals a value it never takes, so the compiler keeps
// every FMA and the kernel stores nothing (the store would go to a small
// file-scope device array, never to a caller's pointer).  Timed with CUDA events on the
// caller's stream at the clocks the GPU runs (no clock or power setting is
// touched).
#include <cuda_runtime.h>

#include <string>

#include "snow_engine.hpp"
#include "snow_gpu.h"

namespace snow {
namespace {

constexpr int kChains = 8;
constexpr int kThreads = 256;

__device__ double g_sink_d[kThreads];
__device__ float g_sink_f[kThreads];
__device__ __forceinline__ void sink(double v) { g_sink_d[threadIdx.x] = v; }
__device__ __forceinline__ void sink(float v) { g_sink_f[threadIdx.x] = v; }

template <typename T>
__global__ void __launch_bounds__(kThreads) k_fma_scalar(int iters, T b, T c) {
  T a[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) a[k] = (T)(threadIdx.x + k) * (T)1e-3;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = fma(a[k], b, c);
  }
  T s = 0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += a[k];
  if (s == (T)-12345.678) sink(s);
}

// Packed two-wide float FMA (__ffma2_rn: two fmaf per instruction).
__global__ void __launch_bounds__(kThreads) k_fma_packed(int iters, float b, float c) {
  float2 a[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) a[k] = make_float2((threadIdx.x + k) * 1e-3f, (threadIdx.x - k) * 1e-3f);
  const float2 b2 = make_float2(b, b), c2 = make_float2(c, c);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = __ffma2_rn(a[k], b2, c2);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += a[k].x + a[k].y;
  if (s == -12345.678f) sink(s);
}

}  // namespace
}  // namespace snow

using namespace snow;

extern "C" int snow_gpu_measure_fma_peak(int kind, double* flops_per_s, double* ms_out, void* stream) {
  try {
    if (kind < SNOW_PEAK_FP64 || kind > SNOW_PEAK_FP32X2 || !flops_per_s)
      throw Error(SNOW_E_ARG, "snow_gpu_measure_fma_peak: bad kind or output pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int dev = 0, sms = 0, per_sm = 0;
    check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
    if (kind == SNOW_PEAK_FP64)
      check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fma_scalar<double>, kThreads, 0),
                 "occupancy");
    else if (kind == SNOW_PEAK_FP32)
      check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fma_scalar<float>, kThreads, 0),
                 "occupancy");
    else
      check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fma_packed, kThreads, 0), "occupancy");
    const int blocks = sms * (per_sm > 0 ? per_sm : 1);
    cudaEvent_t e0, e1;
    check_cuda(cudaEventCreate(&e0), "event");
    check_cuda(cudaEventCreate(&e1), "event");
    auto launch = [&](int iters) {
      if (kind == SNOW_PEAK_FP64)
        k_fma_scalar<double><<<blocks, kThreads, 0, s>>>(iters, 0.999999, 1e-7);
      else if (kind == SNOW_PEAK_FP32)
        k_fma_scalar<float><<<blocks, kThreads, 0, s>>>(iters, 0.999999f, 1e-7f);
      else
        k_fma_packed<<<blocks, kThreads, 0, s>>>(iters, 0.999999f, 1e-7f);
    };
    launch(1024);  // warm-up (module load, clocks up)
    int iters = 1 << 14;
    float ms = 0.f;
    // grow the run until it lasts at least 20 ms
    for (int tries = 0; tries < 8; ++tries) {
      check_cuda(cudaEventRecord(e0, s), "event");
      launch(iters);
      check_cuda(cudaEventRecord(e1, s), "event");
      check_cuda(cudaEventSynchronize(e1), "fma peak run");
      check_cuda(cudaEventElapsedTime(&ms, e0, e1), "event time");
      if (ms >= 20.f || iters >= (1 << 22)) break;
      iters *= 4;
    }
    check_cuda(cudaGetLastError(), "fma peak launch");
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const double fma_per_thread = (double)iters * kChains * (kind == SNOW_PEAK_FP32X2 ? 2 : 1);
    *flops_per_s = 2.0 * fma_per_thread * blocks * kThreads / (ms * 1e-3);
    if (ms_out) *ms_out = ms;
    return SNOW_OK;
  } catch (const Error& e) {
    return set_error(e.code, e.what());
  } catch (const std::exception& e) {
    return set_error(SNOW_E_ARG, e.what());
  }
}
