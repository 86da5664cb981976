// sfnl_probe.cu -- throughput of B200's FP64 pipe, the denominator of the FP64 forms' roofline.
//
// The FAST kernels issue mma.sync.m8n8k4.f64 (DMMA) and FP64 FMAs (DFMA); on B200 both run on the same
// FP64 resources.  This diagnostic measures each one alone with CUDA events: every warp runs long chains
// of independent operations on register operands (no memory traffic inside the loop), the grid covers
// every SM several times, and the best of a few launches is reported.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/sfemans_nl.h"
#include "sfnl_internal.h"

namespace sfnl {
namespace {

constexpr int kChains = 8;  // independent accumulators per warp (DMMA) or per thread (DFMA)

__global__ void __launch_bounds__(256) dmma_loop(int iters, double *sink) {
  double acc[kChains][2];
  const double a = 1.0 + 1e-9 * threadIdx.x, b = 1.0 - 1e-9 * threadIdx.x;
#pragma unroll
  for (int c = 0; c < kChains; ++c) acc[c][0] = acc[c][1] = 0.0;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c)
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                   : "+d"(acc[c][0]), "+d"(acc[c][1])
                   : "d"(a), "d"(b));
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += acc[c][0] + acc[c][1];
  if (s == 12345.678) sink[0] = s;  // keeps the chains live
}

__global__ void __launch_bounds__(256) dfma_loop(int iters, double *sink) {
  double acc[kChains];
  const double a = 1.0 + 1e-9 * threadIdx.x, b = 1.0 - 1e-9 * threadIdx.x;
#pragma unroll
  for (int c = 0; c < kChains; ++c) acc[c] = 0.5 * c;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) acc[c] = fma(acc[c], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += acc[c];
  if (s == 12345.678) sink[0] = s;
}

// Best CUDA-event time of `reps` launches (milliseconds).
template <typename K>
int best_ms(K kern, int blocks, int iters, double *sink, int reps, float *out) {
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
    return set_error(SFNL_ERR_CUDA, "cudaEventCreate failed");
  float best = 1e30f;
  int rc = SFNL_OK;
  for (int r = 0; r < reps && rc == SFNL_OK; ++r) {
    cudaEventRecord(e0);
    kern<<<blocks, 256>>>(iters, sink);
    cudaEventRecord(e1);
    if (cudaEventSynchronize(e1) != cudaSuccess) {
      rc = check_launch("FP64 throughput probe");
      if (!rc) rc = set_error(SFNL_ERR_CUDA, "FP64 throughput probe failed");
      break;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r > 0 && ms < best) best = ms;  // the first launch is a warm-up
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *out = best;
  return rc;
}

}  // namespace
}  // namespace sfnl

using namespace sfnl;

extern "C" int sfnl_probe_fp64_tflops(double *dmma_tflops, double *dfma_tflops) {
  if (!dmma_tflops || !dfma_tflops) return set_error(SFNL_ERR_ARG, "null pointer");
  double *sink = nullptr;
  if (cudaMalloc(&sink, sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    return set_error(SFNL_ERR_ALLOC, "cudaMalloc failed");
  }
  const int blocks = num_sms() * 8, iters = 4096, reps = 6;
  const double warps = (double)blocks * 8.0;
  float ms = 0.f;
  int rc = best_ms(dmma_loop, blocks, iters, sink, reps, &ms);
  if (!rc) *dmma_tflops = warps * iters * kChains * 512.0 / (ms * 1e-3) / 1e12;  // 8x8x4 FMAs per DMMA
  if (!rc) rc = best_ms(dfma_loop, blocks, iters * 4, sink, reps, &ms);
  if (!rc) *dfma_tflops = warps * 32.0 * iters * 4 * kChains * 2.0 / (ms * 1e-3) / 1e12;
  cudaFree(sink);
  return rc;
}
