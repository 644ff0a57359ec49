// FP64 throughput probes: the denominators of the FP64 roofline fractions the bench reports for
// the stencil kernels (DFMA) and the dense ring-LU products (DMMA); the HBM denominator is a
// measured copy bandwidth, these are its FP64 counterparts. In the DFMA probe every thread runs
// kChains independent chains of fused multiply-adds, enough to cover the pipeline latency, on a
// grid of eight 256-thread CTAs per SM; the chains' sum goes to `sink` so that no work is
// optimised away.

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/euler_b200.h"

namespace eb {

int fail(int code, const char* msg);
int check_launch(const char* what);

namespace {

constexpr int kChains = 8;

__global__ void __launch_bounds__(256) k_fp64_fma(int64_t iterations, double a, double b,
                                                   double* sink) {
  double x[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) x[k] = threadIdx.x * 1e-9 + k;
  for (int64_t i = 0; i < iterations; ++i) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) x[k] = fma(x[k], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += x[k];
  if (s == 12345.678) sink[0] = s;  // practically never true; keeps the chains live
}

// The FP64 tensor-core counterpart (the dense kernels' denominator): kTiles independent 8 x 8
// accumulators per warp, each updated by mma.sync.m8n8k4.f64 (512 flops per warp instruction).
constexpr int kTiles = 8;

__global__ void __launch_bounds__(256) k_fp64_mma(int64_t iterations, double* sink) {
  const int lane = threadIdx.x & 31;
  const double a = 1.0 + lane * 1e-9, b = 0.999999999;
  double d[kTiles][2];
#pragma unroll
  for (int k = 0; k < kTiles; ++k) d[k][0] = d[k][1] = k * 1e-3;
  for (int64_t i = 0; i < iterations; ++i) {
#pragma unroll
    for (int k = 0; k < kTiles; ++k)
      asm volatile(
          "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
          : "+d"(d[k][0]), "+d"(d[k][1])
          : "d"(a), "d"(b));
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < kTiles; ++k) s += d[k][0] + d[k][1];
  if (s == 12345.678) sink[0] = s;  // practically never true; keeps the accumulators live
}

}  // namespace
}  // namespace eb

extern "C" int eb_fp64_mma_probe(int64_t iterations, int sms, double* sink, void* stream) {
  if (iterations < 1 || sms < 1 || !sink) return eb::fail(EB_ERR_ARG, "mma probe: bad arguments");
  eb::k_fp64_mma<<<4 * sms, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(iterations, sink);
  return eb::check_launch("mma probe");
}

extern "C" int eb_fp64_fma_probe(int64_t iterations, int sms, double* sink, void* stream) {
  if (iterations < 1 || sms < 1 || !sink) return eb::fail(EB_ERR_ARG, "fma probe: bad arguments");
  eb::k_fp64_fma<<<8 * sms, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      iterations, 0.999999999, 1e-9, sink);
  return eb::check_launch("fma probe");
}
