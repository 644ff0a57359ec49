// FP64 throughput probe: the denominator of the FP64 roofline fractions the bench reports for
// the stencil kernels (the HBM denominator is a measured copy bandwidth; this is its FP64
// counterpart). Every thread runs kChains independent chains of fused multiply-adds, enough to
// cover the pipeline latency, on a grid of eight 256-thread CTAs per SM; the chains' sum goes
// to `sink` so that no work is optimised away.

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

}  // namespace
}  // namespace eb

extern "C" int eb_fp64_fma_probe(int64_t iterations, int sms, double* sink, void* stream) {
  if (iterations < 1 || sms < 1 || !sink) return eb::fail(EB_ERR_ARG, "fma probe: bad arguments");
  eb::k_fp64_fma<<<8 * sms, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      iterations, 0.999999999, 1e-9, sink);
  return eb::check_launch("fma probe");
}
