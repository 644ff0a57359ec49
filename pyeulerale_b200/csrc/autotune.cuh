// Launch-variant autotuner of the stencil kernels.
//
// A kernel with several launch variants that compute identical results (different tile shapes,
// dual widths or occupancy targets) calls launch_tuned. The first call for a problem key (the
// device, the kernel, and the problem's sizes) runs every variant twice on the caller's stream,
// a warm-up and a run timed with CUDA events, and keeps the fastest; later calls launch the kept
// variant directly. A call made while the stream is being captured into a CUDA graph, or with
// the environment variable EB_AUTOTUNE=0, launches the default variant without timing (and
// caches nothing); EB_AUTOTUNE=v<k> launches variant k. The choices and their times are listed
// by eb_autotune_report.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <string>

namespace eb {
namespace tune {

// Launches variant `v` (0 .. n_variants - 1) and returns its EB_* status.
using Launch = std::function<int(int v)>;

int launch_tuned(const char* kernel, int64_t key_a, int64_t key_b, int n_variants,
                 int default_variant, const char* const* names, cudaStream_t st,
                 const Launch& launch);

}  // namespace tune
}  // namespace eb
