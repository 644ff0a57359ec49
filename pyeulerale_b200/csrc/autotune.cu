// Launch-variant autotuner (autotune.cuh) and its report entry point.

#include "autotune.cuh"

#include <cstdio>
#include <algorithm>
#include <cstdlib>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "../../include/euler_b200.h"

namespace eb {

int fail(int code, const char* msg);
int check_launch(const char* what);

namespace tune {
namespace {

struct Entry {
  int choice = 0;
  std::vector<float> ms;
  std::vector<std::string> names;
};

using Key = std::tuple<int, std::string, int64_t, int64_t>;

std::mutex g_mutex;
std::map<Key, Entry> g_table;

// EB_AUTOTUNE: unset or "1" tune; "0" the default variant; "v<k>" variant k (checks that the
// variants agree). Returns the variant to launch untimed, or -1 to tune.
int fixed_variant(int n_variants, int default_variant) {
  const char* v = std::getenv("EB_AUTOTUNE");
  if (!v) return -1;
  if (v[0] == '0') return default_variant;
  if (v[0] == 'v') return std::min(std::max(std::atoi(v + 1), 0), n_variants - 1);
  return -1;
}

}  // namespace

int launch_tuned(const char* kernel, int64_t key_a, int64_t key_b, int n_variants,
                 int default_variant, const char* const* names, cudaStream_t st,
                 const Launch& launch) {
  const int fixed = fixed_variant(n_variants, default_variant);
  if (fixed >= 0) return launch(fixed);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (n_variants < 2 || cudaStreamIsCapturing(st, &cap) != cudaSuccess ||
      cap != cudaStreamCaptureStatusNone) {
    cudaGetLastError();
    return launch(default_variant);
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return check_launch("autotune device");
  const Key key{dev, kernel, key_a, key_b};
  {
    std::lock_guard<std::mutex> lock(g_mutex);
    auto it = g_table.find(key);
    if (it != g_table.end()) return launch(it->second.choice);
  }
  Entry e;
  cudaEvent_t a = nullptr, b = nullptr;
  if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
    if (a) cudaEventDestroy(a);
    return check_launch("autotune events");
  }
  int rc = EB_OK;
  float best = 0.0f;
  for (int v = 0; v < n_variants && rc == EB_OK; ++v) {
    rc = launch(v);  // warm-up (first launch of the variant)
    if (rc != EB_OK) break;
    cudaEventRecord(a, st);
    rc = launch(v);
    cudaEventRecord(b, st);
    if (rc != EB_OK || cudaEventSynchronize(b) != cudaSuccess) {
      rc = rc != EB_OK ? rc : check_launch("autotune timing");
      break;
    }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a, b);
    e.ms.push_back(ms);
    e.names.push_back(names ? names[v] : std::to_string(v));
    if (v == 0 || ms < best) {
      best = ms;
      e.choice = v;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (rc != EB_OK) return rc;
  {
    std::lock_guard<std::mutex> lock(g_mutex);
    g_table[key] = e;
  }
  return launch(e.choice);  // the result of the kept variant, as every later call
}

}  // namespace tune
}  // namespace eb

extern "C" int eb_autotune_report(char* buf, int len) {
  using namespace eb::tune;
  std::string s;
  {
    std::lock_guard<std::mutex> lock(g_mutex);
    for (const auto& kv : g_table) {
      char line[160];
      std::snprintf(line, sizeof line, "device %d %s (%lld, %lld): ", std::get<0>(kv.first),
                    std::get<1>(kv.first).c_str(), (long long)std::get<2>(kv.first),
                    (long long)std::get<3>(kv.first));
      s += line;
      for (size_t v = 0; v < kv.second.ms.size(); ++v) {
        std::snprintf(line, sizeof line, "%s%s %.4f ms%s", v ? ", " : "",
                      kv.second.names[v].c_str(), kv.second.ms[v],
                      (int)v == kv.second.choice ? " (kept)" : "");
        s += line;
      }
      s += "\n";
    }
  }
  if (buf && len > 0) {
    const size_t n = std::min<size_t>(s.size(), (size_t)len - 1);
    s.copy(buf, n);
    buf[n] = '\0';
  }
  return (int)s.size();
}
