// Launch-shape autotuner (tune.cuh): the tuning loop, the table and its file.
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <tuple>
#include "../../include/zfmm.h"
#include "devmem.cuh"
#include "tune.cuh"

namespace zf {
namespace {

struct Key {
  std::string kernel;
  int bucket, device;
  bool operator<(const Key& o) const {
    return std::tie(kernel, bucket, device) < std::tie(o.kernel, o.bucket, o.device);
  }
};

std::mutex g_mu;
std::map<Key, int> g_table;
std::atomic<int> g_on{-1};  // -1: not yet read from the environment

int bucket_of(long work) {
  int b = 0;
  while (work > 1 && b < 62) {
    work >>= 1;
    b++;
  }
  return b;
}

}  // namespace

bool autotune_enabled() {
  int v = g_on.load();
  if (v < 0) {
    const char* e = getenv("ZFMM_AUTOTUNE");
    v = (e && *e && strcmp(e, "0") != 0) ? 1 : 0;
    g_on.store(v);
  }
  return v == 1;
}

int tuned_launch(const char* name, long work, int dflt, const std::vector<int>& cands,
                 const std::function<void(int)>& launch, cudaStream_t s,
                 const std::function<void()>& reset) {
  if (!autotune_enabled() || cands.empty()) {
    launch(dflt);
    return dflt;
  }
  int dev = 0;
  ZF_CUDA(cudaGetDevice(&dev));
  Key k{name, bucket_of(work), dev};
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_table.find(k);
    if (it != g_table.end()) {
      launch(it->second);
      return it->second;
    }
  }
  cudaEvent_t e0, e1;
  ZF_CUDA(cudaEventCreate(&e0));
  ZF_CUDA(cudaEventCreate(&e1));
  int best = dflt;
  float best_ms = 1e30f;
  for (int b : cands) {
    float ms = 0;
    for (int rep = 0; rep < 2; rep++) {
      if (reset) reset();
      ZF_CUDA(cudaEventRecord(e0, s));
      launch(b);
      ZF_CUDA(cudaEventRecord(e1, s));
      ZF_CUDA(cudaEventSynchronize(e1));
      ZF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    }
    if (ms < best_ms) {
      best_ms = ms;
      best = b;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (reset) reset();
  launch(best);
  std::lock_guard<std::mutex> lk(g_mu);
  g_table[k] = best;
  return best;
}

}  // namespace zf

using namespace zf;

extern "C" {

void zfmm_set_autotune(int on) { g_on.store(on ? 1 : 0); }

int zfmm_autotune_entries(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  return (int)g_table.size();
}

int zfmm_autotune_save(const char* path) {
  if (!path) return 1;
  std::lock_guard<std::mutex> lk(g_mu);
  std::ofstream f(path);
  if (!f) return 1;
  for (auto& kv : g_table)
    f << kv.first.kernel << ' ' << kv.first.bucket << ' ' << kv.first.device << ' '
      << kv.second << '\n';
  return f ? 0 : 1;
}

int zfmm_autotune_load(const char* path) {
  if (!path) return 1;
  std::ifstream f(path);
  if (!f) return 1;
  std::map<Key, int> t;
  std::string line;
  while (std::getline(f, line)) {
    if (line.empty()) continue;
    std::istringstream ss(line);
    Key k;
    int b;
    if (!(ss >> k.kernel >> k.bucket >> k.device >> b) || b < 32 || b > 1024 || b % 32)
      return 1;  // the whole file is refused on any bad line
    t[k] = b;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  for (auto& kv : t) g_table[kv.first] = kv.second;
  return 0;
}

}  // extern "C"
