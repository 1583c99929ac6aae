// Per-kernel device timing with CUDA events, off unless pmg_profile_enable(1) is called.
// Each instrumented launch records an event pair on its own stream; queries wait for the
// recorded events and accumulate their elapsed times by kernel label.
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "pmg_internal.hpp"

namespace pmg {
namespace prof {
namespace {

struct Entry {
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending;
  double total_ms = 0.0;
  int64_t launches = 0;
};

std::mutex g_mu;
bool g_on = false;
std::map<std::string, Entry> g_entries;

void drain(Entry &e) {
  for (auto &pr : e.pending) {
    float ms = 0.f;
    PMG_CUDA(cudaEventSynchronize(pr.second));
    PMG_CUDA(cudaEventElapsedTime(&ms, pr.first, pr.second));
    e.total_ms += ms;
    e.launches += 1;
    cudaEventDestroy(pr.first);
    cudaEventDestroy(pr.second);
  }
  e.pending.clear();
}

} // namespace

bool enabled() { return g_on; }

void set_enabled(bool on) {
  std::lock_guard<std::mutex> lock(g_mu);
  g_on = on;
}

void reset() {
  std::lock_guard<std::mutex> lock(g_mu);
  for (auto &kv : g_entries) drain(kv.second);
  g_entries.clear();
}

Scope::Scope(const char *name_, cudaStream_t s_) : name(name_), s(s_) {
  if (!g_on) return;
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &st) != cudaSuccess || st != cudaStreamCaptureStatusNone) {
    (void)cudaGetLastError();
    return; // no timing events inside a stream capture
  }
  PMG_CUDA(cudaEventCreate(&a));
  PMG_CUDA(cudaEventRecord(a, s));
}

Scope::~Scope() {
  if (!a) return;
  cudaEvent_t b = nullptr;
  if (cudaEventCreate(&b) != cudaSuccess || cudaEventRecord(b, s) != cudaSuccess) {
    (void)cudaGetLastError();
    cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    return;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  g_entries[name].pending.emplace_back(a, b);
}

void query(const char *name, double *ms, int64_t *launches) {
  std::lock_guard<std::mutex> lock(g_mu);
  auto it = g_entries.find(name);
  if (it == g_entries.end()) {
    *ms = 0.0;
    *launches = 0;
    return;
  }
  drain(it->second);
  *ms = it->second.total_ms;
  *launches = it->second.launches;
}

} // namespace prof
} // namespace pmg
