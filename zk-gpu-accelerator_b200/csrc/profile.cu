// profile.cu — the stage timer behind profile.h and its C ABI.
#include <atomic>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "profile.h"

namespace zkb {

namespace {
struct Span {
  const char* name;
  cudaEvent_t start, stop;
};
std::atomic<bool> g_on{false};
std::mutex g_mu;
std::vector<Span> g_spans;
std::vector<cudaEvent_t> g_free;  // reusable events

cudaEvent_t take_event() {
  if (!g_free.empty()) {
    cudaEvent_t e = g_free.back();
    g_free.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
  return e;
}
}  // namespace

bool prof_enabled() { return g_on.load(std::memory_order_relaxed); }

int prof_begin(const char* name, cudaStream_t s) {
  if (!prof_enabled()) return -1;
  std::lock_guard<std::mutex> lock(g_mu);
  Span sp{name, take_event(), take_event()};
  if (!sp.start || !sp.stop) return -1;
  cudaEventRecord(sp.start, s);
  g_spans.push_back(sp);
  return (int)g_spans.size() - 1;
}

void prof_end(int id, cudaStream_t s) {
  if (id < 0) return;
  std::lock_guard<std::mutex> lock(g_mu);
  if (id < (int)g_spans.size()) cudaEventRecord(g_spans[id].stop, s);
}

}  // namespace zkb

extern "C" {

void zkb_profile_enable(int on) {
  std::lock_guard<std::mutex> lock(zkb::g_mu);
  for (auto& sp : zkb::g_spans) {
    zkb::g_free.push_back(sp.start);
    zkb::g_free.push_back(sp.stop);
  }
  zkb::g_spans.clear();
  zkb::g_on.store(on != 0);
}

int zkb_profile_report(char* buf, size_t len) {
  std::lock_guard<std::mutex> lock(zkb::g_mu);
  std::map<std::string, std::pair<long, double>> agg;
  for (auto& sp : zkb::g_spans) {
    if (cudaEventSynchronize(sp.stop) != cudaSuccess) continue;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, sp.start, sp.stop) != cudaSuccess) continue;
    auto& a = agg[sp.name];
    a.first += 1;
    a.second += ms;
  }
  std::string out;
  for (auto& kv : agg) {
    char line[256];
    snprintf(line, sizeof line, "%s %ld %.6f\n", kv.first.c_str(), kv.second.first, kv.second.second);
    out += line;
  }
  if (buf && len) {
    size_t n = out.size() < len - 1 ? out.size() : len - 1;
    std::memcpy(buf, out.data(), n);
    buf[n] = 0;
  }
  return (int)out.size() + 1;
}

}  // extern "C"
