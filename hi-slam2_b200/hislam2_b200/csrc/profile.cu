// Opt-in per-kernel timing with CUDA events recorded on the launching stream.
//
// When enabled (hs2_profile_enable(1)), every kernel launch of the library is
// bracketed by a pair of events from a pool; hs2_profile_report() waits for the
// recorded events, sums the elapsed time per kernel name and returns one line
// per kernel: "<name> <launches> <total_ms>".  Disabled (the default), the
// bracketing costs one branch per launch.
#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "profile.cuh"

namespace hs2 {

namespace {
struct Rec {
  const char* name;
  cudaEvent_t start, stop;
};
std::mutex g_mu;
std::atomic<bool> g_enabled{false};   // read without the lock on every launch
std::vector<Rec> g_recs;        // recorded pairs since the last reset
std::vector<cudaEvent_t> g_pool;  // spare events
}  // namespace

static cudaEvent_t take_event() {
  if (!g_pool.empty()) {
    cudaEvent_t e = g_pool.back();
    g_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
  return e;
}

ProfScope::ProfScope(const char* name, cudaStream_t s) : name_(name), stream_(s), start_(nullptr) {
  if (!g_enabled.load(std::memory_order_relaxed)) return;
  std::lock_guard<std::mutex> lk(g_mu);
  start_ = take_event();
  if (start_) cudaEventRecord(start_, stream_);
}

ProfScope::~ProfScope() {
  if (!start_) return;
  std::lock_guard<std::mutex> lk(g_mu);
  cudaEvent_t stop = take_event();
  if (!stop) return;
  cudaEventRecord(stop, stream_);
  g_recs.push_back({name_, start_, stop});
}

}  // namespace hs2

extern "C" void hs2_profile_enable(int on) {
  hs2::g_enabled.store(on != 0, std::memory_order_relaxed);
}

extern "C" int hs2_profile_report(char* buf, size_t len, int reset) {
  using namespace hs2;
  std::lock_guard<std::mutex> lk(g_mu);
  std::vector<std::string> names;
  std::vector<double> total;
  std::vector<long> count;
  for (const Rec& r : g_recs) {
    float ms = 0.f;
    if (cudaEventSynchronize(r.stop) != cudaSuccess) return cuda_status(cudaGetLastError(), "cudaEventSynchronize");
    if (cudaEventElapsedTime(&ms, r.start, r.stop) != cudaSuccess) ms = 0.f;
    size_t k = 0;
    while (k < names.size() && names[k] != r.name) ++k;
    if (k == names.size()) {
      names.emplace_back(r.name);
      total.push_back(0.0);
      count.push_back(0);
    }
    total[k] += ms;
    count[k] += 1;
  }
  std::string out;
  char line[256];
  for (size_t k = 0; k < names.size(); ++k) {
    snprintf(line, sizeof(line), "%s %ld %.6f\n", names[k].c_str(), count[k], total[k]);
    out += line;
  }
  if (buf && len) {
    strncpy(buf, out.c_str(), len - 1);
    buf[len - 1] = 0;
  }
  if (reset) {
    for (const Rec& r : g_recs) {
      g_pool.push_back(r.start);
      g_pool.push_back(r.stop);
    }
    g_recs.clear();
  }
  return (int)out.size();
}
