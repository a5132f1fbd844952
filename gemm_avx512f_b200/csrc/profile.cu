// profile.cu -- launch counting and optional per-kernel CUDA-event timing.
#include <stdio.h>
#include <string.h>

#include <atomic>
#include <map>
#include <string>
#include <vector>

#include "b2_internal.cuh"
#include "b2_profile.cuh"

namespace b2 {

static std::atomic<long long> g_launches{0};

namespace {
struct Rec {
  const char *name;
  cudaEvent_t a, b;
};
struct ProfState {
  bool on = false;
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> pool;
  ~ProfState() {
    for (auto &r : recs) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    for (auto e : pool) cudaEventDestroy(e);
  }
  cudaEvent_t get() {
    if (!pool.empty()) { cudaEvent_t e = pool.back(); pool.pop_back(); return e; }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) { (void)cudaGetLastError(); return nullptr; }
    return e;
  }
};
thread_local ProfState g_prof;
}  // namespace

ProfScope::ProfScope(const char *name, cudaStream_t s) : name_(name), s_(s) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (!g_prof.on) return;
  a_ = g_prof.get();
  if (a_) cudaEventRecord((cudaEvent_t)a_, s);
}

ProfScope::~ProfScope() {
  if (!a_) return;
  cudaEvent_t b = g_prof.get();
  if (!b) return;
  cudaEventRecord(b, s_);
  g_prof.recs.push_back(Rec{name_, (cudaEvent_t)a_, b});
}

}  // namespace b2

using namespace b2;

extern "C" {

long long b2_launch_count(void) { return g_launches.load(); }

int b2_profile_enable(int on) {
  g_prof.on = on != 0;
  return B2_OK;
}

int b2_profile_report(char *buf, int len) {
  std::map<std::string, std::pair<long, double>> agg;
  for (auto &r : g_prof.recs) {
    float ms = 0.f;
    if (cudaEventSynchronize(r.b) == cudaSuccess && cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
      auto &v = agg[r.name];
      v.first += 1;
      v.second += ms;
    } else {
      (void)cudaGetLastError();
    }
    g_prof.pool.push_back(r.a);
    g_prof.pool.push_back(r.b);
  }
  g_prof.recs.clear();
  if (buf && len > 0) {
    buf[0] = 0;
    int off = 0;
    for (auto &kv : agg) {
      int w = snprintf(buf + off, (size_t)(len - off), "%s %ld %.6f\n", kv.first.c_str(),
                       kv.second.first, kv.second.second);
      if (w < 0 || off + w >= len) break;
      off += w;
    }
  }
  return (int)agg.size();
}

int b2_profile_timeline(char *buf, int len) {
  int n = 0, off = 0;
  if (buf && len > 0) buf[0] = 0;
  // Launches on two streams can start in another order than they were
  // recorded: times count from the earliest start of all.
  cudaEvent_t t0 = g_prof.recs.empty() ? nullptr : g_prof.recs.front().a;
  std::vector<float> at(g_prof.recs.size(), 0.f), bt(g_prof.recs.size(), 0.f);
  std::vector<char> ok(g_prof.recs.size(), 0);
  float first = 0.f;
  for (size_t i = 0; i < g_prof.recs.size(); ++i) {
    const Rec &r = g_prof.recs[i];
    if (cudaEventSynchronize(r.b) == cudaSuccess && cudaEventElapsedTime(&at[i], t0, r.a) == cudaSuccess &&
        cudaEventElapsedTime(&bt[i], t0, r.b) == cudaSuccess) {
      ok[i] = 1;
      if (at[i] < first) first = at[i];
    } else {
      (void)cudaGetLastError();
    }
  }
  for (size_t i = 0; i < g_prof.recs.size(); ++i) {
    const Rec &r = g_prof.recs[i];
    if (ok[i]) {
      const float a = at[i] - first, b = bt[i] - first;
      if (buf && len > 0 && off < len) {
        int w = snprintf(buf + off, (size_t)(len - off), "%s %.6f %.6f\n", r.name, a, b);
        if (w > 0 && off + w < len) {
          off += w;
          ++n;
        } else {
          buf[off] = 0;  // the line did not fit: drop it and stop listing
          off = len;
        }
      }
    }
  }
  for (auto &r : g_prof.recs) {
    g_prof.pool.push_back(r.a);
    g_prof.pool.push_back(r.b);
  }
  g_prof.recs.clear();
  return n;
}

}  // extern "C"
