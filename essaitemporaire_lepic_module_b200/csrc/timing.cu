// Per-kernel CUDA-event timers.  When enabled, every named launch is
// bracketed by two events recorded on its own stream; lepic_timing_read()
// waits for the pending events and accumulates device time per name.  This
// measures the kernels themselves, not the host gaps between launches.
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "lepic_internal.cuh"

namespace lepic {

namespace {
struct Pending {
  std::string name;
  cudaEvent_t a, b;
};
std::mutex g_tmu;
bool g_on = false;
std::vector<Pending> g_pending;
std::vector<cudaEvent_t> g_pool;
std::map<std::string, std::pair<double, long long>> g_tot;

cudaEvent_t take() {
  if (!g_pool.empty()) {
    cudaEvent_t e = g_pool.back();
    g_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

void collect_locked() {
  for (auto &p : g_pending) {
    cudaEventSynchronize(p.b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, p.a, p.b);
    auto &t = g_tot[p.name];
    t.first += ms;
    t.second += 1;
    g_pool.push_back(p.a);
    g_pool.push_back(p.b);
  }
  g_pending.clear();
}
}  // namespace

int timer_start(const char *name, cudaStream_t s) {
  std::lock_guard<std::mutex> lk(g_tmu);
  if (!g_on) return -1;
  if (g_pending.size() > 4096) collect_locked();
  Pending p;
  p.name = name;
  p.a = take();
  p.b = take();
  cudaEventRecord(p.a, s);
  g_pending.push_back(p);
  return (int)g_pending.size() - 1;
}

void timer_stop(int id, cudaStream_t s) {
  if (id < 0) return;
  std::lock_guard<std::mutex> lk(g_tmu);
  if (id < (int)g_pending.size()) cudaEventRecord(g_pending[id].b, s);
}

}  // namespace lepic

extern "C" {

void lepic_timing_enable(int on) {
  std::lock_guard<std::mutex> lk(lepic::g_tmu);
  lepic::g_on = on != 0;
}

void lepic_timing_reset(void) {
  std::lock_guard<std::mutex> lk(lepic::g_tmu);
  lepic::collect_locked();
  lepic::g_tot.clear();
}

// Names separated by '\n' into buf; per name total device ms and launches.
int lepic_timing_read(char *buf, int buflen, double *ms, long long *launches, int max_names) {
  std::lock_guard<std::mutex> lk(lepic::g_tmu);
  lepic::collect_locked();
  int k = 0;
  std::string all;
  for (auto &kv : lepic::g_tot) {
    if (k >= max_names) break;
    ms[k] = kv.second.first;
    launches[k] = kv.second.second;
    all += kv.first;
    all += '\n';
    ++k;
  }
  if (buf && buflen > 0) {
    size_t n = all.size() < (size_t)buflen - 1 ? all.size() : (size_t)buflen - 1;
    memcpy(buf, all.data(), n);
    buf[n] = 0;
  }
  return k;
}

}  // extern "C"
