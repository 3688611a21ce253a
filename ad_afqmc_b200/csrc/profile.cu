// Instrumentation: a launch counter per kernel family and optional CUDA-event
// timing of one family, recorded on the stream each launch uses.
#include <atomic>
#include <mutex>

#include "afqmc_b200.h"
#include "profile.cuh"

namespace afq {

namespace {
std::atomic<unsigned long long> g_launches[K_COUNT];
std::mutex g_mu;
int g_target = -1;
constexpr int kMaxEvents = 16384;
cudaEvent_t g_ev[2][kMaxEvents];
bool g_created = false;
int g_n = 0;
}  // namespace

void prof_before(int id, cudaStream_t st) {
  g_launches[id].fetch_add(1, std::memory_order_relaxed);
  if (id != g_target) return;
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_target == id && g_n < kMaxEvents) cudaEventRecord(g_ev[0][g_n], st);
}

void prof_after(int id, cudaStream_t st) {
  if (id != g_target) return;
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_target == id && g_n < kMaxEvents) {
    cudaEventRecord(g_ev[1][g_n], st);
    ++g_n;
  }
}

}  // namespace afq

using namespace afq;

extern "C" {

int afq_launch_count(int kernel_id, unsigned long long* count) {
  if (!count) return AFQ_ERR_NULL;
  if (kernel_id < 0) {
    unsigned long long s = 0;
    for (int i = 0; i < K_COUNT; ++i) s += g_launches[i].load();
    *count = s;
    return AFQ_OK;
  }
  if (kernel_id >= K_COUNT) return AFQ_ERR_ARG;
  *count = g_launches[kernel_id].load();
  return AFQ_OK;
}

int afq_profile_begin(int kernel_id) {
  if (kernel_id < 0 || kernel_id >= K_COUNT) return AFQ_ERR_ARG;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_created) {
    for (int i = 0; i < kMaxEvents; ++i) {
      if (cudaEventCreate(&g_ev[0][i]) != cudaSuccess) return AFQ_ERR_CUDA;
      if (cudaEventCreate(&g_ev[1][i]) != cudaSuccess) return AFQ_ERR_CUDA;
    }
    g_created = true;
  }
  g_n = 0;
  g_target = kernel_id;
  return AFQ_OK;
}

int afq_profile_end(double* total_ms, int* launches) {
  if (!total_ms || !launches) return AFQ_ERR_NULL;
  std::lock_guard<std::mutex> lk(g_mu);
  g_target = -1;
  double tot = 0.0;
  for (int i = 0; i < g_n; ++i) {
    if (cudaEventSynchronize(g_ev[1][i]) != cudaSuccess) return AFQ_ERR_CUDA;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, g_ev[0][i], g_ev[1][i]) != cudaSuccess) return AFQ_ERR_CUDA;
    tot += ms;
  }
  *total_ms = tot;
  *launches = g_n;
  g_n = 0;
  return AFQ_OK;
}

}  // extern "C"
