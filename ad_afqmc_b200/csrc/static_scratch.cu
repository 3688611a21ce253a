// Walker overlaps without any device allocation by library or caller.
//
// Some callers cannot hand this library a workspace: a host framework that
// owns the whole device memory pool and runs foreign kernels inside its own
// execution (for example an XLA custom call from a JAX program such as the
// reference implementation, which preallocates most of the GPU and gives a
// custom call no way to cudaMalloc mid-computation), or code that records its
// launches into a CUDA graph under a capture mode that forbids allocation.
// For them afq_calc_overlap_static keeps its per-walker scratch in a
// fixed-size array that lives in the library's own device image.
//
// Capacity: kStaticMaxWalkers walkers (16 doubles each, 1 MiB per device).
// Every GPU that loads the library holds this array until the process exits.
// The first call on a device looks the array's device address up with
// cudaGetSymbolAddress (the host-side name is only a stand-in, never a device
// address); make that first call before any stream capture.  All calls share
// the array: calls that overlap on the GPU (different streams, no ordering)
// race on it.  Nothing in it has to start at zero: each call writes every
// slot it later reads.
#include <cuda_runtime.h>

#include <mutex>

#include "afqmc_b200.h"
#include "layout.cuh"
#include "ops.h"

namespace afq {
namespace {

constexpr int kStaticMaxWalkers = 8192;
constexpr int kScratchPerWalker = 16;  // doubles (per-walker scalars of the Green's kernel)
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_overlap_scratch[kStaticMaxWalkers * kScratchPerWalker];

std::mutex g_mu;
double* g_scratch_dev[kMaxDevices] = {};

// device address of g_overlap_scratch on the current device (set up once)
int scratch_address(double** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return AFQ_ERR_CUDA;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_dev[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_overlap_scratch) != cudaSuccess || !p) return AFQ_ERR_CUDA;
    g_scratch_dev[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_dev[dev];
  return AFQ_OK;
}

}  // namespace
}  // namespace afq

using namespace afq;

extern "C" int afq_calc_overlap_static(const afq_dims* d, const double* const mo[2],
                                       const double* const walkers[2], double* overlaps,
                                       void* stream) {
  Layout L;
  int rc = make_layout(d, L);
  if (rc != AFQ_OK) return rc;
  if (L.W > kStaticMaxWalkers) return AFQ_ERR_LIMIT;
  if (!overlaps || !mo || !mo[0] || (L.uhf_trial && !mo[1])) return AFQ_ERR_NULL;
  if (!walkers || !walkers[0] || (L.ns == 2 && !walkers[1])) return AFQ_ERR_NULL;
  for (int s = 0; s < L.ns; ++s)
    if (reinterpret_cast<uintptr_t>(walkers[s]) & 15u) return AFQ_ERR_ALIGN;
  double* scratch = nullptr;
  if ((rc = scratch_address(&scratch)) != AFQ_OK) return rc;

  GreenArgs a{};
  a.N = L.N;
  a.W = L.W;
  a.ns = L.ns;
  a.wscal = scratch;
  a.gpl = nullptr;
  a.ldg = L.Kfb;
  a.npc = L.npc;
  for (int i = 0; i < 3; ++i) a.gplb[i] = nullptr;
  a.ldgb = L.Kb;
  for (int s = 0; s < L.ns; ++s) {
    a.sec[s].walk = walkers[s];
    a.sec[s].mo = mo[L.uhf_trial ? s : 0];
    a.sec[s].rh1 = nullptr;
    a.sec[s].no = L.no[s];
    a.sec[s].koff = L.koff[s];
    a.sec[s].theta = nullptr;
    a.sec[s].gout = nullptr;
    for (int i = 0; i < 3; ++i) a.sec[s].gtb[i] = nullptr;
    a.sec[s].ldtb = L.Nb;
  }
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (launch_green(a, st) != cudaSuccess) return AFQ_ERR_CUDA;
  if (launch_ovlp_combine(L.W, L.ns, L.mult, scratch, overlaps, 2, st) != cudaSuccess)
    return AFQ_ERR_CUDA;
  return AFQ_OK;
}
