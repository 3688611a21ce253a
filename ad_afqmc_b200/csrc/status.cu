// Device-side failure status of one workspace.
//
// The tensor-core kernels never spin without bound: every mbarrier wait polls
// a limited number of times (umma.cuh), and a wait that runs out sets an int
// flag in the caller's workspace, unwinds its CTA (drains its pipeline with
// bounded waits, frees TMEM) and returns.  The launching call has returned
// AFQ_OK long before, since every entry point is asynchronous, so the walkers
// or energies of that call are garbage and the flag is the only record.
// afq_check_status reads and clears it (once per block is enough: the flag
// stays set until read); afq_status_flag gives its device address to code that
// copies it out inside a CUDA graph.  afq_test_wait_timeout makes one bounded
// wait run out on purpose, on an mbarrier that nothing arrives at and with no
// copy or MMA in flight, so tests can exercise this path without a fault.
#include <cuda_runtime.h>

#include "afqmc_b200.h"
#include "layout.cuh"
#include "umma.cuh"

namespace afq {
namespace {

int flag_ptr(const afq_dims* d, void* work, size_t work_bytes, int** out) {
  Layout L;
  const int rc = make_layout(d, L);
  if (rc != AFQ_OK) return rc;
  if (!work) return AFQ_ERR_NULL;
  if ((reinterpret_cast<uintptr_t>(work) & 15u) != 0) return AFQ_ERR_ALIGN;
  if (work_bytes < (size_t)L.work * sizeof(double)) return AFQ_ERR_WORKSPACE;
  *out = reinterpret_cast<int*>(static_cast<double*>(work) + L.w_misc);
  return AFQ_OK;
}

// One thread waits, with the same bounded poll loop as the GEMM pipelines,
// for phase 0 of a fresh mbarrier whose single expected arrival never comes.
__global__ void wait_timeout_kernel(int* flag, uint32_t polls) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x != 0) return;
  mbar_init(&bar, 1);
  fence_barrier_init();
  if (!mbar_wait(&bar, 0, polls)) atomicExch(flag, 1);
}

}  // namespace
}  // namespace afq

using namespace afq;

extern "C" {

int afq_check_status(const afq_dims* d, void* work, size_t work_bytes, void* stream) {
  int* flag = nullptr;
  int rc = flag_ptr(d, work, work_bytes, &flag);
  if (rc != AFQ_OK) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  int host = 0;
  if (cudaMemcpyAsync(&host, flag, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return AFQ_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return AFQ_ERR_CUDA;
  if (host == 0) return AFQ_OK;
  if (cudaMemsetAsync(flag, 0, sizeof(int), st) != cudaSuccess) return AFQ_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return AFQ_ERR_CUDA;
  return host == 2 ? AFQ_ERR_BOUNDS : AFQ_ERR_TIMEOUT;
}

int afq_status_flag(const afq_dims* d, void* work, size_t work_bytes, int32_t** flag) {
  if (!flag) return AFQ_ERR_NULL;
  int* p = nullptr;
  const int rc = flag_ptr(d, work, work_bytes, &p);
  if (rc != AFQ_OK) return rc;
  *flag = p;
  return AFQ_OK;
}

int afq_test_wait_timeout(const afq_dims* d, void* work, size_t work_bytes, uint32_t polls,
                          void* stream) {
  int* flag = nullptr;
  int rc = flag_ptr(d, work, work_bytes, &flag);
  if (rc != AFQ_OK) return rc;
  if (polls < 1 || polls > 4096) return AFQ_ERR_ARG;
  wait_timeout_kernel<<<1, 32, 0, reinterpret_cast<cudaStream_t>(stream)>>>(flag, polls);
  return cudaGetLastError() == cudaSuccess ? AFQ_OK : AFQ_ERR_CUDA;
}

}  // extern "C"
