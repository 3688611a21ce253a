// Launch counting and per-kernel CUDA-event timing (instrumentation only).
#pragma once

#include <cuda_runtime.h>

namespace afq {

enum KernelId {
  K_GREEN = 0, K_FB = 1, K_PREP = 2, K_VHS = 3, K_PROP = 4, K_EXCH = 5, K_ECOMB = 6,
  K_WEIGHT = 7, K_QR = 8, K_SR = 9, K_GATHER = 10, K_BLOCKEND = 11, K_NORMAL = 12,
  K_MISC = 13, K_COUNT = 14
};

// Called around every kernel launch of the library, on the launch stream.
void prof_before(int id, cudaStream_t st);
void prof_after(int id, cudaStream_t st);

struct ProfScope {
  int id;
  cudaStream_t st;
  ProfScope(int i, cudaStream_t s) : id(i), st(s) { prof_before(id, st); }
  ~ProfScope() { prof_after(id, st); }
};

}  // namespace afq
