// Shared device helpers for the phaseless-AFQMC walker kernels (sm_100a).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "afqmc_b200.h"

namespace afq {

constexpr int kMaxNocc = 64;     // largest occupied block a walker kernel accepts
constexpr int kMaxWalkers = 1 << 16;

// ---------------------------------------------------------------------------
// small complex helpers (interleaved re, im as double2)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 csub(double2 a, double2 b) {
  return make_double2(a.x - b.x, a.y - b.y);
}
__device__ __forceinline__ double2 cscale(double2 a, double s) {
  return make_double2(a.x * s, a.y * s);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
// complex division a / b, scaled (Smith) to avoid overflow
__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  if (fabs(b.x) >= fabs(b.y)) {
    double r = b.y / b.x, d = b.x + b.y * r;
    return make_double2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  } else {
    double r = b.x / b.y, d = b.y + b.x * r;
    return make_double2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
  }
}

// ---------------------------------------------------------------------------
// cp.async (16-byte, zero-fill) and the FP64 tensor-core MMA (DMMA m8n8k4)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
// copies src_bytes (0, 8 or 16) and zero-fills the rest of the 16-byte chunk
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(smem)),
               "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// D = A(8x4, row) * B(4x8, col) + D ; per lane: a = A[g][t], b = B[t][g],
// d0,d1 = D[g][2t], D[g][2t+1]  with g = lane/4, t = lane%4.
__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// ---------------------------------------------------------------------------
// bf16 operand pieces: x ~= p0 + p1 (+ p2), each rounded to nearest from the remainder
// ---------------------------------------------------------------------------
typedef __nv_bfloat16 bf16;

__device__ __forceinline__ void put_pieces(double x, int np, bf16* const* P, long long idx) {
  const bf16 a = __double2bfloat16(x);
  P[0][idx] = a;
  double r = x - (double)__bfloat162float(a);
  const bf16 b = __double2bfloat16(r);
  P[1][idx] = b;
  if (np > 2) {
    r -= (double)__bfloat162float(b);
    P[2][idx] = __double2bfloat16(r);
  }
}

__device__ __forceinline__ void put_pieces_f(float x, int np, bf16* const* P, long long idx) {
  const bf16 a = __float2bfloat16_rn(x);
  P[0][idx] = a;
  float r = x - __bfloat162float(a);
  const bf16 b = __float2bfloat16_rn(r);
  P[1][idx] = b;
  if (np > 2) {
    r -= __bfloat162float(b);
    P[2][idx] = __float2bfloat16_rn(r);
  }
}

// ---------------------------------------------------------------------------
// block-level reductions
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum over the block; every thread receives the result.  `red` needs
// blockDim.x/32 doubles of shared memory.  Deterministic for a fixed launch.
__device__ __forceinline__ double block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
  for (int i = 0; i < nw; ++i) s += red[i];
  return s;
}

}  // namespace afq

#define AFQ_CUDA_TRY(expr)                                   \
  do {                                                       \
    cudaError_t _e = (expr);                                 \
    if (_e != cudaSuccess) return AFQ_ERR_CUDA;              \
  } while (0)

#define AFQ_LAUNCH_CHECK()                                   \
  do {                                                       \
    cudaError_t _e = cudaGetLastError();                     \
    if (_e != cudaSuccess) return AFQ_ERR_CUDA;              \
  } while (0)
