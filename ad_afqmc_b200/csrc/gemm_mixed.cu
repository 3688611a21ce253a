// Split-BF16 tcgen05 contractions: host helpers (tensor maps, piece
// splitting) and a general entry point used by the mixed-precision path and
// its tests.
#include <cuda.h>
#include <cuda_bf16.h>

#include <mutex>

#include "afqmc_b200.h"
#include "common.cuh"
#include "ops.h"
#include "profile.cuh"
#include "umma_gemm.cuh"

namespace afq {

namespace {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

int g_num_sms = 0;
int num_sms() {
  if (g_num_sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_num_sms <= 0) g_num_sms = 148;
  }
  return g_num_sms;
}

// x = p0 + p1 (+ p2) in bf16, each piece rounded to nearest from the remainder
__global__ void split_kernel(const double* x, long long n, int np, __nv_bfloat16* o0,
                             __nv_bfloat16* o1, __nv_bfloat16* o2) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    double r = x[i];
    const __nv_bfloat16 a = __double2bfloat16(r);
    o0[i] = a;
    if (np > 1) {
      r -= (double)__bfloat162float(a);
      const __nv_bfloat16 b = __double2bfloat16(r);
      o1[i] = b;
      if (np > 2) {
        r -= (double)__bfloat162float(b);
        o2[i] = __double2bfloat16(r);
      }
    }
  }
}

struct StoreF32Epi {
  float* C;
  long long ldc, bstride;
  template <int BN>
  __device__ void tile(int b, int mti, int nti, int row, const AccSrc& src, const UmmaShape& s,
                       uint8_t*) const {
    const int m = mti * s.a_step + row;
#pragma unroll 1
    for (int ch = 0; ch < BN / 16; ++ch) {
      float v[16];
      src.load16(ch * 16, v);
      const int n0 = nti * s.b_step + ch * 16;
      if (m >= s.M) continue;
      float* r = C + b * bstride + (long long)m * ldc;
#pragma unroll
      for (int i = 0; i < 16; ++i)
        if (n0 + i < s.N) r[n0 + i] = v[i];
    }
  }
};

}  // namespace

int make_tmap_bf16(CUtensorMap* map, const void* base, long long K, long long rows,
                   long long batch, long long row_stride_elems, long long batch_stride_elems,
                   int box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return AFQ_ERR_CUDA;
  if ((reinterpret_cast<uintptr_t>(base) & 15u) != 0) return AFQ_ERR_ALIGN;
  if ((row_stride_elems * 2) % 16 != 0 || (batch_stride_elems * 2) % 16 != 0) return AFQ_ERR_ALIGN;
  cuuint64_t dims[3] = {(cuuint64_t)K, (cuuint64_t)rows, (cuuint64_t)batch};
  cuuint64_t strides[2] = {(cuuint64_t)row_stride_elems * 2, (cuuint64_t)batch_stride_elems * 2};
  cuuint32_t box[3] = {(cuuint32_t)kUBK, (cuuint32_t)box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(base), dims, strides,
                  box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? AFQ_OK : AFQ_ERR_ARG;
}

cudaError_t launch_split(const double* x, long long n, int np, void* o0, void* o1, void* o2,
                         cudaStream_t st) {
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  if (blocks < 1) blocks = 1;
  ProfScope ps(K_MISC, st);
  split_kernel<<<(int)blocks, 256, 0, st>>>(x, n, np, static_cast<__nv_bfloat16*>(o0),
                                           static_cast<__nv_bfloat16*>(o1),
                                           static_cast<__nv_bfloat16*>(o2));
  return cudaGetLastError();
}

int sm_count() { return num_sms(); }

}  // namespace afq

using namespace afq;

extern "C" {

int afq_split_bf16(const double* x, int64_t n, int npieces, void* const pieces[3], void* stream) {
  if (!x || !pieces) return AFQ_ERR_NULL;
  if (npieces < 1 || npieces > 3 || n < 0) return AFQ_ERR_ARG;
  for (int i = 0; i < npieces; ++i)
    if (!pieces[i]) return AFQ_ERR_NULL;
  if (n == 0) return AFQ_OK;
  if (launch_split(x, n, npieces, pieces[0], pieces[1], pieces[2],
                   reinterpret_cast<cudaStream_t>(stream)) != cudaSuccess)
    return AFQ_ERR_CUDA;
  return AFQ_OK;
}

int afq_gemm_split_bf16(const void* const a_pieces[3], int npa, const void* const b_pieces[3],
                        int npb, int npairs, const int32_t* pairs, int M, int N, int K, int batch,
                        int64_t lda, int64_t a_bstride, int64_t ldb, int64_t b_bstride, float* C,
                        int64_t ldc, int64_t c_bstride, int32_t* err_flag, void* stream) {
  if (!a_pieces || !b_pieces || !pairs || !C || !err_flag) return AFQ_ERR_NULL;
  if (npa < 1 || npa > 3 || npb < 1 || npb > 3 || npairs < 1 || npairs > 6) return AFQ_ERR_ARG;
  if (M <= 0 || N <= 0 || K <= 0 || batch <= 0) return AFQ_ERR_SHAPE;
  UmmaParams<StoreF32Epi> P{};
  for (int i = 0; i < npa; ++i) {
    if (!a_pieces[i]) return AFQ_ERR_NULL;
    int rc = make_tmap_bf16(&P.ta[i], a_pieces[i], K, M, batch, lda, a_bstride ? a_bstride : lda * M,
                            kUBM);
    if (rc != AFQ_OK) return rc;
  }
  constexpr int BN = 128;
  for (int j = 0; j < npb; ++j) {
    if (!b_pieces[j]) return AFQ_ERR_NULL;
    int rc = make_tmap_bf16(&P.tb[j], b_pieces[j], K, N, batch, ldb, b_bstride ? b_bstride : ldb * N,
                            BN);
    if (rc != AFQ_OK) return rc;
  }
  P.s.a_batched = 1;
  P.s.ngroups = 1;
  P.s.kc = 0;
  P.s.stages = umma_pick_stages(BN, npa, npb, 0);
  P.s.M = M;
  P.s.N = N;
  P.s.K = K;
  P.s.batch = batch;
  P.s.mt = (M + kUBM - 1) / kUBM;
  P.s.nt = (N + BN - 1) / BN;
  P.s.a_step = kUBM;
  P.s.b_step = BN;
  P.s.ksplit = 1;
  P.s.kchunk = (K + kUBK - 1) / kUBK * kUBK;
  P.s.npa = npa;
  P.s.npb = npb;
  P.s.npairs = npairs;
  for (int p = 0; p < npairs; ++p) {
    if (pairs[2 * p] < 0 || pairs[2 * p] >= npa || pairs[2 * p + 1] < 0 || pairs[2 * p + 1] >= npb)
      return AFQ_ERR_ARG;
    P.s.pa[p] = pairs[2 * p];
    P.s.pb[p] = pairs[2 * p + 1];
  }
  P.s.err = err_flag;
  P.epi.C = C;
  P.epi.ldc = ldc;
  P.epi.bstride = c_bstride;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  ProfScope ps(K_MISC, st);
  if (launch_umma<BN>(P, num_sms(), st) != cudaSuccess) return AFQ_ERR_CUDA;
  return AFQ_OK;
}

}  // extern "C"
