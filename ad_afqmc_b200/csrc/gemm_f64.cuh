// FP64 tensor-core (DMMA m8n8k4) tile GEMM core for the walker path.
//
// Every FP64 contraction of the step (force bias, VHS build, one-body
// half-steps, Taylor chain, exchange energy) is one instantiation of this
// CTA-level main loop with its own epilogue.  Operands stream through a
// multistage cp.async pipeline into padded shared-memory tiles whose row
// strides (== 4 mod 16 doubles) make every fragment read conflict-free.
//
// Operand addressing (element (k, n) of B, (m, k) of A):
//   A          : ptr + b*bstride + m*ld + k                  (k contiguous)
//   B, KMAJOR  : ptr + b*bstride + k*ld + col(n)             (n contiguous)
//   B, NMAJOR  : ptr + b*bstride + col(n)*ld + k             (k contiguous)
//   col(n)     = (n / seg) * segstride + n % seg             (walker batches
//                laid side by side along n; seg = 1<<30 means plain)
// `rot` applies x -> i*x to interleaved complex columns of B on the fly:
//   B'[k][2j] = -B[k][2j+1], B'[k][2j+1] = B[k][2j]
// which turns a complex x complex product into one real GEMM with K doubled.
#pragma once

#include "common.cuh"

namespace afq {

template <int FM_, int FN_, int WM_, int WN_, int BK_ = 16, int STAGES_ = 3>
struct F64Cfg {
  static constexpr int FM = FM_, FN = FN_, WM = WM_, WN = WN_, BK = BK_, STAGES = STAGES_;
  static constexpr int TM = FM * 8, TN = FN * 8;   // warp tile
  static constexpr int BM = WM * TM, BN = WN * TN; // CTA tile
  static constexpr int NT = WM * WN * 32;
  static constexpr int AS = BK + 4;   // A tile row stride
  static constexpr int BSN = BN + 4;  // B tile row stride, n-contiguous [BK][BSN]
  static constexpr int BSK = BK + 4;  // B tile row stride, k-contiguous [BN][BSK]
  static constexpr int A_STAGE = BM * AS;
  static constexpr int B_STAGE = (BK * BSN > BN * BSK) ? BK * BSN : BN * BSK;
  static constexpr int STAGE = A_STAGE + B_STAGE;
  static constexpr size_t SMEM = size_t(STAGES) * STAGE * sizeof(double);
  static_assert(BK % 4 == 0, "BK multiple of 4");
  static_assert((BSN % 16) == 4 || (BSN % 16) == 12, "conflict-free B stride");
};

struct F64Operand {
  const double* ptr;
  long long ld;
  long long bstride;
  long long segstride;  // only B: stride between column segments
  int seg;              // only B: columns per segment (1<<30 = unsegmented)
};

enum { B_KMAJOR = 0, B_NMAJOR = 1 };

// Accumulates acc += A[m0:m0+BM, k_begin:k_end] * B[k_begin:k_end, n0:n0+BN]
// (rows >= M_lim and columns >= N_lim read as zero).
template <class Cfg, int BMODE>
__device__ __forceinline__ void f64_mainloop(double (&acc)[Cfg::FM][Cfg::FN][2],
                                             const F64Operand& A, const F64Operand& B,
                                             int M_lim, int N_lim, int k_begin, int k_end,
                                             int m0, int n0, int batch, bool rot,
                                             double* smem) {
  constexpr int BM = Cfg::BM, BN = Cfg::BN, BK = Cfg::BK, NT = Cfg::NT, ST = Cfg::STAGES;
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int wm = warp / Cfg::WN, wn = warp % Cfg::WN;
  const int g = lane >> 2, t = lane & 3;

  const double* Ab = A.ptr + (long long)batch * A.bstride;
  const double* Bb = B.ptr + (long long)batch * B.bstride;
  const int K = k_end - k_begin;
  const int KT = (K + BK - 1) / BK;

  auto load_stage = [&](int stage, int kt) {
    double* As = smem + stage * Cfg::STAGE;
    double* Bs = As + Cfg::A_STAGE;
    const int k0 = k_begin + kt * BK;
    // A tile: BM x BK, chunks of 2 doubles along k
    constexpr int ACH = BM * BK / 2;
    for (int c = tid; c < ACH; c += NT) {
      const int r = c / (BK / 2), kc = (c % (BK / 2)) * 2;
      const int gm = m0 + r, gk = k0 + kc;
      int bytes = 0;
      const double* src = Ab;
      if (gm < M_lim && gk < k_end) {
        bytes = (gk + 1 < k_end) ? 16 : 8;
        src = Ab + (long long)gm * A.ld + gk;
      }
      cp_async16(As + r * Cfg::AS + kc, src, bytes);
    }
    if (BMODE == B_KMAJOR) {
      constexpr int BCH = BK * BN / 2;
      for (int c = tid; c < BCH; c += NT) {
        const int r = c / (BN / 2), nc = (c % (BN / 2)) * 2;
        const int gk = k0 + r, gn = n0 + nc;
        int bytes = 0;
        const double* src = Bb;
        if (gk < k_end && gn < N_lim) {
          bytes = (gn + 1 < N_lim) ? 16 : 8;
          const long long col = (long long)(gn / B.seg) * B.segstride + (gn % B.seg);
          src = Bb + (long long)gk * B.ld + col;
        }
        cp_async16(Bs + r * Cfg::BSN + nc, src, bytes);
      }
    } else {
      constexpr int BCH = BN * BK / 2;
      for (int c = tid; c < BCH; c += NT) {
        const int r = c / (BK / 2), kc = (c % (BK / 2)) * 2;
        const int gn = n0 + r, gk = k0 + kc;
        int bytes = 0;
        const double* src = Bb;
        if (gn < N_lim && gk < k_end) {
          bytes = (gk + 1 < k_end) ? 16 : 8;
          src = Bb + (long long)gn * B.ld + gk;
        }
        cp_async16(Bs + r * Cfg::BSK + kc, src, bytes);
      }
    }
  };

  const double sgn = rot ? ((g & 1) ? 1.0 : -1.0) : 1.0;
  const int cx = rot ? 1 : 0;

#pragma unroll 1
  for (int s = 0; s < ST - 1; ++s) {
    if (s < KT) load_stage(s, s);
    cp_async_commit();
  }
#pragma unroll 1
  for (int kt = 0; kt < KT; ++kt) {
    cp_async_wait<ST - 2>();
    __syncthreads();
    const int nk = kt + ST - 1;
    if (nk < KT) load_stage(nk % ST, nk);
    cp_async_commit();

    const double* As = smem + (kt % ST) * Cfg::STAGE;
    const double* Bs = As + Cfg::A_STAGE;
#pragma unroll
    for (int kk = 0; kk < BK / 4; ++kk) {
      double a[Cfg::FM], b[Cfg::FN];
#pragma unroll
      for (int i = 0; i < Cfg::FM; ++i)
        a[i] = As[(wm * Cfg::TM + i * 8 + g) * Cfg::AS + kk * 4 + t];
#pragma unroll
      for (int j = 0; j < Cfg::FN; ++j) {
        const int col = wn * Cfg::TN + j * 8 + g;
        if (BMODE == B_KMAJOR)
          b[j] = sgn * Bs[(kk * 4 + t) * Cfg::BSN + (col ^ cx)];
        else
          b[j] = Bs[col * Cfg::BSK + kk * 4 + t];
      }
#pragma unroll
      for (int i = 0; i < Cfg::FM; ++i)
#pragma unroll
        for (int j = 0; j < Cfg::FN; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
  }
  cp_async_wait<0>();
  __syncthreads();
}

template <class Cfg>
__device__ __forceinline__ void f64_zero(double (&acc)[Cfg::FM][Cfg::FN][2]) {
#pragma unroll
  for (int i = 0; i < Cfg::FM; ++i)
#pragma unroll
    for (int j = 0; j < Cfg::FN; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
}

// Calls epi(m, n, v0, v1) for every accumulator pair: values of C[m][n], C[m][n+1].
template <class Cfg, class F>
__device__ __forceinline__ void f64_foreach(const double (&acc)[Cfg::FM][Cfg::FN][2], int m0,
                                            int n0, F&& epi) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = warp / Cfg::WN, wn = warp % Cfg::WN;
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int i = 0; i < Cfg::FM; ++i)
#pragma unroll
    for (int j = 0; j < Cfg::FN; ++j)
      epi(m0 + wm * Cfg::TM + i * 8 + g, n0 + wn * Cfg::TN + j * 8 + 2 * t, acc[i][j][0],
          acc[i][j][1]);
}

}  // namespace afq
