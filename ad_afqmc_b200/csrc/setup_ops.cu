// Per-solve Hamiltonian intermediates on the device (FP64).
//
//  measurement   h1[s] <- (h1[s] + h1[s]^T) / 2 ;  rot_h1 = C^T h ;  rot_chol[g] = C^T L_g
//                (rhf/uhf._build_measurement_intermediates, wavefunctions.py:1215-1232, 1472-1496)
//  propagation   mf_shifts[g] = i sum(L_g o rho) ;  h0_prop = -h0 - sum(mf^2) / 2 ;
//                v0 = 1/2 sum_g L_g L_g ;  v1 = sum_g Re(i mf_g) L_g ;
//                exp_h1 = expm(-dt/2 (h1 - v0 - v1))
//                (propagator_afqmc._build_propagation_intermediates, propagation.py:378-438)
//  natural orbitals  eigenpairs of a symmetric matrix, descending
//                (wave_function.get_init_walkers, wavefunctions.py:427-466)
//
// The contractions run on the FP64 tensor cores through the same DMMA main
// loop as the walker kernels (gemm_f64.cuh), which copies 16-byte pieces:
// every operand it reads has an even leading dimension (odd N: the Cholesky
// vectors and square matrices are first copied to padded rows).  v0 is a split-K GEMM over the
// Cholesky index with partial sums added in a fixed order, so results do not
// depend on the device.  The matrix exponential is scaling and squaring of
// a truncated Taylor series (Moler and Van Loan, "Nineteen dubious ways to
// compute the exponential of a matrix, twenty-five years later", SIAM Review
// 45 (2003), method 3), with the degree chosen from the remainder bound
// theta^(m+1) / (m+1)! * e^theta <= 2^-53 for theta = ||A / 2^s||_1 <= 1/2.
// The eigensolver is the cyclic two-sided Jacobi method in the parallel
// round-robin ordering (Golub and Van Loan, Matrix Computations, 4th ed.,
// sections 8.5.2 and 8.5.5), run by one CTA on a copy of the matrix.
#include <cuda_runtime.h>

#include <math.h>

#include <algorithm>
#include <vector>

#include "afqmc_b200.h"
#include "common.cuh"
#include "gemm_f64.cuh"
#include "ops.h"
#include "profile.cuh"

namespace afq {
namespace {

constexpr int kUnsegS = 1 << 30;
using CfgS = F64Cfg<2, 4, 4, 2>;    // 64 x 64, 8 warps: rot_chol, rot_h1, expm
using CfgV0 = F64Cfg<4, 8, 4, 2>;   // 128 x 128, 8 warps: v0

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }
inline bool al16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }
inline long long even(long long x) { return (x + 1) & ~1LL; }

// C[z] = alpha * sum_{b in batches of z} A[b] B[b] (+ beta Cin[z]) (+ diag on the diagonal)
struct DgemmArgs {
  F64Operand A, B;
  int M, N, K;
  int nbatch;      // input batches
  int bsum;        // 0: output z uses input batch z; > 0: output z sums batches [z bsum, (z+1) bsum)
  double alpha, beta, diag;
  const double* cin;
  long long ldcin, cin_bs;
  double* C;
  long long ldc, c_bs;
};

template <class Cfg, int BMODE = B_KMAJOR>
__global__ void __launch_bounds__(Cfg::NT) dgemm_kernel(DgemmArgs a) {
  extern __shared__ double smem[];
  const int m0 = blockIdx.x * Cfg::BM, n0 = blockIdx.y * Cfg::BN, z = blockIdx.z;
  double acc[Cfg::FM][Cfg::FN][2];
  f64_zero<Cfg>(acc);
  int b0 = z, b1 = z + 1;
  if (a.bsum > 0) {
    b0 = z * a.bsum;
    b1 = min(a.nbatch, b0 + a.bsum);
  }
  for (int b = b0; b < b1; ++b)
    f64_mainloop<Cfg, BMODE>(acc, a.A, a.B, a.M, a.N, 0, a.K, m0, n0, b, false, smem);
  double* Cz = a.C + (long long)z * a.c_bs;
  const double* Iz = a.cin ? a.cin + (long long)z * a.cin_bs : nullptr;
  f64_foreach<Cfg>(acc, m0, n0, [&](int m, int n, double v0, double v1) {
    if (m >= a.M) return;
    double v[2] = {v0, v1};
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int c = n + j;
      if (c >= a.N) continue;
      double x = a.alpha * v[j];
      if (Iz) x += a.beta * Iz[(long long)m * a.ldcin + c];
      if (m == c) x += a.diag;
      Cz[(long long)m * a.ldc + c] = x;
    }
  });
}

// B_KMAJOR: B element (k, n) at ptr + k ld + n;  B_NMAJOR: at ptr + n ld + k
template <class Cfg, int BMODE = B_KMAJOR>
cudaError_t dgemm(const DgemmArgs& a, int zdim, cudaStream_t st) {
  cudaError_t e = cudaFuncSetAttribute(dgemm_kernel<Cfg, BMODE>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::SMEM);
  if (e != cudaSuccess) return e;
  dim3 grid((a.M + Cfg::BM - 1) / Cfg::BM, (a.N + Cfg::BN - 1) / Cfg::BN, zdim);
  ProfScope ps(K_MISC, st);
  dgemm_kernel<Cfg, BMODE><<<grid, Cfg::NT, Cfg::SMEM, st>>>(a);
  return cudaGetLastError();
}

// C (M x N, ldc) = alpha A (M x K, lda) B, B k-major (K x N, ldb) or n-major (N x K, ldb)
template <int BMODE>
cudaError_t gemm2(int M, int N, int K, const double* A, long long lda, const double* B, long long ldb,
                  double alpha, double* C, long long ldc, cudaStream_t st) {
  DgemmArgs a{};
  a.A = F64Operand{A, lda, 0, 0, kUnsegS};
  a.B = F64Operand{B, ldb, 0, 0, kUnsegS};
  a.M = M;
  a.N = N;
  a.K = K;
  a.nbatch = 1;
  a.alpha = alpha;
  a.C = C;
  a.ldc = ldc;
  return dgemm<CfgS, BMODE>(a, 1, st);
}

// plain square product C = alpha A B (+ diag I), n x n row-major, all with the
// (even) row stride ld
cudaError_t square_gemm(int n, long long ld, const double* A, const double* B, double alpha,
                        double diag, double* C, cudaStream_t st) {
  DgemmArgs a{};
  a.A = F64Operand{A, ld, 0, 0, kUnsegS};
  a.B = F64Operand{B, ld, 0, 0, kUnsegS};
  a.M = a.N = a.K = n;
  a.nbatch = 1;
  a.alpha = alpha;
  a.diag = diag;
  a.C = C;
  a.ldc = ld;
  return dgemm<CfgS>(a, 1, st);
}

// dst[r * ldd + c] = src[r * lds + c] for r < rows, c < cols
__global__ void copy2d_kernel(long long rows, int cols, const double* src, long long lds, double* dst,
                              long long ldd) {
  const long long n = rows * cols;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const long long r = e / cols;
    const int c = (int)(e - r * cols);
    dst[r * ldd + c] = src[r * lds + c];
  }
}

cudaError_t copy2d(long long rows, int cols, const double* src, long long lds, double* dst,
                   long long ldd, cudaStream_t st) {
  long long blocks = (rows * cols + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  if (blocks < 1) blocks = 1;
  ProfScope ps(K_MISC, st);
  copy2d_kernel<<<(int)blocks, 256, 0, st>>>(rows, cols, src, lds, dst, ldd);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// measurement intermediates
// ---------------------------------------------------------------------------
// h1[s] <- (h1[s] + h1[s]^T)/2 in place for both spins; hrot[0] = RHF: (h1[0]+h1[1])/2,
// UHF: h1[0]; hrot[1] = h1[1] (UHF only); mot[s] = mo[s]^T (no x N)
__global__ void sym_kernel(int n, double* h1, double* hrot, long long ldh, int uhf) {
  const long long nn = (long long)n * n, hs = (long long)n * ldh;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nn;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e / n), j = (int)(e % n);
    if (i > j) continue;
    double a[2];
    for (int s = 0; s < 2; ++s) {
      a[s] = 0.5 * (h1[s * nn + (long long)i * n + j] + h1[s * nn + (long long)j * n + i]);
    }
    for (int s = 0; s < 2; ++s) {
      h1[s * nn + (long long)i * n + j] = a[s];
      h1[s * nn + (long long)j * n + i] = a[s];
    }
    if (uhf) {
      for (int s = 0; s < 2; ++s) {
        hrot[s * hs + (long long)i * ldh + j] = a[s];
        hrot[s * hs + (long long)j * ldh + i] = a[s];
      }
    } else {
      const double v = 0.5 * (a[0] + a[1]);
      hrot[(long long)i * ldh + j] = v;
      hrot[(long long)j * ldh + i] = v;
    }
  }
}

// out (cols x rows, row stride ldo) = in (rows x cols, row stride ldi)^T
__global__ void transpose_kernel(int rows, int cols, const double* in, long long ldi, double* out,
                                 long long ldo) {
  const long long nn = (long long)rows * cols;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nn;
       e += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(e / cols), c = (int)(e % cols);
    out[(long long)c * ldo + r] = in[(long long)r * ldi + c];
  }
}

// ---------------------------------------------------------------------------
// propagation intermediates
// ---------------------------------------------------------------------------
// s_g = sum_ij L_g[ij] rho[ij] (one CTA per g); mf[g] = (0, s_g)
__global__ void __launch_bounds__(256) mf_kernel(long long nn, const double* chol, const double* rho,
                                                 double* mf) {
  __shared__ double red[8];
  const int g = blockIdx.x;
  const double* L = chol + (long long)g * nn;
  double s = 0.0;
  for (long long e = threadIdx.x; e < nn; e += blockDim.x) s += L[e] * rho[e];
  s = block_sum(s, red);
  if (threadIdx.x == 0) {
    mf[2 * g] = 0.0;
    mf[2 * g + 1] = s;
  }
}

// h0_prop = -h0 - sum_g mf_g^2 / 2 with mf_g = i s_g: -h0 + sum s_g^2 / 2 (real), one CTA
__global__ void __launch_bounds__(256) h0prop_kernel(int G, const double* mf, double h0,
                                                     double* h0p) {
  __shared__ double red[8];
  double s = 0.0;
  for (int g = threadIdx.x; g < G; g += blockDim.x) s += mf[2 * g + 1] * mf[2 * g + 1];
  s = block_sum(s, red);
  if (threadIdx.x == 0) {
    h0p[0] = -h0 + 0.5 * s;
    h0p[1] = 0.0;
  }
}

// v1 partial sums: part[z][ij] = sum_{g in z-th range} (-s_g) L_g[ij]
__global__ void __launch_bounds__(256) v1_kernel(long long nn, int G, int gper, const double* chol,
                                                 const double* mf, double* part) {
  const int z = blockIdx.y;
  const int g0 = z * gper, g1 = min(G, g0 + gper);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nn;
       e += (long long)gridDim.x * blockDim.x) {
    double v = 0.0;
    for (int g = g0; g < g1; ++g) v -= mf[2 * g + 1] * chol[(long long)g * nn + e];
    part[(long long)z * nn + e] = v;
  }
}

// out[s] = scale * (h[s] - 1/2 sum_z v0part[z] - sum_z v1part[z]) for s < np
// (h: restricted (h1[0]+h1[1])/2, unrestricted h1[s])
__global__ void hmod_kernel(long long nn, int np, const double* h1, int avg, const double* v0p,
                            int nz0, const double* v1p, int nz1, double scale, double* out) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nn;
       e += (long long)gridDim.x * blockDim.x) {
    double v0 = 0.0, v1 = 0.0;
    for (int z = 0; z < nz0; ++z) v0 += v0p[(long long)z * nn + e];
    for (int z = 0; z < nz1; ++z) v1 += v1p[(long long)z * nn + e];
    const double v = 0.5 * v0 + v1;
    for (int s = 0; s < np; ++s) {
      const double h = avg ? 0.5 * (h1[e] + h1[nn + e]) : h1[s * nn + e];
      out[s * nn + e] = scale * (h - v);
    }
  }
}

// ---------------------------------------------------------------------------
// matrix exponential helpers
// ---------------------------------------------------------------------------
// ||A||_1 (largest column sum of |a_ij|), one CTA
__global__ void __launch_bounds__(256) norm1_kernel(int n, const double* A, long long lda, double* out) {
  __shared__ double red[256];
  double m = 0.0;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += fabs(A[(long long)i * lda + j]);
    m = fmax(m, s);
  }
  red[threadIdx.x] = m;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

// P = I + B / m  (the innermost Horner factor); both with row stride ld
__global__ void horner_init_kernel(int n, long long ld, const double* B, double inv_m, double* P) {
  const long long nn = (long long)n * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nn;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e / n), j = (int)(e % n);
    P[i * ld + j] = B[i * ld + j] * inv_m + (i == j ? 1.0 : 0.0);
  }
}

// ---------------------------------------------------------------------------
// Jacobi eigensolver (one CTA)
// ---------------------------------------------------------------------------
constexpr int kJacobiThreads = 1024;
constexpr int kJacobiMaxSweeps = 40;
constexpr int kJacobiMaxN = 2048;

// round-robin pairing: position k of round r (n even, positions 0..n-1)
__device__ __forceinline__ int rr_index(int k, int r, int n) {
  if (k == 0) return 0;
  return 1 + (k - 1 + r) % (n - 1);
}

// Symmetric matrix storage: the packed upper triangle in shared memory
// (PACKED) or the full matrix in global memory.
template <bool PACKED>
struct SymMat {
  double* a;
  int n;
  __device__ __forceinline__ double* at(int i, int j) const {
    if (PACKED) {
      if (i > j) {
        const int t = i;
        i = j;
        j = t;
      }
      return a + (i * (2 * n - i + 1)) / 2 + (j - i);
    }
    return a + (long long)i * n + j;
  }
};
__host__ __device__ inline long long packed_len(int n) { return (long long)n * (n + 1) / 2; }

// Eigenpairs of the symmetric matrix in M: one round applies the npair
// disjoint rotations of the round-robin ordering at once.  The 2x2 block of A
// on rows {p1, q1} and columns {p2, q2} becomes J1^T A J2 (J = [[c, s], [-s,
// c]] on (p, q)); only blocks with k1 <= k2 are updated (the others are their
// transposes, the same storage), and the rotated pair's off-diagonal element
// is set to zero.  The eigenvectors accumulate transposed in VT (global, row p
// of VT is column p of V, so a rotation updates two contiguous rows).  The
// padding index n (odd n) is a phantom without rotations.  Sweeps stop when
// the off-diagonal Frobenius norm is at most 4 n eps of the matrix's, or when a
// sweep no longer reduces it (the rounding floor).
template <bool PACKED>
__device__ void jacobi_body(const SymMat<PACKED> M, double* VT, double* evals, double* evecs,
                            int* sweeps_out, double* cs, double* sn, int* pp, int* qq) {
  __shared__ double red[32];
  const int n = M.n;
  const int np = (n + 1) & ~1;
  const int npair = np / 2;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int e = tid; e < n * n; e += nt) VT[e] = ((e / n) == (e % n)) ? 1.0 : 0.0;
  double fro = 0.0;
  for (int e = tid; e < n * n; e += nt) {
    const double x = *M.at(e / n, e % n);
    fro += x * x;
  }
  fro = block_sum(fro, red);
  const double eps = 2.220446049250313e-16;
  const double tol2 = fro * (4.0 * n * eps) * (4.0 * n * eps);
  double prev = -1.0;
  int sweep = 0;
  for (; sweep < kJacobiMaxSweeps; ++sweep) {
    double off = 0.0;
    for (int e = tid; e < n * n; e += nt) {
      const int i = e / n, j = e - i * n;
      if (i != j) {
        const double x = *M.at(i, j);
        off += x * x;
      }
    }
    off = block_sum(off, red);
    if (off <= tol2 || fro == 0.0 || (prev >= 0.0 && off >= prev)) break;
    prev = off;
    for (int r = 0; r < np - 1; ++r) {
      // rotation parameters (Golub & Van Loan, Algorithm 8.5.1, sym.schur2)
      for (int k = tid; k < npair; k += nt) {
        int p = rr_index(k, r, np), q = rr_index(np - 1 - k, r, np);
        if (p > q) {
          const int t = p;
          p = q;
          q = t;
        }
        double c = 1.0, s = 0.0;
        if (q < n) {
          const double apq = *M.at(p, q);
          if (apq != 0.0) {
            const double app = *M.at(p, p), aqq = *M.at(q, q);
            const double tau = (aqq - app) / (2.0 * apq);
            const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            c = 1.0 / sqrt(1.0 + t * t);
            s = t * c;
          }
        }
        cs[k] = c;
        sn[k] = s;
        pp[k] = p;
        qq[k] = q < n ? q : -1;
      }
      __syncthreads();
      // A <- J^T A J, one 2x2 block per (k1 <= k2)
      const int nblk = npair * (npair + 1) / 2;
      for (int it = tid; it < nblk; it += nt) {
        // it -> (k1, k2), k1 <= k2, row-major over the upper triangle of pairs
        int k1 = (int)((2.0 * npair + 1.0 - sqrt((2.0 * npair + 1.0) * (2.0 * npair + 1.0) - 8.0 * it)) * 0.5);
        while (k1 > 0 && k1 * (2 * npair - k1 + 1) / 2 > it) --k1;
        while ((k1 + 1) * (2 * npair - k1) / 2 <= it) ++k1;
        const int k2 = k1 + (it - k1 * (2 * npair - k1 + 1) / 2);
        const int p1 = pp[k1], q1 = qq[k1], p2 = pp[k2], q2 = qq[k2];
        const double c1 = cs[k1], s1 = sn[k1], c2 = cs[k2], s2 = sn[k2];
        if (s1 == 0.0 && s2 == 0.0) continue;
        if (k1 == k2) {  // the pair's own symmetric 2x2 block
          if (q1 < 0) continue;
          const double x00 = *M.at(p1, p1), x01 = *M.at(p1, q1), x11 = *M.at(q1, q1);
          const double a00 = c1 * x00 - s1 * x01, a01 = s1 * x00 + c1 * x01;
          const double a10 = c1 * x01 - s1 * x11, a11 = s1 * x01 + c1 * x11;
          *M.at(p1, p1) = c1 * a00 - s1 * a10;
          *M.at(q1, q1) = s1 * a01 + c1 * a11;
          *M.at(p1, q1) = 0.0;
          if (!PACKED) *M.at(q1, p1) = 0.0;
          continue;
        }
        const double x00 = *M.at(p1, p2);
        const double x01 = q2 >= 0 ? *M.at(p1, q2) : 0.0;
        const double x10 = q1 >= 0 ? *M.at(q1, p2) : 0.0;
        const double x11 = (q1 >= 0 && q2 >= 0) ? *M.at(q1, q2) : 0.0;
        // columns: [y0 y1] = [x0 x1] J2, then rows: J1^T
        const double a00 = c2 * x00 - s2 * x01, a01 = s2 * x00 + c2 * x01;
        const double a10 = c2 * x10 - s2 * x11, a11 = s2 * x10 + c2 * x11;
        const double b00 = c1 * a00 - s1 * a10, b01 = c1 * a01 - s1 * a11;
        const double b10 = s1 * a00 + c1 * a10, b11 = s1 * a01 + c1 * a11;
        *M.at(p1, p2) = b00;
        if (!PACKED) *M.at(p2, p1) = b00;
        if (q2 >= 0) {
          *M.at(p1, q2) = b01;
          if (!PACKED) *M.at(q2, p1) = b01;
        }
        if (q1 >= 0) {
          *M.at(q1, p2) = b10;
          if (!PACKED) *M.at(p2, q1) = b10;
          if (q2 >= 0) {
            *M.at(q1, q2) = b11;
            if (!PACKED) *M.at(q2, q1) = b11;
          }
        }
      }
      // V <- V J: rows p, q of VT
      for (int it = tid; it < npair * n; it += nt) {
        const int k = it / n, i = it - k * n;
        const int p = pp[k], q = qq[k];
        const double s = sn[k];
        if (q < 0 || s == 0.0) continue;
        const double c = cs[k];
        double* vp = VT + (long long)p * n + i;
        double* vq = VT + (long long)q * n + i;
        const double u = *vp, w = *vq;
        *vp = c * u - s * w;
        *vq = s * u + c * w;
      }
      __syncthreads();
    }
  }
  // descending order: rank of eigenvalue i (ties by index)
  for (int i = tid; i < n; i += nt) {
    const double li = *M.at(i, i);
    int rank = 0;
    for (int j = 0; j < n; ++j) {
      const double lj = *M.at(j, j);
      if (lj > li || (lj == li && j < i)) ++rank;
    }
    evals[rank] = li;
    for (int row = 0; row < n; ++row) evecs[(long long)row * n + rank] = VT[(long long)i * n + row];
  }
  if (tid == 0 && sweeps_out) *sweeps_out = sweep;
}

// A: the input matrix (n x n, ld n, global, read only); Ag: global scratch
// (n x n) for the matrix when its packed upper triangle does not fit shared memory
__global__ void __launch_bounds__(kJacobiThreads) jacobi_kernel(int n, int packed, const double* A,
                                                                double* Ag, double* VT,
                                                                double* evals, double* evecs,
                                                                int* sweeps_out) {
  extern __shared__ double js[];
  const int npair = ((n + 1) & ~1) / 2;
  double* cs = js;
  double* sn = cs + npair;
  int* pp = reinterpret_cast<int*>(sn + npair);
  int* qq = pp + npair;
  double* As = reinterpret_cast<double*>(qq + npair);  // 24 npair bytes in: 8-byte aligned
  if (packed) {
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
      const int i = e / n, j = e - i * n;
      if (i <= j) As[(i * (2 * n - i + 1)) / 2 + (j - i)] = A[e];
    }
    __syncthreads();
    jacobi_body<true>(SymMat<true>{As, n}, VT, evals, evecs, sweeps_out, cs, sn, pp, qq);
  } else {
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) Ag[e] = A[e];
    __syncthreads();
    jacobi_body<false>(SymMat<false>{Ag, n}, VT, evals, evecs, sweeps_out, cs, sn, pp, qq);
  }
}

// ---------------------------------------------------------------------------
// natural orbitals by subspace iteration
// ---------------------------------------------------------------------------
// In place on the p x p Gram matrix S (row stride ld): S = R^T R (Cholesky,
// R upper triangular), then S <- R^-T (lower triangular; the strict upper
// part zeroed).  One CTA; p <= kNatMaxP.  Returns status in *ok (0: not
// positive definite).
constexpr int kNatMaxP = 72;  // subspace width: up to 64 orbitals plus 8
__global__ void __launch_bounds__(256) chol_inv_kernel(int p, double* S, long long ld, int* ok) {
  __shared__ double R[kNatMaxP * (kNatMaxP + 1)];
  __shared__ int bad;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int lr = p + 1;
  for (int e = tid; e < p * p; e += nt) R[(e / p) * lr + e % p] = S[(long long)(e / p) * ld + e % p];
  if (tid == 0) bad = 0;
  __syncthreads();
  // right-looking Cholesky, upper factor in R (rows k: R[k][k..p))
  for (int k = 0; k < p; ++k) {
    if (tid == 0) {
      const double d = R[k * lr + k];
      if (!(d > 0.0)) bad = 1;
      R[k * lr + k] = d > 0.0 ? sqrt(d) : 1.0;
    }
    __syncthreads();
    const double rkk = R[k * lr + k];
    for (int j = k + 1 + tid; j < p; j += nt) R[k * lr + j] /= rkk;
    __syncthreads();
    for (int e = tid; e < (p - k - 1) * (p - k - 1); e += nt) {
      const int i = k + 1 + e / (p - k - 1), j = k + 1 + e % (p - k - 1);
      if (j >= i) R[i * lr + j] -= R[k * lr + i] * R[k * lr + j];
    }
    __syncthreads();
  }
  // R^-1 by back substitution, column by column (thread per column)
  for (int c = tid; c < p; c += nt) {
    // solve R x = e_c, x stored in column c of S's upper part (x_i = 0 for i > c)
    for (int i = p - 1; i >= 0; --i) {
      double v = (i == c) ? 1.0 : 0.0;
      if (i <= c)
        for (int j = i + 1; j <= c; ++j) v -= R[i * lr + j] * S[(long long)j * ld + c];
      S[(long long)i * ld + c] = i <= c ? v / R[i * lr + i] : 0.0;
    }
  }
  __syncthreads();
  // transpose in place: S <- (R^-1)^T (lower)
  for (int e = tid; e < p * p; e += nt) {
    const int i = e / p, j = e % p;
    if (i < j) {
      const double a = S[(long long)i * ld + j];
      S[(long long)j * ld + i] = a;
      S[(long long)i * ld + j] = 0.0;
    }
  }
  if (tid == 0) *ok = bad ? 0 : 1;
}

// residual of the Ritz pairs: res[c] = || (Z^T rho)[c] - theta_c Z^T[c] ||  for c < k
// (ZR = Z^T rho, ZT = Z^T, rows of length n, stride ld); one warp per row
__global__ void ritz_residual_kernel(int k, int n, long long ld, const double* ZR, const double* ZT,
                                     const double* theta, double* res) {
  const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (c >= k) return;
  double s = 0.0;
  for (int i = lane; i < n; i += 32) {
    const double r = ZR[(long long)c * ld + i] - theta[c] * ZT[(long long)c * ld + i];
    s += r * r;
  }
  s = warp_sum(s);
  if (lane == 0) res[c] = sqrt(s);
}

size_t jacobi_smem(int n, bool* packed) {
  const int npair = ((n + 1) & ~1) / 2;
  const size_t base = (size_t)npair * (2 * sizeof(double) + 2 * sizeof(int)) + 8;
  const size_t full = base + (size_t)packed_len(n) * sizeof(double);
  *packed = full <= 220 * 1024;
  return *packed ? full : base;
}

int vsplits(int n, int G, int* bsum) {
  const int tiles = ((n + CfgV0::BM - 1) / CfgV0::BM) * ((n + CfgV0::BN - 1) / CfgV0::BN);
  int want = (296 + tiles - 1) / tiles;
  if (want > G) want = G;
  if (want < 1) want = 1;
  const int per = (G + want - 1) / want;
  *bsum = per;
  return (G + per - 1) / per;
}

constexpr int kV1Split = 16;

// doubles of afq_expm's scratch: padded A, two Horner/squaring buffers, the norm
long long expm_work(int n) {
  const long long ld = even(n);
  return 3 * (long long)n * ld + 8;
}

}  // namespace
}  // namespace afq

using namespace afq;

extern "C" {

int afq_intermediates_workspace_size(int32_t norb, int32_t nchol, size_t* bytes) {
  if (!bytes) return AFQ_ERR_NULL;
  if (norb <= 0 || nchol <= 0 || norb > kJacobiMaxN) return AFQ_ERR_SHAPE;
  const long long nn = (long long)norb * norb, ld = even(norb);
  int bsum = 0;
  const int nz = vsplits(norb, nchol, &bsum);
  // v0 partials, v1 partials, h1_mod (2 spins), the exponential's scratch, and
  // (odd N) the Cholesky vectors with padded rows; the measurement set-up uses
  // the front of the same space
  long long d = even(nz * nn) + even((long long)kV1Split * nn) + even(2 * nn) + expm_work(norb);
  if (norb & 1) d += (long long)nchol * norb * ld;
  d += 64;
  *bytes = (size_t)d * sizeof(double);
  return AFQ_OK;
}

int afq_measurement_intermediates(int32_t norb, const int32_t nocc[2], int32_t nchol, int32_t trial_type,
                                  const double* const mo[2], double* h1, const double* chol,
                                  double* const rot_h1[2], double* const rot_chol[2], void* work,
                                  size_t work_bytes, void* stream) {
  if (!nocc || !mo || !h1 || !chol || !rot_h1 || !rot_chol || !work) return AFQ_ERR_NULL;
  if (trial_type != AFQ_TRIAL_RHF && trial_type != AFQ_TRIAL_UHF) return AFQ_ERR_ARG;
  const int ns = trial_type == AFQ_TRIAL_UHF ? 2 : 1;
  if (norb <= 0 || nchol <= 0) return AFQ_ERR_SHAPE;
  for (int s = 0; s < ns; ++s) {
    if (nocc[s] <= 0 || nocc[s] > norb) return AFQ_ERR_SHAPE;
    if (!mo[s] || !rot_h1[s] || !rot_chol[s]) return AFQ_ERR_NULL;
  }
  size_t need = 0;
  const int rc0 = afq_intermediates_workspace_size(norb, nchol, &need);
  if (rc0 != AFQ_OK) return rc0;
  if (work_bytes < need) return AFQ_ERR_WORKSPACE;
  if (!al16(work) || !al16(chol)) return AFQ_ERR_ALIGN;
  cudaStream_t st = as_stream(stream);
  const int n = norb;
  const long long ld = even(n), hs = (long long)n * ld;
  double* hrot = static_cast<double*>(work);  // 2 spins, row stride ld
  double* mot = hrot + 2 * hs;                // no x n per spin, row stride ld
  double* cholp = mot + 2 * hs;               // odd n: chol with padded rows
  const double* B = chol;
  if (n & 1) {
    if (copy2d((long long)nchol * n, n, chol, n, cholp, ld, st) != cudaSuccess) return AFQ_ERR_CUDA;
    B = cholp;
  }
  {
    ProfScope ps(K_MISC, st);
    sym_kernel<<<(int)((hs + 255) / 256), 256, 0, st>>>(n, h1, hrot, ld, ns == 2);
    if (cudaGetLastError() != cudaSuccess) return AFQ_ERR_CUDA;
  }
  for (int s = 0; s < ns; ++s) {
    const int no = nocc[s];
    double* mt = mot + s * hs;
    {
      ProfScope ps(K_MISC, st);
      transpose_kernel<<<(int)(((long long)n * no + 255) / 256), 256, 0, st>>>(n, no, mo[s], no, mt, ld);
      if (cudaGetLastError() != cudaSuccess) return AFQ_ERR_CUDA;
    }
    // rot_h1[s] = mo^T h (no x n)
    DgemmArgs a{};
    a.A = F64Operand{mt, ld, 0, 0, kUnsegS};
    a.B = F64Operand{hrot + s * hs, ld, 0, 0, kUnsegS};
    a.M = no;
    a.N = n;
    a.K = n;
    a.nbatch = 1;
    a.alpha = 1.0;
    a.C = rot_h1[s];
    a.ldc = n;
    if (dgemm<CfgS>(a, 1, st) != cudaSuccess) return AFQ_ERR_CUDA;
    // rot_chol[s][g] = mo^T L_g (no x n), batched over g
    DgemmArgs b{};
    b.A = F64Operand{mt, ld, 0, 0, kUnsegS};
    b.B = F64Operand{B, ld, (long long)n * ld, 0, kUnsegS};
    b.M = no;
    b.N = n;
    b.K = n;
    b.nbatch = nchol;
    b.alpha = 1.0;
    b.C = rot_chol[s];
    b.ldc = n;
    b.c_bs = (long long)no * n;
    if (dgemm<CfgS>(b, nchol, st) != cudaSuccess) return AFQ_ERR_CUDA;
  }
  return AFQ_OK;
}

int afq_expm(int32_t n, const double* A, double scale, double* out, void* work, size_t work_bytes,
             void* stream) {
  if (!A || !out || !work) return AFQ_ERR_NULL;
  if (n <= 0 || n > kJacobiMaxN) return AFQ_ERR_SHAPE;
  if (work_bytes < (size_t)expm_work(n) * sizeof(double)) return AFQ_ERR_WORKSPACE;
  if (!al16(work)) return AFQ_ERR_ALIGN;
  if (out == A) return AFQ_ERR_ARG;
  cudaStream_t st = as_stream(stream);
  const long long ld = even(n), ms = (long long)n * ld;
  double* Ap = static_cast<double*>(work);  // A with padded rows
  double* P = Ap + ms;
  double* Q = P + ms;
  double* nrm = Q + ms;
  const int blocks = (int)(((long long)n * n + 255) / 256);
  if (copy2d(n, n, A, n, Ap, ld, st) != cudaSuccess) return AFQ_ERR_CUDA;
  {
    ProfScope ps(K_MISC, st);
    norm1_kernel<<<1, 256, 0, st>>>(n, Ap, ld, nrm);
    if (cudaGetLastError() != cudaSuccess) return AFQ_ERR_CUDA;
  }
  double theta0 = 0.0;
  if (cudaMemcpyAsync(&theta0, nrm, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return AFQ_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return AFQ_ERR_CUDA;
  theta0 *= fabs(scale);
  if (!isfinite(theta0)) return AFQ_ERR_ARG;
  int s = 0;
  while (theta0 / ldexp(1.0, s) > 0.5 && s < 1000) ++s;
  const double theta = theta0 / ldexp(1.0, s);
  // smallest degree m with theta^(m+1)/(m+1)! e^theta <= 2^-53
  int m = 1;
  {
    double term = theta * theta / 2.0;  // theta^(m+1)/(m+1)! for m = 1
    while (m < 30 && term * exp(theta) > ldexp(1.0, -53)) {
      ++m;
      term *= theta / (m + 1);
    }
  }
  const double bscale = scale / ldexp(1.0, s);
  // Horner: P = I + B/m ; P <- I + B P / k for k = m-1 .. 1 ; B = bscale A
  {
    ProfScope ps(K_MISC, st);
    horner_init_kernel<<<blocks, 256, 0, st>>>(n, ld, Ap, bscale / m, P);
    if (cudaGetLastError() != cudaSuccess) return AFQ_ERR_CUDA;
  }
  double* cur = P;
  double* nxt = Q;
  for (int k = m - 1; k >= 1; --k) {
    if (square_gemm(n, ld, Ap, cur, bscale / k, 1.0, nxt, st) != cudaSuccess) return AFQ_ERR_CUDA;
    double* t = cur;
    cur = nxt;
    nxt = t;
  }
  // squaring
  for (int i = 0; i < s; ++i) {
    if (square_gemm(n, ld, cur, cur, 1.0, 0.0, nxt, st) != cudaSuccess) return AFQ_ERR_CUDA;
    double* t = cur;
    cur = nxt;
    nxt = t;
  }
  if (copy2d(n, n, cur, ld, out, n, st) != cudaSuccess) return AFQ_ERR_CUDA;
  return AFQ_OK;
}

int afq_propagation_intermediates(int32_t norb, int32_t nchol, int32_t walker_type, const double* h1,
                                  const double* rdm1, const double* chol, double h0, double dt,
                                  double* mf_shifts, double* h0_prop, double* exp_h1, void* work,
                                  size_t work_bytes, void* stream) {
  if (!h1 || !rdm1 || !chol || !mf_shifts || !h0_prop || !exp_h1 || !work) return AFQ_ERR_NULL;
  if (walker_type != AFQ_RESTRICTED && walker_type != AFQ_UNRESTRICTED) return AFQ_ERR_ARG;
  if (norb <= 0 || nchol <= 0 || norb > kJacobiMaxN) return AFQ_ERR_SHAPE;
  size_t need = 0;
  afq_intermediates_workspace_size(norb, nchol, &need);
  if (work_bytes < need) return AFQ_ERR_WORKSPACE;
  if (!al16(work) || !al16(chol)) return AFQ_ERR_ALIGN;
  cudaStream_t st = as_stream(stream);
  const int n = norb, G = nchol;
  const long long nn = (long long)n * n, ld = even(n);
  const int np = walker_type == AFQ_UNRESTRICTED ? 2 : 1;
  int bsum = 0;
  const int nz = vsplits(n, G, &bsum);
  double* v0p = static_cast<double*>(work);
  double* v1p = v0p + even(nz * nn);
  double* hm = v1p + even((long long)kV1Split * nn);
  double* ew = hm + even(2 * nn);  // the exponential's scratch
  double* cholp = ew + expm_work(n);
  const double* Bc = chol;
  if (n & 1) {
    if (copy2d((long long)G * n, n, chol, n, cholp, ld, st) != cudaSuccess) return AFQ_ERR_CUDA;
    Bc = cholp;
  }
  const int blocks = (int)((nn + 255) / 256);
  {
    ProfScope ps(K_MISC, st);
    // rdm1 is (2, n, n): rho = rdm1[0] + rdm1[1], formed in the exponential's scratch
    hmod_kernel<<<blocks, 256, 0, st>>>(nn, 1, rdm1, 1, nullptr, 0, nullptr, 0, 2.0, ew);
    mf_kernel<<<G, 256, 0, st>>>(nn, chol, ew, mf_shifts);
    h0prop_kernel<<<1, 256, 0, st>>>(G, mf_shifts, h0, h0_prop);
    const int gper = (G + kV1Split - 1) / kV1Split;
    v1_kernel<<<dim3((unsigned)((nn + 255) / 256), kV1Split), 256, 0, st>>>(nn, G, gper, chol,
                                                                             mf_shifts, v1p);
    if (cudaGetLastError() != cudaSuccess) return AFQ_ERR_CUDA;
  }
  // v0 partials: part[z] = sum_{g in z} L_g L_g
  {
    DgemmArgs a{};
    a.A = F64Operand{Bc, ld, (long long)n * ld, 0, kUnsegS};
    a.B = F64Operand{Bc, ld, (long long)n * ld, 0, kUnsegS};
    a.M = a.N = a.K = n;
    a.nbatch = G;
    a.bsum = bsum;
    a.alpha = 1.0;
    a.C = v0p;
    a.ldc = n;
    a.c_bs = nn;
    if (dgemm<CfgV0>(a, nz, st) != cudaSuccess) return AFQ_ERR_CUDA;
  }
  // h1_mod per spin, then exp(-dt/2 h1_mod)
  {
    ProfScope ps(K_MISC, st);
    hmod_kernel<<<blocks, 256, 0, st>>>(nn, np, h1, np == 1, v0p, nz, v1p, kV1Split, 1.0, hm);
    if (cudaGetLastError() != cudaSuccess) return AFQ_ERR_CUDA;
  }
  for (int s = 0; s < np; ++s) {
    const int rc = afq_expm(n, hm + s * nn, -0.5 * dt, exp_h1 + s * nn, ew,
                            (size_t)expm_work(n) * sizeof(double), stream);
    if (rc != AFQ_OK) return rc;
  }
  return AFQ_OK;
}

int afq_natural_orbitals_workspace_size(int32_t n, int32_t k, size_t* bytes) {
  if (!bytes) return AFQ_ERR_NULL;
  if (n <= 0 || k <= 0 || k > n || n > kJacobiMaxN || k + 8 > kNatMaxP) return AFQ_ERR_SHAPE;
  const long long ld = even(n);
  const int p = std::min(n, k + 8);
  const long long pp = even(p);
  // X^T, Y^T, Z^T (p x ld), small p x pp matrices (Gram / H, U, scratch for the
  // Ritz values and residuals), then either the padded rdm (odd n) or the
  // full-eigensolver fallback (values, vectors and its scratch)
  const long long nn2 = even((long long)n * n);
  long long d = 3 * p * ld + 4 * p * pp + 4 * pp + std::max((long long)n * ld, ld + nn2 + 2 * nn2 + 8) + 64;
  *bytes = (size_t)d * sizeof(double);
  return AFQ_OK;
}

int afq_natural_orbitals(int32_t n, int32_t k, const double* rdm, double* orbs, double* occ, void* work,
                         size_t work_bytes, void* stream) {
  if (!rdm || !orbs || !work) return AFQ_ERR_NULL;
  size_t need = 0;
  int rc = afq_natural_orbitals_workspace_size(n, k, &need);
  if (rc != AFQ_OK) return rc;
  if (work_bytes < need) return AFQ_ERR_WORKSPACE;
  if (!al16(work) || !al16(rdm)) return AFQ_ERR_ALIGN;
  cudaStream_t st = as_stream(stream);
  const long long ld = even(n);
  const int p = std::min(n, k + 8);
  const long long pp = even(p);
  double* XT = static_cast<double*>(work);  // p x ld
  double* YT = XT + p * ld;
  double* ZT = YT + p * ld;
  double* S = ZT + p * ld;   // p x pp
  double* U = S + p * pp;    // p x pp (eigenvectors of H as columns)
  double* H = U + p * pp;    // p x pp
  double* T2 = H + p * pp;   // p x pp
  double* theta = T2 + p * pp;
  double* res = theta + pp;
  int* ok = reinterpret_cast<int*>(res + pp);
  double* full = reinterpret_cast<double*>(ok) + 2 * pp;  // fallback scratch
  double* rho = full;        // rdm with padded rows when n is odd (inside the fallback space)
  const double* R = rdm;
  if (n & 1) {
    if (copy2d(n, n, rdm, n, rho, ld, st) != cudaSuccess) return AFQ_ERR_CUDA;
    R = rho;
  }
  // start: p deterministic Gaussian rows
  if (launch_normal(XT, (long long)p * ld, 0x5eedULL, 0, st) != cudaSuccess) return AFQ_ERR_CUDA;
  const int max_iter = 40;
  std::vector<double> hres(k), hth(p);
  int hok = 0;
  for (int it = 0; it < max_iter; ++it) {
    // Y^T = X^T rho ; orthonormalize: S = Y^T Y, S = R^-T, X^T = R^-T Y^T (twice: CholeskyQR2)
    if (gemm2<B_KMAJOR>(p, n, n, XT, ld, R, ld, 1.0, YT, ld, st) != cudaSuccess) return AFQ_ERR_CUDA;
    for (int pass = 0; pass < 2; ++pass) {
      double* src = pass == 0 ? YT : XT;
      double* dst = pass == 0 ? XT : YT;
      if (gemm2<B_NMAJOR>(p, p, n, src, ld, src, ld, 1.0, S, pp, st) != cudaSuccess) return AFQ_ERR_CUDA;
      chol_inv_kernel<<<1, 256, 0, st>>>(p, S, pp, ok);
      if (cudaGetLastError() != cudaSuccess) return AFQ_ERR_CUDA;
      if (gemm2<B_KMAJOR>(p, n, p, S, pp, src, ld, 1.0, dst, ld, st) != cudaSuccess) return AFQ_ERR_CUDA;
    }
    // Q^T in YT.  Rayleigh-Ritz: T^T = Q^T rho (in XT), H = Q^T T (p x p)
    if (gemm2<B_KMAJOR>(p, n, n, YT, ld, R, ld, 1.0, XT, ld, st) != cudaSuccess) return AFQ_ERR_CUDA;
    if (gemm2<B_NMAJOR>(p, p, n, YT, ld, XT, ld, 1.0, H, pp, st) != cudaSuccess) return AFQ_ERR_CUDA;
    if (pp != p) {  // the small eigensolver reads a dense p x p matrix
      if (copy2d(p, p, H, pp, T2, p, st) != cudaSuccess) return AFQ_ERR_CUDA;
    } else if (cudaMemcpyAsync(T2, H, sizeof(double) * p * p, cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
      return AFQ_ERR_CUDA;
    }
    bool packed = false;
    const size_t smem = jacobi_smem(p, &packed);
    if (!packed) return AFQ_ERR_SHAPE;
    if (cudaFuncSetAttribute(jacobi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
      return AFQ_ERR_CUDA;
    {
      ProfScope ps(K_MISC, st);
      // eigenvalues (descending) into theta, eigenvectors as columns of U (p x p, dense)
      jacobi_kernel<<<1, kJacobiThreads, smem, st>>>(p, 1, T2, nullptr, H, theta, U, nullptr);
      if (cudaGetLastError() != cudaSuccess) return AFQ_ERR_CUDA;
    }
    // Ritz vectors Z^T = U^T Q^T: U^T as the A operand (p x p): transpose U into S
    {
      ProfScope ps(K_MISC, st);
      transpose_kernel<<<(p * p + 255) / 256, 256, 0, st>>>(p, p, U, p, S, pp);
      if (cudaGetLastError() != cudaSuccess) return AFQ_ERR_CUDA;
    }
    if (gemm2<B_KMAJOR>(p, n, p, S, pp, YT, ld, 1.0, ZT, ld, st) != cudaSuccess) return AFQ_ERR_CUDA;
    // residuals of the first k: (Z^T rho) in XT
    if (gemm2<B_KMAJOR>(k, n, n, ZT, ld, R, ld, 1.0, XT, ld, st) != cudaSuccess) return AFQ_ERR_CUDA;
    {
      ProfScope ps(K_MISC, st);
      ritz_residual_kernel<<<(k + 7) / 8, 256, 0, st>>>(k, n, ld, XT, ZT, theta, res);
      if (cudaGetLastError() != cudaSuccess) return AFQ_ERR_CUDA;
    }
    if (cudaMemcpyAsync(hres.data(), res, sizeof(double) * k, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(hth.data(), theta, sizeof(double) * p, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(&hok, ok, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess)
      return AFQ_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return AFQ_ERR_CUDA;
    if (!hok) break;  // rank-deficient iterate: use the full eigensolver
    double scale = 0.0, worst = 0.0;
    for (int i = 0; i < p; ++i) scale = std::max(scale, fabs(hth[i]));
    for (int i = 0; i < k; ++i) worst = std::max(worst, hres[i]);
    if (worst <= 1e-13 * std::max(scale, 1e-300) * sqrt((double)n)) {
      // converged: orbitals = (Z^T)^T restricted to k columns, occupations theta[0..k)
      {
        ProfScope ps(K_MISC, st);
        transpose_kernel<<<(int)(((long long)k * n + 255) / 256), 256, 0, st>>>(k, n, ZT, ld, orbs, k);
        if (cudaGetLastError() != cudaSuccess) return AFQ_ERR_CUDA;
      }
      if (occ && cudaMemcpyAsync(occ, theta, sizeof(double) * k, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return AFQ_ERR_CUDA;
      return AFQ_OK;
    }
    // next iterate: X^T = Z^T (all p Ritz vectors)
    if (cudaMemcpyAsync(XT, ZT, sizeof(double) * p * ld, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
      return AFQ_ERR_CUDA;
  }
  // not converged (nearly equal occupations at the cut): the full eigensolver
  double* vals = full;  // n
  double* vecs = vals + ld;  // n x n
  double* jw = vecs + even((long long)n * n);  // its own scratch (16-byte aligned)
  rc = afq_eigh_desc(n, rdm, vals, vecs, jw, (size_t)(2 * even((long long)n * n) + 8) * sizeof(double),
                     stream);
  if (rc != AFQ_OK) return rc;
  if (copy2d(n, k, vecs, n, orbs, k, st) != cudaSuccess) return AFQ_ERR_CUDA;
  if (occ && cudaMemcpyAsync(occ, vals, sizeof(double) * k, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return AFQ_ERR_CUDA;
  return AFQ_OK;
}

int afq_eigh_desc(int32_t n, const double* A, double* evals, double* evecs, void* work,
                  size_t work_bytes, void* stream) {
  if (!A || !evals || !evecs || !work) return AFQ_ERR_NULL;
  if (n <= 0 || n > kJacobiMaxN) return AFQ_ERR_SHAPE;
  const long long nn = (long long)n * n;
  if (work_bytes < (size_t)(2 * even(nn) + 8) * sizeof(double)) return AFQ_ERR_WORKSPACE;
  if (!al16(work)) return AFQ_ERR_ALIGN;
  cudaStream_t st = as_stream(stream);
  double* Ag = static_cast<double*>(work);
  double* V = Ag + even(nn);
  int* sweeps = reinterpret_cast<int*>(V + even(nn));
  bool packed = false;
  const size_t smem = jacobi_smem(n, &packed);
  if (cudaFuncSetAttribute(jacobi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return AFQ_ERR_CUDA;
  ProfScope ps(K_MISC, st);
  jacobi_kernel<<<1, kJacobiThreads, smem, st>>>(n, packed ? 1 : 0, A, Ag, V, evals, evecs, sweeps);
  return cudaGetLastError() == cudaSuccess ? AFQ_OK : AFQ_ERR_CUDA;
}

}  // extern "C"
