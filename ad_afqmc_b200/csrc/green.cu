// Overlap, half-rotated Green's function and one-body energy per walker.
//
// One CTA per (walker, spin sector).  For a walker W (N x No, complex) and
// a real trial C (N x No):
//   S     = C^T W                       (No x No)
//   det S , S^-1  by in-place Gauss-Jordan with partial pivoting
//            (pivot = first max of |re|+|im|, as LAPACK izamax)
//   Theta = W S^-1                      (N x No)  -> energy operand
//   G     = Theta^T                     (No x N)  -> force-bias operand
//   E1    = sum_ij G[i,j] rot_h1[i,j]
// Follows rhf._calc_green (wavefunctions.py:1089-1100), uhf._calc_green
// (:1289-1312), rhf/uhf overlaps (:1064-1074, :1259-1268) and the one-body
// part of the energies (:1128-1174, :1331-1363).  All arithmetic is FP64.
#include "common.cuh"
#include "ops.h"
#include "profile.cuh"

namespace afq {

namespace {

constexpr int kGreenThreads = 256;
constexpr int kRowChunk = 32;

__global__ void __launch_bounds__(kGreenThreads) green_kernel(GreenArgs a) {
  extern __shared__ double2 sm[];
  const int w = blockIdx.x, sct = blockIdx.y;
  const GreenSector& S_ = a.sec[sct];
  const int N = a.N, no = S_.no, tid = threadIdx.x;
  constexpr int T = kGreenThreads;

  double2* S = sm;                          // no*no
  double2* colk = S + no * no;              // 64
  double2* stage = colk + 64;               // kRowChunk*no   (walker rows, C^T W phase)
  double* moc = reinterpret_cast<double*>(stage + kRowChunk * no);  // kRowChunk*no
  double2* tstage = reinterpret_cast<double2*>(moc + kRowChunk * no);  // kRowChunk*(no+1)
  const int ts = no + 1;  // padded row stride of tstage (conflict-free column reads)
  __shared__ double red[2 * (T / 32)];
  __shared__ int perm[64];
  __shared__ int piv_s;

  const double2* Wg =
      reinterpret_cast<const double2*>(S_.walk) + (long long)w * N * no;

  // ---- S = C^T W -----------------------------------------------------------
  const int npairs = no * no;
  double2 acc[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) acc[q] = make_double2(0.0, 0.0);
  for (int p0 = 0; p0 < N; p0 += kRowChunk) {
    const int rows = min(kRowChunk, N - p0);
    for (int e = tid; e < rows * no; e += T) {
      stage[e] = Wg[(long long)p0 * no + e];
      moc[e] = S_.mo[(long long)p0 * no + e];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int pr = tid + q * T;
      if (pr < npairs) {
        const int i = pr / no, j = pr - (pr / no) * no;
        double2 s = acc[q];
        for (int r = 0; r < rows; ++r) {
          const double c = moc[r * no + i];
          const double2 x = stage[r * no + j];
          s.x = fma(c, x.x, s.x);
          s.y = fma(c, x.y, s.y);
        }
        acc[q] = s;
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    const int pr = tid + q * T;
    if (pr < npairs) S[pr] = acc[q];
  }
  __syncthreads();

  // ---- Gauss-Jordan inverse with partial pivoting, det ----------------------
  double2 det = make_double2(1.0, 0.0);
  for (int k = 0; k < no; ++k) {
    if (tid < 32) {
      double best = -1.0;
      int bi = k;
      for (int r = k + tid; r < no; r += 32) {
        const double2 v = S[r * no + k];
        const double m = fabs(v.x) + fabs(v.y);
        if (m > best) { best = m; bi = r; }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
      }
      if (tid == 0) { piv_s = bi; perm[k] = bi; }
    }
    __syncthreads();
    const int pv = piv_s;
    if (pv != k) {
      for (int j = tid; j < no; j += T) {
        const double2 t0 = S[k * no + j];
        S[k * no + j] = S[pv * no + j];
        S[pv * no + j] = t0;
      }
    }
    __syncthreads();
    const double2 pk = S[k * no + k];
    const double2 ipk = cdiv(make_double2(1.0, 0.0), pk);
    for (int i = tid; i < no; i += T) colk[i] = S[i * no + k];
    if (tid == 0) {
      det = cmul(det, pk);
      if (pv != k) det = make_double2(-det.x, -det.y);
    }
    __syncthreads();
    for (int j = tid; j < no; j += T) S[k * no + j] = (j == k) ? ipk : cmul(S[k * no + j], ipk);
    __syncthreads();
    for (int e = tid; e < npairs; e += T) {
      const int i = e / no, j = e - (e / no) * no;
      if (i == k) continue;
      const double2 f = colk[i];
      if (j == k) {
        const double2 t0 = cmul(f, ipk);
        S[e] = make_double2(-t0.x, -t0.y);
      } else {
        S[e] = csub(S[e], cmul(f, S[k * no + j]));
      }
    }
    __syncthreads();
  }
  for (int k = no - 1; k >= 0; --k) {
    const int pv = perm[k];
    if (pv != k) {
      for (int i = tid; i < no; i += T) {
        const double2 t0 = S[i * no + k];
        S[i * no + k] = S[i * no + pv];
        S[i * no + pv] = t0;
      }
    }
    __syncthreads();
  }
  if (tid == 0 && a.wscal) {
    a.wscal[(long long)w * 16 + 4 + 2 * sct] = det.x;
    a.wscal[(long long)w * 16 + 5 + 2 * sct] = det.y;
  }

  const bool need_theta = S_.theta || S_.gout || a.gpl || S_.rh1 || a.gplb[0] || S_.gtb[0];
  if (!need_theta) return;

  // ---- Theta = W S^-1, transposed copies, E1 --------------------------------
  double2 e1 = make_double2(0.0, 0.0);
  double2* th = S_.theta ? reinterpret_cast<double2*>(S_.theta) + (long long)w * N * no : nullptr;
  double2* go = S_.gout ? reinterpret_cast<double2*>(S_.gout) + (long long)w * no * N : nullptr;
  double* gre = a.gpl ? a.gpl + (2LL * w) * a.ldg + S_.koff : nullptr;
  double* gim = a.gpl ? a.gpl + (2LL * w + 1) * a.ldg + S_.koff : nullptr;
  const bool gb = a.gplb[0] != nullptr;
  const bool tb = S_.gtb[0] != nullptr;
  for (int p0 = 0; p0 < N; p0 += kRowChunk) {
    const int rows = min(kRowChunk, N - p0);
    // walker rows of this chunk into shared memory
    for (int e = tid; e < rows * no; e += T) stage[e] = Wg[(long long)p0 * no + e];
    __syncthreads();
    for (int e = tid; e < rows * no; e += T) {
      const int r = e / no, j = e - (e / no) * no;
      const double2* wrow = stage + r * no;
      double2 s = make_double2(0.0, 0.0);
      for (int i = 0; i < no; ++i) {
        const double2 x = wrow[i];
        const double2 y = S[i * no + j];
        s.x = fma(x.x, y.x, fma(-x.y, y.y, s.x));
        s.y = fma(x.x, y.y, fma(x.y, y.x, s.y));
      }
      tstage[r * ts + j] = s;
      if (th) th[(long long)(p0 + r) * no + j] = s;
      if (S_.rh1) {
        const double h = S_.rh1[(long long)j * N + p0 + r];
        e1.x = fma(s.x, h, e1.x);
        e1.y = fma(s.y, h, e1.y);
      }
    }
    __syncthreads();
    if (go || gre || gb || tb) {
      for (int e = tid; e < rows * no; e += T) {
        const int j = e / rows, r = e - (e / rows) * rows;
        const double2 v = tstage[r * ts + j];
        if (go) go[(long long)j * N + p0 + r] = v;
        if (gre) {
          gre[(long long)j * N + p0 + r] = v.x;
          gim[(long long)j * N + p0 + r] = v.y;
        }
        if (gb) {
          const long long o = S_.koff + (long long)j * N + p0 + r;
          put_pieces(v.x, a.npc, a.gplb, (2LL * w) * a.ldgb + o);
          put_pieces(v.y, a.npc, a.gplb, (2LL * w + 1) * a.ldgb + o);
        }
        if (tb) {
          const long long rr = (long long)w * 2 * no + 2 * j;
          put_pieces(v.x, a.npc, S_.gtb, rr * S_.ldtb + p0 + r);
          put_pieces(v.y, a.npc, S_.gtb, (rr + 1) * S_.ldtb + p0 + r);
        }
      }
    }
    __syncthreads();
  }
  if (S_.rh1 && a.wscal) {
    const double ex = block_sum(e1.x, red);
    const double ey = block_sum(e1.y, red + T / 32);
    if (tid == 0) {
      a.wscal[(long long)w * 16 + 8 + 2 * sct] = ex;
      a.wscal[(long long)w * 16 + 9 + 2 * sct] = ey;
    }
  }
}

__global__ void ovlp_combine_kernel(int W, int ns, int mult, const double* wscal, double* out,
                                    int out_stride) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= W) return;
  const double2 d0 = make_double2(wscal[(long long)w * 16 + 4], wscal[(long long)w * 16 + 5]);
  double2 o;
  if (ns == 1) {
    o = (mult == 2) ? cmul(d0, d0) : d0;
  } else {
    const double2 d1 = make_double2(wscal[(long long)w * 16 + 6], wscal[(long long)w * 16 + 7]);
    o = cmul(d0, d1);
  }
  out[(long long)w * out_stride] = o.x;
  out[(long long)w * out_stride + 1] = o.y;
}

}  // namespace

cudaError_t launch_green(const GreenArgs& a, cudaStream_t st) {
  int nomax = 0;
  for (int s = 0; s < a.ns; ++s) nomax = a.sec[s].no > nomax ? a.sec[s].no : nomax;
  const size_t smem = (size_t(nomax) * nomax + 64 + kRowChunk * nomax) * sizeof(double2) +
                      size_t(kRowChunk) * nomax * sizeof(double) +
                      size_t(kRowChunk) * (nomax + 1) * sizeof(double2);
  cudaError_t e = cudaFuncSetAttribute(green_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid(a.W, a.ns);
  ProfScope ps(K_GREEN, st);
  green_kernel<<<grid, kGreenThreads, smem, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_ovlp_combine(int W, int ns, int mult, const double* wscal, double* out,
                                int out_stride, cudaStream_t st) {
  ProfScope ps(K_MISC, st);
  ovlp_combine_kernel<<<(W + 255) / 256, 256, 0, st>>>(W, ns, mult, wscal, out, out_stride);
  return cudaGetLastError();
}

}  // namespace afq
