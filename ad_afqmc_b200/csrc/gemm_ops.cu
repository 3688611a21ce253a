// FP64 dense contractions of the phaseless step and of the local energy.
//
//  force bias   fb[w,g]   = mult * sum_k Gpl[(w,c),k] * RCcat[g,k]
//               (wavefunctions.py:1102-1126, 1314-1329)
//  field prep   x~ = x - fs, fs = -sqrt(dt)(i fb - mf), shift/fb terms
//               (propagation.py:295-301)
//  VHS          VHS[w] = i sqrt(dt) sum_g x~[w,g] L_g   (propagation.py:196-203)
//  propagator   y = e^{-dt h/2} w; y += sum_n VHS^n y / n!; w' = e^{-dt h/2} y
//               (propagation.py:154-176, 206-229)
//  exchange     f[g,w] = rot_chol[g] Theta_w ; c = tr f ; x = sum f o f^T
//               fused: f lives only in registers/shared memory
//               (wavefunctions.py:1128-1174, 1331-1363)
#include "common.cuh"
#include "gemm_f64.cuh"
#include "ops.h"
#include "profile.cuh"

namespace afq {

namespace {

constexpr int kUnseg = 1 << 30;

using CfgBig = F64Cfg<4, 8, 4, 2>;   // 128 x 128, 8 warps
using CfgP32 = F64Cfg<2, 2, 2, 2>;   // 32 x 32,  4 warps
using CfgP80 = F64Cfg<5, 5, 1, 2>;   // 40 x 80,  2 warps
using CfgP120 = F64Cfg<5, 5, 1, 3>;  // 40 x 120, 3 warps
using CfgX80 = F64Cfg<5, 5, 3, 2>;   // 120 x 80,  6 warps (exchange)
using CfgX120 = F64Cfg<5, 5, 3, 3>;  // 120 x 120, 9 warps (exchange)
using CfgX160 = F64Cfg<4, 5, 4, 4>;  // 128 x 160, 16 warps (exchange, No > 60)

template <class Cfg>
cudaError_t set_smem(const void* fn, size_t bytes) {
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// ---------------------------------------------------------------------------
// force bias: C[z] (2W x G) = Gpl (2W x Kfb) * RCcat^T, K split over z
// ---------------------------------------------------------------------------
template <class Cfg>
__global__ void __launch_bounds__(Cfg::NT) fb_gemm_kernel(F64Operand A, F64Operand B, int M,
                                                          int N, int K, int kchunk, double* C,
                                                          long long ldc, long long zstride) {
  extern __shared__ double smem[];
  const int m0 = blockIdx.x * Cfg::BM, n0 = blockIdx.y * Cfg::BN, z = blockIdx.z;
  const int kb = z * kchunk, ke = min(K, kb + kchunk);
  double acc[Cfg::FM][Cfg::FN][2];
  f64_zero<Cfg>(acc);
  f64_mainloop<Cfg, B_NMAJOR>(acc, A, B, M, N, kb, ke, m0, n0, 0, false, smem);
  double* Cz = C + (long long)z * zstride;
  f64_foreach<Cfg>(acc, m0, n0, [&](int m, int n, double v0, double v1) {
    if (m < M) {
      if (n < N) Cz[(long long)m * ldc + n] = v0;
      if (n + 1 < N) Cz[(long long)m * ldc + n + 1] = v1;
    }
  });
}

// ---------------------------------------------------------------------------
// field preparation (one CTA per walker)
// ---------------------------------------------------------------------------
// one compiled copy for the solo and the grouped kernel (identical rounding)
// fbpart: split-K partial sums of the force bias, FP64 (FP64 path) or FP32
// (f32: the tensor-core path's FP32 accumulators, stored as they are)
__device__ __noinline__ void prep_body(int W, int G, long long Gpad, int splitk,
                                          const void* fbpart, int f32, double alpha, const double* fields,
                                          const double* mf, double sdt, double* xt, double* wscal,
                                          double* fb_out, int npc, bf16* xb0, bf16* xb1, bf16* xb2,
                                          long long ldxb, int w) {
  bf16* const xb[3] = {xb0, xb1, xb2};
  __shared__ double red[4 * 8];
  const int tid = threadIdx.x;
  const long long zs = 2LL * W * Gpad;
  double sr = 0, si = 0, br = 0, bi = 0;
  for (int g = tid; g < G; g += blockDim.x) {
    double fr = 0.0, fi = 0.0;
    if (f32) {
      const float* fp = static_cast<const float*>(fbpart);
      for (int z = 0; z < splitk; ++z) {
        fr += (double)fp[z * zs + (2LL * w) * Gpad + g];
        fi += (double)fp[z * zs + (2LL * w + 1) * Gpad + g];
      }
    } else {
      const double* dp = static_cast<const double*>(fbpart);
      for (int z = 0; z < splitk; ++z) {
        fr += dp[z * zs + (2LL * w) * Gpad + g];
        fi += dp[z * zs + (2LL * w + 1) * Gpad + g];
      }
    }
    fr *= alpha;
    fi *= alpha;
    if (fb_out) {
      fb_out[2 * ((long long)w * G + g)] = fr;
      fb_out[2 * ((long long)w * G + g) + 1] = fi;
    }
    if (fields) {
      const double mfr = mf[2 * g], mfi = mf[2 * g + 1];
      // field_shifts = -sqrt(dt) * (i*fb - mf_shifts)
      const double fsr = -sdt * (-fi - mfr);
      const double fsi = -sdt * (fr - mfi);
      const double x = fields[(long long)w * G + g];
      const double xr = x - fsr, xi = -fsi;  // shifted field
      sr += xr * mfr - xi * mfi;
      si += xr * mfi + xi * mfr;
      br += x * fsr - (fsr * fsr - fsi * fsi) / 2.0;
      bi += x * fsi - (2.0 * fsr * fsi) / 2.0;
      // VHS = i sqrt(dt) x~ L  ->  rows (w,0)=Re VHS, (w,1)=Im VHS
      if (xb0) {
        put_pieces(-sdt * xi, npc, xb, (2LL * w) * ldxb + g);
        put_pieces(sdt * xr, npc, xb, (2LL * w + 1) * ldxb + g);
      } else {
        xt[(2LL * w) * Gpad + g] = -sdt * xi;
        xt[(2LL * w + 1) * Gpad + g] = sdt * xr;
      }
    }
  }
  if (fields) {
    sr = block_sum(sr, red);
    si = block_sum(si, red + 8);
    br = block_sum(br, red + 16);
    bi = block_sum(bi, red + 24);
    if (tid == 0) {
      double* s = wscal + (long long)w * 16;
      s[0] = sr;
      s[1] = si;
      s[2] = br;
      s[3] = bi;
    }
  }
}

__global__ void __launch_bounds__(256) prep_kernel(int W, int G, long long Gpad, int splitk,
                                                   const void* fbpart, int f32, double alpha,
                                                   const double* fields, const double* mf,
                                                   double sdt, double* xt, double* wscal,
                                                   double* fb_out, int npc, bf16* xb0, bf16* xb1,
                                                   bf16* xb2, long long ldxb) {
  prep_body(W, G, Gpad, splitk, fbpart, f32, alpha, fields, mf, sdt, xt, wscal, fb_out, npc, xb0,
            xb1, xb2, ldxb, blockIdx.x);
}

__global__ void __launch_bounds__(256) prep_kernel_grouped(const PrepArgs* A, BlockMap m, int step) {
  int local;
  const PrepArgs& a = A[block_owner(m, blockIdx.x, local)];
  prep_body(a.W, a.G, a.Gpad, a.splitk, a.fbpart, a.f32, a.alpha, a.fields + (long long)step * a.field_step,
            a.mf, a.sdt, a.xt, a.wscal, nullptr, a.npc, a.xb[0], a.xb[1], a.xb[2], a.ldxb, local);
}

// ---------------------------------------------------------------------------
// VHS: C (2W x N*N) = Xt (2W x G) * chol (G x N*N), scattered to (W, N, 2Npad)
// ---------------------------------------------------------------------------
template <class Cfg>
__global__ void __launch_bounds__(Cfg::NT) vhs_gemm_kernel(F64Operand A, F64Operand B, int M,
                                                           int NN, int K, int N, long long Npad,
                                                           double* vhs) {
  extern __shared__ double smem[];
  const int m0 = blockIdx.x * Cfg::BM, n0 = blockIdx.y * Cfg::BN;
  double acc[Cfg::FM][Cfg::FN][2];
  f64_zero<Cfg>(acc);
  f64_mainloop<Cfg, B_KMAJOR>(acc, A, B, M, NN, 0, K, m0, n0, 0, false, smem);
  const long long ld = 2 * Npad;
  f64_foreach<Cfg>(acc, m0, n0, [&](int m, int n, double v0, double v1) {
    if (m >= M) return;
    const int w = m >> 1, c = m & 1;
    double* base = vhs + (long long)w * N * ld + c * Npad;
    if (n < NN) {
      const int p = n / N, r = n - p * N;
      base[(long long)p * ld + r] = v0;
    }
    if (n + 1 < NN) {
      const int p = (n + 1) / N, r = (n + 1) - p * N;
      base[(long long)p * ld + r] = v1;
    }
  });
}

// ---------------------------------------------------------------------------
// batched per-walker GEMM for the one-body half-steps and the Taylor chain
//   mode 0: out = A*B
//   mode 1: t = s*(A*B); out = t; acc = yin + t
//   mode 2: t = s*(A*B); out = t; acc += t
//   mode 3: t = s*(A*B);           acc += t
// nseg == 2 adds A2 * rot(B) (imaginary part of a complex A).
// ---------------------------------------------------------------------------
struct PropEpi {
  int mode;
  double scale;
  double* out;
  const double* yin;
  double* acc;
  long long ld, bstride;
};

template <class Cfg>
__global__ void __launch_bounds__(Cfg::NT) prop_gemm_kernel(F64Operand A1, F64Operand A2,
                                                            F64Operand B, int M, int N, int K,
                                                            int nseg, PropEpi e) {
  extern __shared__ double smem[];
  const int m0 = blockIdx.x * Cfg::BM, n0 = blockIdx.y * Cfg::BN, b = blockIdx.z;
  double acc[Cfg::FM][Cfg::FN][2];
  f64_zero<Cfg>(acc);
  f64_mainloop<Cfg, B_KMAJOR>(acc, A1, B, M, N, 0, K, m0, n0, b, false, smem);
  if (nseg == 2) f64_mainloop<Cfg, B_KMAJOR>(acc, A2, B, M, N, 0, K, m0, n0, b, true, smem);
  const long long boff = (long long)b * e.bstride;
  f64_foreach<Cfg>(acc, m0, n0, [&](int m, int n, double v0, double v1) {
    if (m >= M) return;
    const long long o = boff + (long long)m * e.ld + n;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      if (n + q >= N) break;
      const double v = q ? v1 : v0;
      if (e.mode == 0) {
        e.out[o + q] = v;
      } else {
        const double tv = v * e.scale;
        if (e.mode != 3) e.out[o + q] = tv;
        if (e.mode == 1)
          e.acc[o + q] = e.yin[o + q] + tv;
        else
          e.acc[o + q] += tv;
      }
    }
  });
}

// ---------------------------------------------------------------------------
// fused exchange: tile = gpt Cholesky vectors x wpt walkers
// ---------------------------------------------------------------------------
template <class Cfg>
__global__ void __launch_bounds__(Cfg::NT) exch_kernel(F64Operand A, F64Operand B, int G, int no,
                                                       int N, int W, int gpt, int wpt,
                                                       double* cout, double* excout) {
  extern __shared__ double smem[];
  const int mt = blockIdx.x, nt = blockIdx.y;
  const int g0 = mt * gpt, w0 = nt * wpt;
  const int gcount = min(gpt, G - g0), wcount = min(wpt, W - w0);
  const int m0 = g0 * no, n0 = w0 * 2 * no;
  const int M_lim = (g0 + gcount) * no, N_lim = (w0 + wcount) * 2 * no;
  double acc[Cfg::FM][Cfg::FN][2];
  f64_zero<Cfg>(acc);
  f64_mainloop<Cfg, B_KMAJOR>(acc, A, B, M_lim, N_lim, 0, N, m0, n0, 0, false, smem);

  constexpr int CS = Cfg::BN + 2;  // staged tile row stride (doubles)
  double* Ct = smem;
  double2* blk = reinterpret_cast<double2*>(smem + Cfg::BM * CS);
  f64_foreach<Cfg>(acc, 0, 0, [&](int m, int n, double v0, double v1) {
    *reinterpret_cast<double2*>(Ct + m * CS + n) = make_double2(v0, v1);
  });
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = Cfg::NT / 32;
  const int nblk = gcount * wcount;
  for (int bi = warp; bi < nblk; bi += nwarps) {
    const int gl = bi % gcount, wl = bi / gcount;
    const double* F = Ct + gl * no * CS + wl * 2 * no;
    double er = 0, ei = 0, cr = 0, ci = 0;
    for (int e = lane; e < no * no; e += 32) {
      const int i = e / no, j = e - (e / no) * no;
      const double2 fij = *reinterpret_cast<const double2*>(F + i * CS + 2 * j);
      const double2 fji = *reinterpret_cast<const double2*>(F + j * CS + 2 * i);
      er += fij.x * fji.x - fij.y * fji.y;
      ei += fij.x * fji.y + fij.y * fji.x;
      if (i == j) {
        cr += fij.x;
        ci += fij.y;
      }
    }
    er = warp_sum(er);
    ei = warp_sum(ei);
    cr = warp_sum(cr);
    ci = warp_sum(ci);
    if (lane == 0) {
      const long long co = 2 * ((long long)(w0 + wl) * G + g0 + gl);
      cout[co] = cr;
      cout[co + 1] = ci;
      blk[gl * wpt + wl] = make_double2(er, ei);
    }
  }
  __syncthreads();
  for (int wl = threadIdx.x; wl < wcount; wl += Cfg::NT) {
    double sx = 0, sy = 0;
    for (int gl = 0; gl < gcount; ++gl) {
      const double2 v = blk[gl * wpt + wl];
      sx += v.x;
      sy += v.y;
    }
    excout[2 * ((long long)mt * W + w0 + wl)] = sx;
    excout[2 * ((long long)mt * W + w0 + wl) + 1] = sy;
  }
}

// ---------------------------------------------------------------------------
// LNO orbital energy (rhf_lno._calc_orbenergy, wavefunctions.py:6904-6923):
// f = RC[g] . Theta_vir per (Cholesky vector, walker), Theta's occupied rows
// zeroed beforehand (so only rot_chol's virtual columns contribute), staged
// in shared memory as in the exchange.  With m = sum_r p_r^T p_r (prjlo rows
// p_r): c = tr f, s1 = sum_r p_r f p_r^T (= sum f o m), s2 = sum_r (p_r f).(f
// p_r^T) (= sum (f f) o m); the tile's partial sum_g (2 c s1 - s2) per walker.
// ---------------------------------------------------------------------------
constexpr int kMaxLo = 8;

template <class Cfg>
__global__ void __launch_bounds__(Cfg::NT) orb_kernel(F64Operand A, F64Operand B, int G, int no,
                                                      int N, int W, int gpt, int wpt,
                                                      const double* prj, int nlo, double* orbout) {
  extern __shared__ double smem[];
  const int mt = blockIdx.x, nt = blockIdx.y;
  const int g0 = mt * gpt, w0 = nt * wpt;
  const int gcount = min(gpt, G - g0), wcount = min(wpt, W - w0);
  const int m0 = g0 * no, n0 = w0 * 2 * no;
  const int M_lim = (g0 + gcount) * no, N_lim = (w0 + wcount) * 2 * no;
  double acc[Cfg::FM][Cfg::FN][2];
  f64_zero<Cfg>(acc);
  f64_mainloop<Cfg, B_KMAJOR>(acc, A, B, M_lim, N_lim, 0, N, m0, n0, 0, false, smem);

  constexpr int CS = Cfg::BN + 2;
  double* Ct = smem;
  double* P = smem + Cfg::BM * CS;  // nlo x no projector rows
  double2* blk = reinterpret_cast<double2*>(P + kMaxLo * 64);
  f64_foreach<Cfg>(acc, 0, 0, [&](int m, int n, double v0, double v1) {
    *reinterpret_cast<double2*>(Ct + m * CS + n) = make_double2(v0, v1);
  });
  for (int e = threadIdx.x; e < nlo * no; e += Cfg::NT) P[e] = prj[e];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = Cfg::NT / 32;
  const int nblk = gcount * wcount;
  for (int bi = warp; bi < nblk; bi += nwarps) {
    const int gl = bi % gcount, wl = bi / gcount;
    const double* F = Ct + gl * no * CS + wl * 2 * no;
    double cr = 0, ci = 0, ar = 0, ai = 0, br = 0, bi_ = 0;
    for (int k = lane; k < no; k += 32) {
      cr += F[k * CS + 2 * k];
      ci += F[k * CS + 2 * k + 1];
    }
    for (int r = 0; r < nlo; ++r) {
      const double* p = P + r * no;
      for (int k = lane; k < no; k += 32) {
        double ur = 0, ui = 0, vr = 0, vi = 0;  // u = (p f)[k], v = (f p^T)[k]
        for (int x = 0; x < no; ++x) {
          ur = fma(p[x], F[x * CS + 2 * k], ur);
          ui = fma(p[x], F[x * CS + 2 * k + 1], ui);
          vr = fma(F[k * CS + 2 * x], p[x], vr);
          vi = fma(F[k * CS + 2 * x + 1], p[x], vi);
        }
        ar = fma(ur, p[k], ar);
        ai = fma(ui, p[k], ai);
        br += ur * vr - ui * vi;
        bi_ += ur * vi + ui * vr;
      }
    }
    cr = warp_sum(cr);
    ci = warp_sum(ci);
    ar = warp_sum(ar);
    ai = warp_sum(ai);
    br = warp_sum(br);
    bi_ = warp_sum(bi_);
    if (lane == 0)  // 2 c s1 - s2
      blk[gl * wpt + wl] = make_double2(2.0 * (cr * ar - ci * ai) - br, 2.0 * (cr * ai + ci * ar) - bi_);
  }
  __syncthreads();
  for (int wl = threadIdx.x; wl < wcount; wl += Cfg::NT) {
    double sx = 0, sy = 0;
    for (int gl = 0; gl < gcount; ++gl) {
      const double2 v = blk[gl * wpt + wl];
      sx += v.x;
      sy += v.y;
    }
    orbout[2 * ((long long)mt * W + w0 + wl)] = sx;
    orbout[2 * ((long long)mt * W + w0 + wl) + 1] = sy;
  }
}

// Theta (W, N, No) complex: rows p < No set to zero (the occupied block)
__global__ void theta_zero_occ_kernel(double2* theta, int W, int N, int no) {
  const long long n = (long long)W * no * no;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const long long w = e / ((long long)no * no), r = e - w * no * no;
    theta[w * N * no + r] = make_double2(0.0, 0.0);
  }
}

// orbital energy per walker: sum of the row-tile partials (one warp per walker)
__global__ void orb_combine_kernel(int W, int mt, const double* part, double* out) {
  const int lane = threadIdx.x & 31;
  const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (w >= W) return;
  double xr = 0, xi = 0;
  for (int m = lane; m < mt; m += 32) {
    xr += part[2 * ((long long)m * W + w)];
    xi += part[2 * ((long long)m * W + w) + 1];
  }
  xr = warp_sum(xr);
  xi = warp_sum(xi);
  if (lane == 0) {
    out[2LL * w] = xr;
    out[2LL * w + 1] = xi;
  }
}

// ---------------------------------------------------------------------------
// local energy from the pieces (one warp per walker)
// ---------------------------------------------------------------------------
__global__ void energy_combine_kernel(int W, int G, int ns, int restricted, const double* scal,
                                      const double* c0, const double* c1, const double* x0,
                                      int mt0, const double* x1, int mt1, const double* wscal,
                                      double* eout, int eout_stride) {
  const int lane = threadIdx.x & 31;
  const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (w >= W) return;
  double jr = 0, ji = 0, xr = 0, xi = 0;
  for (int g = lane; g < G; g += 32) {
    double ar = c0[2 * ((long long)w * G + g)], ai = c0[2 * ((long long)w * G + g) + 1];
    if (ns == 2) {
      ar += c1[2 * ((long long)w * G + g)];
      ai += c1[2 * ((long long)w * G + g) + 1];
    }
    jr += ar * ar - ai * ai;
    ji += 2.0 * ar * ai;
  }
  for (int m = lane; m < mt0; m += 32) {
    xr += x0[2 * ((long long)m * W + w)];
    xi += x0[2 * ((long long)m * W + w) + 1];
  }
  if (ns == 2)
    for (int m = lane; m < mt1; m += 32) {
      xr += x1[2 * ((long long)m * W + w)];
      xi += x1[2 * ((long long)m * W + w) + 1];
    }
  jr = warp_sum(jr);
  ji = warp_sum(ji);
  xr = warp_sum(xr);
  xi = warp_sum(xi);
  if (lane == 0) {
    const double* s = wscal + (long long)w * 16;
    const double h0 = scal[0];
    double er, ei;
    if (restricted) {
      // 2 sum c^2 - exc + 2 E1 + h0
      er = 2.0 * jr - xr + 2.0 * s[8] + h0;
      ei = 2.0 * ji - xi + 2.0 * s[9];
    } else {
      // ((c_up + c_dn)^2 - exc_up - exc_dn) / 2 + E1_up + E1_dn + h0
      er = 0.5 * (jr - xr) + s[8] + s[10] + h0;
      ei = 0.5 * (ji - xi) + s[9] + s[11];
    }
    eout[(long long)w * eout_stride] = er;
    eout[(long long)w * eout_stride + 1] = ei;
  }
}

template <class Cfg>
cudaError_t run_prop(const F64Operand& A1, const F64Operand& A2, const F64Operand& B, int M,
                     int N, int K, int nseg, int batch, const PropEpi& e, cudaStream_t st) {
  cudaError_t err = set_smem<Cfg>((const void*)prop_gemm_kernel<Cfg>, Cfg::SMEM);
  if (err != cudaSuccess) return err;
  dim3 grid((M + Cfg::BM - 1) / Cfg::BM, (N + Cfg::BN - 1) / Cfg::BN, batch);
  ProfScope ps(K_PROP, st);
  prop_gemm_kernel<Cfg><<<grid, Cfg::NT, Cfg::SMEM, st>>>(A1, A2, B, M, N, K, nseg, e);
  return cudaGetLastError();
}

cudaError_t prop_gemm(const F64Operand& A1, const F64Operand& A2, const F64Operand& B, int M,
                      int N, int K, int nseg, int batch, const PropEpi& e, cudaStream_t st) {
  if (N <= 32) return run_prop<CfgP32>(A1, A2, B, M, N, K, nseg, batch, e, st);
  if (N <= 80) return run_prop<CfgP80>(A1, A2, B, M, N, K, nseg, batch, e, st);
  return run_prop<CfgP120>(A1, A2, B, M, N, K, nseg, batch, e, st);
}

}  // namespace

cudaError_t launch_fb_gemm(const Layout& L, const double* prep, double* work, cudaStream_t st) {
  using Cfg = CfgBig;
  const int M = 2 * L.W, N = L.G;
  const long long K = L.Kfb_used;
  F64Operand A{work + L.w_gpl, L.Kfb, 0, 0, kUnseg};
  F64Operand B{prep + L.p_rccat, L.Kfb, 0, 0, kUnseg};
  int kchunk = (int)((K + L.splitk - 1) / L.splitk);
  kchunk = (kchunk + Cfg::BK - 1) / Cfg::BK * Cfg::BK;
  cudaError_t err = set_smem<Cfg>((const void*)fb_gemm_kernel<Cfg>, Cfg::SMEM);
  if (err != cudaSuccess) return err;
  dim3 grid((M + Cfg::BM - 1) / Cfg::BM, (N + Cfg::BN - 1) / Cfg::BN, L.splitk);
  ProfScope ps(K_FB, st);
  fb_gemm_kernel<Cfg><<<grid, Cfg::NT, Cfg::SMEM, st>>>(A, B, M, N, (int)K, kchunk,
                                                        work + L.w_fbpart, L.Gpad,
                                                        2LL * L.W * L.Gpad);
  return cudaGetLastError();
}

cudaError_t launch_prep_grouped(const PrepArgs* args, const BlockMap& m, int step, cudaStream_t st) {
  ProfScope ps(K_PREP, st);
  prep_kernel_grouped<<<m.start[m.n], 256, 0, st>>>(args, m, step);
  return cudaGetLastError();
}

cudaError_t launch_prep(const Layout& L, const double* prep, double* work, const double* fields,
                        double dt, double* fb_out, cudaStream_t st) {
  ProfScope ps(K_PREP, st);
  bf16* xb[3] = {nullptr, nullptr, nullptr};
  if (L.mixed) piece_ptrs(work, L.v_xt, L.v_xt_ps, L.npc, xb);
  prep_kernel<<<L.W, 256, 0, st>>>(L.W, L.G, L.Gpad, L.splitk, work + L.w_fbpart, L.mixed ? 1 : 0,
                                   (double)L.mult, fields, prep + L.p_mf, sqrt(dt),
                                   work + L.w_xt, work + L.w_wscal, fb_out, L.npc, xb[0], xb[1],
                                   xb[2], L.Gb);
  return cudaGetLastError();
}

// Free propagation (propagation.py:338-376): VHS = i sqrt(dt) x L from the raw
// fields x, rows (w, 0) = Re = 0 and (w, 1) = Im = sqrt(dt) x of the VHS operand
__global__ void __launch_bounds__(256) free_fields_kernel(int G, long long Gpad, const double* fields,
                                                          double sdt, double* xt, int npc, bf16* xb0,
                                                          bf16* xb1, bf16* xb2, long long ldxb) {
  bf16* const xb[3] = {xb0, xb1, xb2};
  const int w = blockIdx.x;
  for (int g = threadIdx.x; g < G; g += blockDim.x) {
    const double x = fields[(long long)w * G + g];
    if (xb0) {
      put_pieces(0.0, npc, xb, (2LL * w) * ldxb + g);
      put_pieces(sdt * x, npc, xb, (2LL * w + 1) * ldxb + g);
    } else {
      xt[(2LL * w) * Gpad + g] = 0.0;
      xt[(2LL * w + 1) * Gpad + g] = sdt * x;
    }
  }
}

cudaError_t launch_free_fields(const Layout& L, double* work, const double* fields, double dt,
                               cudaStream_t st) {
  ProfScope ps(K_PREP, st);
  bf16* xb[3] = {nullptr, nullptr, nullptr};
  if (L.mixed) piece_ptrs(work, L.v_xt, L.v_xt_ps, L.npc, xb);
  free_fields_kernel<<<L.W, 256, 0, st>>>(L.G, L.Gpad, fields, sqrt(dt), work + L.w_xt, L.npc, xb[0],
                                          xb[1], xb[2], L.Gb);
  return cudaGetLastError();
}

cudaError_t launch_vhs_gemm(const Layout& L, const double* prep, double* work, cudaStream_t st) {
  using Cfg = CfgBig;
  const int M = 2 * L.W, NN = L.N * L.N, K = L.G;
  F64Operand A{work + L.w_xt, L.Gpad, 0, 0, kUnseg};
  F64Operand B{prep + L.p_chol, L.N2pad, 0, 0, kUnseg};
  cudaError_t err = set_smem<Cfg>((const void*)vhs_gemm_kernel<Cfg>, Cfg::SMEM);
  if (err != cudaSuccess) return err;
  dim3 grid((M + Cfg::BM - 1) / Cfg::BM, (NN + Cfg::BN - 1) / Cfg::BN);
  ProfScope ps(K_VHS, st);
  vhs_gemm_kernel<Cfg><<<grid, Cfg::NT, Cfg::SMEM, st>>>(A, B, M, NN, K, L.N, L.Npad,
                                                         work + L.w_vhs);
  return cudaGetLastError();
}

cudaError_t launch_propagate_walkers(const Layout& L, const double* prep, double* work,
                                     double* const walkers[2], int n_exp_terms,
                                     cudaStream_t st) {
  const int N = L.N;
  const long long vld = 2 * L.Npad;
  for (int s = 0; s < L.np; ++s) {
    const int nc = 2 * L.no[s];
    const long long bs = (long long)N * nc;
    double* wk = walkers[s];
    double* y = work + L.w_y;
    double* acc = work + L.w_acc;
    double* ta = work + L.w_ta;
    double* tb = work + L.w_tb;
    F64Operand E{prep + L.p_exph1[s], L.Npad, 0, 0, kUnseg};
    F64Operand Bw{wk, nc, bs, 0, kUnseg};
    PropEpi ep{0, 1.0, y, nullptr, nullptr, nc, bs};
    cudaError_t err = prop_gemm(E, E, Bw, N, nc, N, 1, L.W, ep, st);
    if (err != cudaSuccess) return err;
    const double* src = y;
    double* bufs[2] = {ta, tb};
    if (n_exp_terms <= 1) {
      F64Operand By{y, nc, bs, 0, kUnseg};
      PropEpi ef{0, 1.0, wk, nullptr, nullptr, nc, bs};
      err = prop_gemm(E, E, By, N, nc, N, 1, L.W, ef, st);
      if (err != cudaSuccess) return err;
      continue;
    }
    F64Operand Vr{work + L.w_vhs, vld, (long long)N * vld, 0, kUnseg};
    F64Operand Vi{work + L.w_vhs + L.Npad, vld, (long long)N * vld, 0, kUnseg};
    for (int n = 1; n < n_exp_terms; ++n) {
      F64Operand Bt{src, nc, bs, 0, kUnseg};
      double* dst = bufs[(n - 1) & 1];
      const int mode = (n == 1) ? 1 : ((n == n_exp_terms - 1) ? 3 : 2);
      PropEpi et{mode, 1.0 / n, dst, y, acc, nc, bs};
      if (n == 1 && n_exp_terms == 2) et.mode = 1;
      err = prop_gemm(Vr, Vi, Bt, N, nc, N, 2, L.W, et, st);
      if (err != cudaSuccess) return err;
      src = dst;
    }
    F64Operand Ba{acc, nc, bs, 0, kUnseg};
    PropEpi el{0, 1.0, wk, nullptr, nullptr, nc, bs};
    err = prop_gemm(E, E, Ba, N, nc, N, 1, L.W, el, st);
    if (err != cudaSuccess) return err;
  }
  return cudaSuccess;
}

template <class Cfg>
static cudaError_t run_exch(const Layout& L, const double* prep, double* work, int s,
                            cudaStream_t st) {
  const ExchTile& X = L.ex[s];
  const int no = L.no[s];
  F64Operand A{prep + L.p_rc[s], L.Npad, 0, 0, kUnseg};
  F64Operand B{work + L.w_theta[s], 2 * no, 0, (long long)L.N * 2 * no, 2 * no};
  const size_t stage = size_t(Cfg::BM) * (Cfg::BN + 2) * sizeof(double) +
                       size_t(X.gpt) * X.wpt * sizeof(double2);
  const size_t smem = stage > Cfg::SMEM ? stage : Cfg::SMEM;
  cudaError_t err = set_smem<Cfg>((const void*)exch_kernel<Cfg>, smem);
  if (err != cudaSuccess) return err;
  dim3 grid(X.mt, (L.W + X.wpt - 1) / X.wpt);
  ProfScope ps(K_EXCH, st);
  exch_kernel<Cfg><<<grid, Cfg::NT, smem, st>>>(A, B, L.G, no, L.N, L.W, X.gpt, X.wpt,
                                                work + L.w_c[s], work + L.w_exc[s]);
  return cudaGetLastError();
}

cudaError_t launch_exchange(const Layout& L, const double* prep, double* work, int s,
                            cudaStream_t st) {
  if (L.ex[s].bn == 80) return run_exch<CfgX80>(L, prep, work, s, st);
  if (L.ex[s].bn == 120) return run_exch<CfgX120>(L, prep, work, s, st);
  if (L.ex[s].bn == 160) return run_exch<CfgX160>(L, prep, work, s, st);
  return cudaErrorInvalidValue;
}

template <class Cfg>
static cudaError_t run_orb(const Layout& L, const double* prep, double* work, const double* prj,
                           int nlo, cudaStream_t st) {
  const ExchTile& X = L.ex[0];
  const int no = L.no[0];
  const int mt = (L.G + X.gpt - 1) / X.gpt;
  F64Operand A{prep + L.p_rc[0], L.Npad, 0, 0, kUnseg};
  F64Operand B{work + L.w_theta[0], 2 * no, 0, (long long)L.N * 2 * no, 2 * no};
  const size_t stage = size_t(Cfg::BM) * (Cfg::BN + 2) * sizeof(double) +
                       size_t(kMaxLo) * 64 * sizeof(double) + size_t(X.gpt) * X.wpt * sizeof(double2);
  const size_t smem = stage > Cfg::SMEM ? stage : Cfg::SMEM;
  cudaError_t err = set_smem<Cfg>((const void*)orb_kernel<Cfg>, smem);
  if (err != cudaSuccess) return err;
  dim3 grid(mt, (L.W + X.wpt - 1) / X.wpt);
  ProfScope ps(K_EXCH, st);
  orb_kernel<Cfg><<<grid, Cfg::NT, smem, st>>>(A, B, L.G, no, L.N, L.W, X.gpt, X.wpt, prj, nlo,
                                               work + L.w_orb);
  return cudaGetLastError();
}

cudaError_t launch_orbenergy(const Layout& L, const double* prep, double* work, const double* prj,
                             int nlo, double* out, cudaStream_t st) {
  if (nlo < 1 || nlo > kMaxLo || L.no[0] > 64) return cudaErrorInvalidValue;
  {
    ProfScope ps(K_MISC, st);
    theta_zero_occ_kernel<<<256, 256, 0, st>>>(reinterpret_cast<double2*>(work + L.w_theta[0]), L.W,
                                               L.N, L.no[0]);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (L.ex[0].bn == 80)
    e = run_orb<CfgX80>(L, prep, work, prj, nlo, st);
  else if (L.ex[0].bn == 120)
    e = run_orb<CfgX120>(L, prep, work, prj, nlo, st);
  else if (L.ex[0].bn == 160)
    e = run_orb<CfgX160>(L, prep, work, prj, nlo, st);
  else
    return cudaErrorInvalidValue;
  if (e != cudaSuccess) return e;
  const int wpb = 8;
  const int mt = (L.G + L.ex[0].gpt - 1) / L.ex[0].gpt;
  ProfScope ps(K_ECOMB, st);
  orb_combine_kernel<<<(L.W + wpb - 1) / wpb, 32 * wpb, 0, st>>>(L.W, mt, work + L.w_orb, out);
  return cudaGetLastError();
}

cudaError_t launch_energy_combine(const Layout& L, const double* prep, double* work, double* eout,
                                  int eout_stride, cudaStream_t st) {
  const int wpb = 8;
  ProfScope ps(K_ECOMB, st);
  energy_combine_kernel<<<(L.W + wpb - 1) / wpb, 32 * wpb, 0, st>>>(
      L.W, L.G, L.ns, L.restricted, prep + L.p_scal, work + L.w_c[0], L.ns == 2 ? work + L.w_c[1] : nullptr,
      work + L.w_exc[0], L.ex[0].mt, L.ns == 2 ? work + L.w_exc[1] : nullptr,
      L.ns == 2 ? L.ex[1].mt : 0, work + L.w_wscal, eout, eout_stride);
  return cudaGetLastError();
}

}  // namespace afq
