// Per-walker scalar and walker-matrix operations of the phaseless path:
//   phaseless weight update      propagation.py:302-335
//   Householder QR (orthonormalize)  linalg_utils.py:51-72 (LAPACK zgeqr2/zung2r)
//   comb reconfiguration         sr.py:24-48 (local), sr.py:52-153 (global, 1 rank)
//   block-end energy statistics  sampling.py:76-94
//   Gaussian auxiliary fields    Philox4x32-10 + Box-Muller (counter based)
#include "common.cuh"
#include "ops.h"
#include "profile.cuh"

namespace afq {

namespace {

// ---------------------------------------------------------------------------
// weight update (single CTA: needs the total weight for the population shift)
// ---------------------------------------------------------------------------
constexpr int kWeightThreads = 1024;

// one compiled copy for the solo and the grouped kernel (identical rounding)
__device__ __noinline__ void weight_body(int W, double dt, const double* scal, const double* wscal,
                                            double* weights, double* overlaps, double* scalars) {
  __shared__ double red[kWeightThreads / 32];
  const double sdt = sqrt(dt);
  const double h0r = scal[1], h0i = scal[2];
  const double est = scalars[0], pop = scalars[1];
  double tot = 0.0;
  for (int w = threadIdx.x; w < W; w += blockDim.x) {
    const double* s = wscal + (long long)w * 16;
    const double2 on = make_double2(s[12], s[13]);
    const double2 oo = make_double2(overlaps[2 * w], overlaps[2 * w + 1]);
    const double2 ratio = cdiv(on, oo);
    // imp = exp(-sqrt(dt) shift + fb_term + dt (pop + h0_prop)) * ratio
    const double ar = -sdt * s[0] + s[2] + dt * (pop + h0r);
    const double ai = -sdt * s[1] + s[3] + dt * h0i;
    const double ea = exp(ar);
    double sn, cs;
    sincos(ai, &sn, &cs);
    const double2 imp = cmul(make_double2(ea * cs, ea * sn), ratio);
    // theta = angle(exp(-sqrt(dt) shift) * ratio)
    const double eb = exp(-sdt * s[0]);
    double sb, cb;
    sincos(-sdt * s[1], &sb, &cb);
    const double2 z = cmul(make_double2(eb * cb, eb * sb), ratio);
    const double th = atan2(z.y, z.x);
    double ipl = hypot(imp.x, imp.y) * cos(th);
    if (isnan(ipl)) ipl = 0.0;
    if (ipl < 1.0e-3) ipl = 0.0;
    if (ipl > 100.0) ipl = 0.0;
    double wn = ipl * weights[w];
    if (wn > 100.0) wn = 0.0;
    weights[w] = wn;
    overlaps[2 * w] = on.x;
    overlaps[2 * w + 1] = on.y;
    tot += wn;
  }
  tot = block_sum(tot, red);
  if (threadIdx.x == 0) scalars[1] = est - 0.1 * log(tot / W) / dt;
}

__global__ void __launch_bounds__(kWeightThreads)
    weight_kernel(int W, double dt, const double* scal, const double* wscal, double* weights,
                  double* overlaps, double* scalars) {
  weight_body(W, dt, scal, wscal, weights, overlaps, scalars);
}

// one CTA per solve of a batch
__global__ void __launch_bounds__(kWeightThreads) weight_kernel_grouped(const WeightArgs* A) {
  const WeightArgs& a = A[blockIdx.x];
  weight_body(a.W, a.dt, a.scal, a.wscal, a.weights, a.overlaps, a.scalars);
}

// ---------------------------------------------------------------------------
// Householder QR, LAPACK convention (zlarfg: beta = -sign(Re a) |x|,
// tau = ((beta - ar)/beta, -ai/beta), v = x / (a - beta)), explicit Q as zung2r.
// A is a generic pointer (shared or global memory), row stride lda (double2).
//
// One warp per column: warp (j mod warps) owns column j for the whole
// factorisation.  Applying a reflector to a column is a warp-local product
// (w_j = v^H a_j by shuffles) and update, so each reflector costs one block
// barrier: in geqr2 the owner of column k + 1 forms the next reflector right
// after the column received reflector k; in zung2r the owner of column i + 1
// turns it into a column of Q just before applying reflector i to it (no
// other warp reads column i + 1 at that step, while column i, which every
// warp reads as the reflector, is left alone until the next step).
// ---------------------------------------------------------------------------
constexpr int kQrThreads = 1024;

__device__ __forceinline__ double2 warp_sum2(double2 v) {
  return make_double2(warp_sum(v.x), warp_sum(v.y));
}

// first column > k owned by this warp
__device__ __forceinline__ int qr_first_col(int k, int warp, int nw) {
  return k + 1 + ((warp - (k + 1)) % nw + nw) % nw;
}

// reflector of column k from its entries k..N-1 (zlarfg); owner warp only
__device__ void qr_reflector(double2* A, int lda, int N, int k, double2* tau, double* beta) {
  const int lane = threadIdx.x & 31;
  double s = 0.0;
  for (int p = k + 1 + lane; p < N; p += 32) {
    const double2 v = A[p * lda + k];
    s += v.x * v.x + v.y * v.y;
  }
  s = warp_sum(s);
  const double2 al = A[k * lda + k];
  double2 tk, sc;
  double b;
  if (s == 0.0 && al.y == 0.0) {
    tk = make_double2(0.0, 0.0);
    b = al.x;
    sc = make_double2(1.0, 0.0);
  } else {
    b = -copysign(sqrt(al.x * al.x + al.y * al.y + s), al.x);
    tk = make_double2((b - al.x) / b, -al.y / b);
    sc = cdiv(make_double2(1.0, 0.0), make_double2(al.x - b, al.y));
  }
  for (int p = k + 1 + lane; p < N; p += 32) A[p * lda + k] = cmul(A[p * lda + k], sc);
  __syncwarp();
  if (lane == 0) {
    tau[k] = tk;
    beta[k] = b;
    A[k * lda + k] = make_double2(b, 0.0);  // R's diagonal; v_k = 1 is implicit
  }
}

// a_j -= c v (v^H a_j) over rows k..N-1, v read from vk (v_k = 1 implicit
// when `unit`, else vk[k] itself); one warp
__device__ __forceinline__ void qr_apply(double2* A, int lda, int N, int k, int j, const double2* vk,
                                         int vstride, bool unit, double2 c) {
  const int lane = threadIdx.x & 31;
  double2 w = make_double2(0.0, 0.0);
  for (int p = k + lane; p < N; p += 32) {
    const double2 vp = (unit && p == k) ? make_double2(1.0, 0.0) : vk[p * vstride];
    w = cadd(w, cmul(cconj(vp), A[p * lda + j]));
  }
  const double2 cw = cmul(c, warp_sum2(w));
  for (int p = k + lane; p < N; p += 32) {
    const double2 vp = (unit && p == k) ? make_double2(1.0, 0.0) : vk[p * vstride];
    A[p * lda + j] = csub(A[p * lda + j], cmul(vp, cw));
  }
}

// column i of Q from reflector i stored in it: -tau v below, 1 - tau on and
// 0 above the diagonal; owner warp only
__device__ __forceinline__ void qr_q_column(double2* A, int lda, int N, int i, double2 ti) {
  const int lane = threadIdx.x & 31;
  for (int p = lane; p < N; p += 32)
    A[p * lda + i] = p < i ? make_double2(0.0, 0.0)
                           : (p == i ? make_double2(1.0 - ti.x, -ti.y)
                                     : cmul(make_double2(-ti.x, -ti.y), A[p * lda + i]));
}

__device__ void qr_inplace(double2* A, int lda, int N, int no, double2* tau, double* beta) {
  const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  // ---- geqr2: R above the diagonal, reflectors below ----------------------
  if (warp == 0) qr_reflector(A, lda, N, 0, tau, beta);
  __syncthreads();
  for (int k = 0; k + 1 < no; ++k) {
    const double2 ct = cconj(tau[k]);  // H^H applied from the left
    const bool active = ct.x != 0.0 || ct.y != 0.0;
    for (int j = qr_first_col(k, warp, nw); j < no; j += nw) {
      if (active) qr_apply(A, lda, N, k, j, A + k, lda, true, ct);
      if (j == k + 1) {
        __syncwarp();
        qr_reflector(A, lda, N, k + 1, tau, beta);
      }
    }
    __syncthreads();
  }
  // ---- zung2r: explicit Q, reflectors applied last to first ---------------
  for (int i = no - 2; i >= 0; --i) {
    const double2 ti = tau[i];
    const bool active = ti.x != 0.0 || ti.y != 0.0;
    for (int j = qr_first_col(i, warp, nw); j < no; j += nw) {
      if (j == i + 1) {
        qr_q_column(A, lda, N, j, tau[j]);
        __syncwarp();
      }
      if (active) qr_apply(A, lda, N, i, j, A + i, lda, true, ti);
    }
    __syncthreads();
  }
  if (warp == 0) qr_q_column(A, lda, N, 0, tau[0]);
  __syncthreads();
}

// ---- the same factorisation with each warp's column rows in registers ----
// Lane l holds rows r0 + l + 32 t (t < RPL) of the column it works on, where
// r0 is the reflector's first row; N <= 32 RPL.  All RPL loads of a column are
// in flight together and the product and update run on registers, so a
// column step costs one round of loads, the shuffles and one round of stores.
template <int RPL>
__device__ __forceinline__ void rcol_load(const double2* A, int lda, int N, int r0, int j,
                                          double2 (&a)[RPL]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int t = 0; t < RPL; ++t) {
    const int p = r0 + lane + 32 * t;
    a[t] = p < N ? A[p * lda + j] : make_double2(0.0, 0.0);
  }
}

template <int RPL>
__device__ __forceinline__ void rcol_store(double2* A, int lda, int N, int r0, int j,
                                           const double2 (&a)[RPL]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int t = 0; t < RPL; ++t) {
    const int p = r0 + lane + 32 * t;
    if (p < N) A[p * lda + j] = a[t];
  }
}

// a -= c v (v^H a); rows beyond N hold zeros in both
template <int RPL>
__device__ __forceinline__ void rcol_reflect(double2 (&a)[RPL], const double2 (&v)[RPL], double2 c) {
  double2 w0 = make_double2(0.0, 0.0), w1 = make_double2(0.0, 0.0);
#pragma unroll
  for (int t = 0; t < RPL; ++t) {
    if (t & 1)
      w1 = cadd(w1, cmul(cconj(v[t]), a[t]));
    else
      w0 = cadd(w0, cmul(cconj(v[t]), a[t]));
  }
  const double2 cw = cmul(c, warp_sum2(cadd(w0, w1)));
#pragma unroll
  for (int t = 0; t < RPL; ++t) a[t] = csub(a[t], cmul(v[t], cw));
}

// reflector k (zlarfg) of a column held from row k - d: pivot in lane d, t = 0
template <int RPL>
__device__ __forceinline__ void rcol_reflector(double2 (&a)[RPL], int d, int k, double2* tau,
                                               double* beta) {
  const int lane = threadIdx.x & 31;
  double s = 0.0;
#pragma unroll
  for (int t = 0; t < RPL; ++t)
    if (t > 0 || lane > d) s += a[t].x * a[t].x + a[t].y * a[t].y;
  s = warp_sum(s);
  const double2 al = make_double2(__shfl_sync(0xffffffffu, a[0].x, d), __shfl_sync(0xffffffffu, a[0].y, d));
  double2 tk, sc;
  double b;
  if (s == 0.0 && al.y == 0.0) {
    tk = make_double2(0.0, 0.0);
    b = al.x;
    sc = make_double2(1.0, 0.0);
  } else {
    b = -copysign(sqrt(al.x * al.x + al.y * al.y + s), al.x);
    tk = make_double2((b - al.x) / b, -al.y / b);
    sc = cdiv(make_double2(1.0, 0.0), make_double2(al.x - b, al.y));
  }
#pragma unroll
  for (int t = 0; t < RPL; ++t)
    if (t > 0 || lane > d) a[t] = cmul(a[t], sc);
  if (lane == d) a[0] = make_double2(b, 0.0);
  if (lane == 0) {
    tau[k] = tk;
    beta[k] = b;
  }
}

// the reflector's rows r0 + l + 32 t (v_r0 = 1) into registers
template <int RPL>
__device__ __forceinline__ void rcol_vector(const double2* A, int lda, int N, int r0,
                                            double2 (&v)[RPL]) {
  rcol_load<RPL>(A, lda, N, r0, r0, v);
  if ((threadIdx.x & 31) == 0) v[0] = make_double2(1.0, 0.0);
}

template <int RPL>
__device__ void qr_inplace_reg(double2* A, int lda, int N, int no, double2* tau, double* beta) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double2 v[RPL], a[RPL];
  // ---- geqr2 ----------------------------------------------------------------
  if (warp == 0) {
    rcol_load<RPL>(A, lda, N, 0, 0, a);
    rcol_reflector<RPL>(a, 0, 0, tau, beta);
    rcol_store<RPL>(A, lda, N, 0, 0, a);
  }
  __syncthreads();
  for (int k = 0; k + 1 < no; ++k) {
    const double2 ct = cconj(tau[k]);
    const bool active = ct.x != 0.0 || ct.y != 0.0;
    const int j0 = qr_first_col(k, warp, nw);
    if (j0 < no) {
      rcol_vector<RPL>(A, lda, N, k, v);
      for (int j = j0; j < no; j += nw) {
        rcol_load<RPL>(A, lda, N, k, j, a);
        if (active) rcol_reflect<RPL>(a, v, ct);
        if (j == k + 1) rcol_reflector<RPL>(a, 1, k + 1, tau, beta);
        rcol_store<RPL>(A, lda, N, k, j, a);
      }
    }
    __syncthreads();
  }
  // ---- zung2r ---------------------------------------------------------------
  for (int i = no - 2; i >= 0; --i) {
    const double2 ti = tau[i];
    const bool active = ti.x != 0.0 || ti.y != 0.0;
    const int j0 = qr_first_col(i, warp, nw);
    if (j0 < no) {
      rcol_vector<RPL>(A, lda, N, i, v);
      for (int j = j0; j < no; j += nw) {
        rcol_load<RPL>(A, lda, N, i, j, a);
        if (j == i + 1) {  // column j of Q from reflector j: window starts one row above it
          const double2 tj = tau[j];
#pragma unroll
          for (int t = 0; t < RPL; ++t) {
            if (t == 0 && lane == 0) a[t] = make_double2(0.0, 0.0);
            else if (t == 0 && lane == 1) a[t] = make_double2(1.0 - tj.x, -tj.y);
            else a[t] = cmul(make_double2(-tj.x, -tj.y), a[t]);
          }
          for (int p = lane; p < i; p += 32) A[p * lda + j] = make_double2(0.0, 0.0);
        }
        if (active) rcol_reflect<RPL>(a, v, ti);
        rcol_store<RPL>(A, lda, N, i, j, a);
      }
    }
    __syncthreads();
  }
  if (warp == 0) {  // column 0 of Q
    rcol_load<RPL>(A, lda, N, 0, 0, a);
    const double2 t0 = tau[0];
#pragma unroll
    for (int t = 0; t < RPL; ++t)
      a[t] = (t == 0 && lane == 0) ? make_double2(1.0 - t0.x, -t0.y) : cmul(make_double2(-t0.x, -t0.y), a[t]);
    rcol_store<RPL>(A, lda, N, 0, 0, a);
  }
  __syncthreads();
}

// grid (W, ns).  use_smem: walker copied to shared memory with row stride no+1.
// RPL > 0: register-resident columns (N <= 32 RPL, 512 threads); 0: the loop
// form for any N (1024 threads).
template <int RPL>
__device__ __forceinline__ void qr_walker(int N, int no0, int no1, double* w0, double* w1,
                                          int sign_fix, int use_smem, double* sector_norm) {
  extern __shared__ double2 qsm[];
  __shared__ double2 tau[64];
  __shared__ double beta[64];
  const int w = blockIdx.x, s = blockIdx.y;
  const int no = s ? no1 : no0;
  double2* G = reinterpret_cast<double2*>(s ? w1 : w0) + (long long)w * N * no;
  double2* A = G;
  int lda = no;
  if (use_smem) {
    lda = no + 1;
    A = qsm;
    for (int e = threadIdx.x; e < N * no; e += blockDim.x) {
      const int p = e / no, j = e - (e / no) * no;
      A[p * lda + j] = G[e];
    }
    __syncthreads();
  }
  if (RPL > 0)
    qr_inplace_reg<(RPL > 0 ? RPL : 1)>(A, lda, N, no, tau, beta);
  else
    qr_inplace(A, lda, N, no, tau, beta);
  // prod diag R (real) and optional sign fix of column 0
  __shared__ double prod_s;
  if (threadIdx.x == 0) {
    double pr = 1.0;
    for (int k = 0; k < no; ++k) pr *= beta[k];
    prod_s = pr;
    if (sector_norm) sector_norm[(long long)s * gridDim.x + w] = pr;
  }
  __syncthreads();
  const double sg = sign_fix ? ((prod_s > 0.0) ? 1.0 : ((prod_s < 0.0) ? -1.0 : 0.0)) : 1.0;
  if (use_smem) {
    for (int e = threadIdx.x; e < N * no; e += blockDim.x) {
      const int p = e / no, j = e - (e / no) * no;
      double2 v = A[p * lda + j];
      if (j == 0) v = cscale(v, sg);
      G[e] = v;
    }
  } else if (sign_fix) {
    for (int p = threadIdx.x; p < N; p += blockDim.x) G[p * no] = cscale(G[p * no], sg);
  }
}

constexpr int kQrRegThreads = 512;

__global__ void __launch_bounds__(kQrThreads, 1)
    qr_kernel(int N, int no0, int no1, double* w0, double* w1, int sign_fix, int use_smem,
              double* sector_norm /* (ns, W) */) {
  qr_walker<0>(N, no0, no1, w0, w1, sign_fix, use_smem, sector_norm);
}

template <int RPL>
__global__ void __launch_bounds__(kQrRegThreads, 1)
    qr_reg_kernel(int N, int no0, int no1, double* w0, double* w1, int sign_fix, int use_smem,
                  double* sector_norm /* (ns, W) */) {
  qr_walker<RPL>(N, no0, no1, w0, w1, sign_fix, use_smem, sector_norm);
}

__global__ void qr_norm_kernel(int W, int ns, int restricted, const double* sector_norm,
                               double* norms) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= W) return;
  double n;
  if (restricted)
    n = sector_norm[w];
  else
    n = fabs(sector_norm[w]) * (ns == 2 ? fabs(sector_norm[W + w]) : 1.0);
  norms[2 * w] = n;
  norms[2 * w + 1] = 0.0;
}

// ---------------------------------------------------------------------------
// comb reconfiguration (single CTA); bit-exact: serial cumsum, explicit
// round-to-nearest arithmetic in the reference's expression order.
// ---------------------------------------------------------------------------
// W slots over `ranks` ranks of W / ranks walkers each (ranks = 1 except for
// the reconfiguration across ranks, which combs the gathered weights)
__global__ void sr_kernel(int W, int ranks, const double* win, double zeta_host,
                          const double* zeta_dev, int mode, double* wout, int* idx) {
  extern __shared__ double cum[];
  const double zeta = zeta_dev ? *zeta_dev : zeta_host;
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < W; ++i) {
      s = __dadd_rn(s, fabs(win[i]));
      cum[i] = s;
    }
  }
  __syncthreads();
  const double total = cum[W - 1];
  const double dW = (double)W;
  const double dWr = (double)(W / ranks), dR = (double)ranks;  // per-rank count, ranks
  for (int i = threadIdx.x; i < W; i += blockDim.x) {
    double z;
    if (mode == AFQ_SR_LOCAL)
      z = __ddiv_rn(__dmul_rn(total, __dadd_rn((double)i, zeta)), dW);
    else  // (i + zeta) / nwalkers / size * total, nwalkers per rank
      z = __dmul_rn(__ddiv_rn(__ddiv_rn(__dadd_rn((double)i, zeta), dWr), dR), total);
    int lo = 0, hi = W;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (cum[mid] < z)
        lo = mid + 1;
      else
        hi = mid;
    }
    idx[i] = lo < W ? lo : W - 1;
    wout[i] = (mode == AFQ_SR_LOCAL) ? __ddiv_rn(total, dW) : __ddiv_rn(__ddiv_rn(total, dWr), dR);
  }
}

__global__ void gather_kernel(long long wd2, const double2* in, double2* out, const int* idx) {
  const int i = blockIdx.y;
  const double2* src = in + (long long)idx[i] * wd2;
  double2* dst = out + (long long)i * wd2;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < wd2;
       e += (long long)gridDim.x * blockDim.x)
    dst[e] = src[e];
}

// ---------------------------------------------------------------------------
// block end: clamp, block energy/weight, population-control shift, killed count
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024)
    block_end_kernel(int W, double dt, const double* wscal, const double* weights,
                     double* scalars, double* block_out) {
  __shared__ double red[3 * 32];
  const double est = scalars[0];
  const double thr = sqrt(2.0 / dt);
  double swe = 0.0, sw = 0.0, nz = 0.0;
  for (int w = threadIdx.x; w < W; w += blockDim.x) {
    double e = wscal[(long long)w * 16 + 14];
    if (fabs(e - est) > thr) e = est;
    const double wt = weights[w];
    swe += e * wt;
    sw += wt;
    nz += (wt != 0.0) ? 1.0 : 0.0;
  }
  swe = block_sum(swe, red);
  sw = block_sum(sw, red + 32);
  nz = block_sum(nz, red + 64);
  if (threadIdx.x == 0) {
    const double be = swe / sw;
    block_out[0] = be;
    block_out[1] = sw;
    scalars[1] = 0.9 * scalars[1] + 0.1 * be;
    scalars[2] += (double)W - nz;
  }
}

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) + Box-Muller
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint4 philox_round(uint4 c, uint2 k) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
  const uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
  return make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
}
__device__ __forceinline__ uint4 philox10(uint4 c, uint2 k) {
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    c = philox_round(c, k);
    k.x += W0;
    k.y += W1;
  }
  return c;
}
__device__ __forceinline__ double u53(uint32_t hi, uint32_t lo) {
  const unsigned long long x = ((unsigned long long)hi << 32) | lo;
  return ((double)(x >> 11) + 0.5) * 0x1.0p-53;  // in (0, 1)
}

__global__ void normal_kernel(double* out, long long n, unsigned long long seed,
                              unsigned long long offset) {
  const long long npair = (n + 1) / 2;
  const uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < npair;
       i += (long long)gridDim.x * blockDim.x) {
    const unsigned long long ctr = offset + (unsigned long long)i;
    const uint4 r = philox10(make_uint4((uint32_t)ctr, (uint32_t)(ctr >> 32), 0u, 0u), key);
    const double u1 = u53(r.x, r.y), u2 = u53(r.z, r.w);
    const double rad = sqrt(-2.0 * log(u1));
    double sn, cs;
    sincospi(2.0 * u2, &sn, &cs);
    out[2 * i] = rad * cs;
    if (2 * i + 1 < n) out[2 * i + 1] = rad * sn;
  }
}

// fields from the Philox stream at a device-resident counter; the counter
// then advances by the pairs consumed (graph replays draw fresh numbers)
__global__ void normal_dev_kernel(double* out, long long n, unsigned long long seed,
                                  const unsigned long long* counter) {
  const long long npair = (n + 1) / 2;
  const uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
  const unsigned long long base = *counter;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < npair;
       i += (long long)gridDim.x * blockDim.x) {
    const unsigned long long ctr = base + (unsigned long long)i;
    const uint4 r = philox10(make_uint4((uint32_t)ctr, (uint32_t)(ctr >> 32), 0u, 0u), key);
    const double u1 = u53(r.x, r.y), u2 = u53(r.z, r.w);
    const double rad = sqrt(-2.0 * log(u1));
    double sn, cs;
    sincospi(2.0 * u2, &sn, &cs);
    out[2 * i] = rad * cs;
    if (2 * i + 1 < n) out[2 * i + 1] = rad * sn;
  }
}

// one U(0,1) at the counter (third word of the Philox block: a stream
// disjoint from the normals), counter advanced by one; then the counter of the
// normals is advanced by `advance`
__global__ void uniform_dev_kernel(double* out, unsigned long long seed,
                                   unsigned long long* counter, unsigned long long advance) {
  const uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
  const unsigned long long ctr = *counter;
  if (out) {
    const uint4 r = philox10(make_uint4((uint32_t)ctr, (uint32_t)(ctr >> 32), 1u, 0u), key);
    *out = u53(r.x, r.y);
  }
  *counter = ctr + advance;
}

__global__ void set_scalars_kernel(double* dst, double a, double b, double c, double d) {
  dst[0] = a;
  dst[1] = b;
  dst[2] = c;
  dst[3] = d;
}

}  // namespace

cudaError_t launch_weight_update(const Layout& L, const double* prep, double* work,
                                 double* weights, double* overlaps, double* scalars, double dt,
                                 cudaStream_t st) {
  ProfScope ps(K_WEIGHT, st);
  weight_kernel<<<1, kWeightThreads, 0, st>>>(L.W, dt, prep + L.p_scal, work + L.w_wscal, weights,
                                              overlaps, scalars);
  return cudaGetLastError();
}

cudaError_t launch_weight_grouped(const WeightArgs* args, int n, cudaStream_t st) {
  ProfScope ps(K_WEIGHT, st);
  weight_kernel_grouped<<<n, kWeightThreads, 0, st>>>(args);
  return cudaGetLastError();
}

template <class K>
static cudaError_t launch_qr_kernel(K kernel, int threads, dim3 grid, size_t dyn, cudaStream_t st,
                                   const Layout& L, double* const walkers[2], int use_smem,
                                   double* secn) {
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
  if (e != cudaSuccess) return e;
  kernel<<<grid, threads, dyn, st>>>(L.N, L.no[0], L.no[1], walkers[0], L.ns == 2 ? walkers[1] : nullptr,
                                     L.restricted ? 0 : 1, use_smem, secn);
  return cudaGetLastError();
}

cudaError_t launch_qr(const Layout& L, double* const walkers[2], double* norms, double* work,
                      cudaStream_t st) {
  const size_t smem = size_t(L.N) * (L.nomax + 1) * sizeof(double2);
  const int use_smem = smem <= 200 * 1024 && L.tune.qr_mode != 2;
  const size_t dyn = use_smem ? smem : 0;
  double* secn = work;  // (ns, W) doubles of scratch at the start of the workspace
  dim3 grid(L.W, L.ns);
  cudaError_t e;
  {
    ProfScope ps(K_QR, st);
    const int N = L.N, T = kQrRegThreads;
    if (N <= 32)
      e = launch_qr_kernel(qr_reg_kernel<1>, T, grid, dyn, st, L, walkers, use_smem, secn);
    else if (N <= 64)
      e = launch_qr_kernel(qr_reg_kernel<2>, T, grid, dyn, st, L, walkers, use_smem, secn);
    else if (N <= 128)
      e = launch_qr_kernel(qr_reg_kernel<4>, T, grid, dyn, st, L, walkers, use_smem, secn);
    else if (N <= 224)
      e = launch_qr_kernel(qr_reg_kernel<7>, T, grid, dyn, st, L, walkers, use_smem, secn);
    else if (N <= 320)
      e = launch_qr_kernel(qr_reg_kernel<10>, T, grid, dyn, st, L, walkers, use_smem, secn);
    else
      e = launch_qr_kernel(qr_kernel, kQrThreads, grid, dyn, st, L, walkers, use_smem, secn);
  }
  if (e != cudaSuccess || !norms) return e;
  ProfScope ps(K_MISC, st);
  qr_norm_kernel<<<(L.W + 255) / 256, 256, 0, st>>>(L.W, L.ns, L.restricted, secn, norms);
  return cudaGetLastError();
}

cudaError_t launch_sr(int W, int ranks, const double* weights_in, double zeta,
                      const double* zeta_dev, int mode, double* weights_out, int* indices,
                      cudaStream_t st) {
  const size_t smem = size_t(W) * sizeof(double);
  cudaError_t e =
      cudaFuncSetAttribute(sr_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  ProfScope ps(K_SR, st);
  sr_kernel<<<1, 1024, smem, st>>>(W, ranks, weights_in, zeta, zeta_dev, mode, weights_out,
                                   indices);
  return cudaGetLastError();
}

cudaError_t launch_gather(int W, long long walker_doubles, const double* in, double* out,
                          const int* indices, cudaStream_t st) {
  const long long wd2 = walker_doubles / 2;
  int bx = (int)((wd2 + 255) / 256);
  if (bx > 64) bx = 64;
  dim3 grid(bx, W);
  ProfScope ps(K_GATHER, st);
  gather_kernel<<<grid, 256, 0, st>>>(wd2, reinterpret_cast<const double2*>(in),
                                      reinterpret_cast<double2*>(out), indices);
  return cudaGetLastError();
}

cudaError_t launch_block_end(const Layout& L, double* work, const double* weights,
                             double* scalars, double dt, double* block_out, cudaStream_t st) {
  ProfScope ps(K_BLOCKEND, st);
  block_end_kernel<<<1, 1024, 0, st>>>(L.W, dt, work + L.w_wscal, weights, scalars, block_out);
  return cudaGetLastError();
}

cudaError_t launch_normal(double* out, long long n, unsigned long long seed,
                          unsigned long long offset, cudaStream_t st) {
  const long long npair = (n + 1) / 2;
  long long blocks = (npair + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks < 1) blocks = 1;
  ProfScope ps(K_NORMAL, st);
  normal_kernel<<<(int)blocks, 256, 0, st>>>(out, n, seed, offset);
  return cudaGetLastError();
}

cudaError_t launch_normal_dev(double* out, long long n, unsigned long long seed,
                              unsigned long long* counter, cudaStream_t st) {
  const long long npair = (n + 1) / 2;
  long long blocks = (npair + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks < 1) blocks = 1;
  {
    ProfScope ps(K_NORMAL, st);
    normal_dev_kernel<<<(int)blocks, 256, 0, st>>>(out, n, seed, counter);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  ProfScope ps(K_MISC, st);
  uniform_dev_kernel<<<1, 1, 0, st>>>(nullptr, seed, counter, (unsigned long long)npair);
  return cudaGetLastError();
}

cudaError_t launch_uniform_dev(double* out, unsigned long long seed, unsigned long long* counter,
                               cudaStream_t st) {
  ProfScope ps(K_MISC, st);
  uniform_dev_kernel<<<1, 1, 0, st>>>(out, seed, counter, 1ull);
  return cudaGetLastError();
}

cudaError_t launch_set_scalars(double* dst, double a, double b, double c, double d,
                               cudaStream_t st) {
  ProfScope ps(K_MISC, st);
  set_scalars_kernel<<<1, 1, 0, st>>>(dst, a, b, c, d);
  return cudaGetLastError();
}

}  // namespace afq
