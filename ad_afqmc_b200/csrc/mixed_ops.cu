// Mixed-precision (tensor-core) contractions of the phaseless step.
//
// Each FP64 contraction of the step has a tcgen05 counterpart built on the
// persistent split-BF16 GEMM (umma_gemm.cuh).  Operands are stored as two
// (AFQ_MIXED) or three (AFQ_MIXED_HI) bf16 pieces; accumulation is FP32 in
// TMEM.  Everything that decides walker survival stays FP64: Green's
// functions, determinants, QR, weights and energy accumulation.
//
//   force bias   C (2W x G)  = Gpl (2W x K) . RCcat (G x K)^T, split over K
//                (wavefunctions.py:1102-1126, 1314-1329)
//   VHS          C (N^2 x 2W) = cholT (N^2 x G) . Xt (2W x G)^T
//                written straight into the propagator's A operand pieces
//                (propagation.py:196-203)
//   propagator   per walker:  y = e^{-dt h/2} w ; t_n = VHS t_{n-1} / n ;
//                w' = e^{-dt h/2} (y + sum t_n)   (propagation.py:154-176)
//                iterates live as transposed bf16 pieces [t^T | (i t)^T] so
//                that VHS (complex) times t is one real GEMM with K = 2N
//   exchange     f = RC . Theta per (Cholesky vector, walker) tile, reduced
//                in the epilogue to tr f and sum f o f^T; f never leaves the SM
//                (wavefunctions.py:1128-1174, 1331-1363)
#include <cuda.h>

#include <cstring>
#include <vector>

#include "afqmc_b200.h"
#include "common.cuh"
#include "ops.h"
#include "profile.cuh"
#include "umma_gemm.cuh"

namespace afq {

int make_tmap_bf16(CUtensorMap* map, const void* base, long long K, long long rows,
                   long long batch, long long row_stride_elems, long long batch_stride_elems,
                   int box_rows);
int sm_count();

namespace {

__device__ __forceinline__ void named_sync_epi() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

inline int pairs_for(int npc, int* pa, int* pb) {
  if (npc == 2) {
    const int a[3] = {0, 0, 1}, b[3] = {0, 1, 0};
    for (int i = 0; i < 3; ++i) { pa[i] = a[i]; pb[i] = b[i]; }
    return 3;
  }
  const int a[6] = {0, 0, 1, 0, 1, 2}, b[6] = {0, 1, 0, 2, 1, 0};
  for (int i = 0; i < 6; ++i) { pa[i] = a[i]; pb[i] = b[i]; }
  return 6;
}

// ---------------------------------------------------------------------------
// operand preparation
// ---------------------------------------------------------------------------
// sub_identity: split (src - I) instead of src (square matrices)
__global__ void split2d_kernel(const double* src, long long rows, long long cols, long long lds,
                               int np, bf16* p0, bf16* p1, bf16* p2, long long ldd,
                               int sub_identity) {
  bf16* P[3] = {p0, p1, p2};
  const long long n = rows * cols;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const long long r = e / cols, c = e - r * cols;
    double x = src[r * lds + c];
    if (sub_identity && r == c) x -= 1.0;
    put_pieces(x, np, P, r * ldd + c);
  }
}

// dst (C x R) = src (R x C)^T, split into pieces; 32x32 tiles through shared memory
__global__ void transpose_split_kernel(const double* src, long long R, long long C, long long lds,
                                       int np, bf16* p0, bf16* p1, bf16* p2, long long ldd) {
  __shared__ double tile[32][33];
  bf16* P[3] = {p0, p1, p2};
  const long long c0 = (long long)blockIdx.x * 32, r0 = (long long)blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const long long r = r0 + i, c = c0 + threadIdx.x;
    tile[i][threadIdx.x] = (r < R && c < C) ? src[r * lds + c] : 0.0;
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const long long c = c0 + i, r = r0 + threadIdx.x;
    if (c < C && r < R) put_pieces(tile[threadIdx.x][i], np, P, c * ldd + r);
  }
}

// walker (W, N, nc) doubles -> pieces of its transpose (W, nc rows, K = N) with row stride ld
__device__ __forceinline__ void walker_t_body(const double* wk, int N, int nc, int np, bf16* p0,
                                              bf16* p1, bf16* p2, long long ld, long long bstride,
                                              float* acc, int bx, int by, int bz) {
  __shared__ double tile[32][33];
  bf16* P[3] = {p0, p1, p2};
  const int b = bz;
  const int p0_ = bx * 32, n0 = by * 32;
  const double* src = wk + (long long)b * N * nc;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int p = p0_ + i, n = n0 + threadIdx.x;
    tile[i][threadIdx.x] = (p < N && n < nc) ? src[(long long)p * nc + n] : 0.0;
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int n = n0 + i, p = p0_ + threadIdx.x;
    if (n < nc && p < N) {
      const double x = tile[threadIdx.x][i];
      put_pieces(x, np, P, (long long)b * bstride + (long long)n * ld + p);
      acc[((long long)b * nc + n) * N + p] = (float)x;  // identity term of the first half-step
    }
  }
}

__global__ void walker_t_kernel(const double* wk, int N, int nc, int np, bf16* p0, bf16* p1,
                                bf16* p2, long long ld, long long bstride, float* acc) {
  walker_t_body(wk, N, nc, np, p0, p1, p2, ld, bstride, acc, blockIdx.x, blockIdx.y, blockIdx.z);
}

__global__ void walker_t_grouped(const WalkerTArgs* A, BlockMap m) {
  int local;
  const WalkerTArgs& a = A[block_owner(m, blockIdx.x, local)];
  const int per = a.gx * a.gy;
  const int bz = local / per, r = local - bz * per;
  walker_t_body(a.wk, a.N, a.nc, a.np, a.p[0], a.p[1], a.p[2], a.ld, a.bstride, a.acc, r % a.gx,
                r / a.gx, bz);
}

// ---------------------------------------------------------------------------
// epilogues
// ---------------------------------------------------------------------------
// C^T: rows g (Cholesky vector) = TMEM lanes, columns (w, re/im); the partial
// sums land in part[z][(w,c)][g] so that a warp's stores are contiguous in g,
// as the FP32 values the accumulator holds (the prep kernel sums them in FP64)
struct FbEpiU {
  float* part;
  long long ld, zstride;
  template <int BN>
  __device__ void tile(int z, int mti, int nti, int row, const AccSrc& src, const UmmaShape& s,
                       uint8_t*) const {
    const int g = mti * s.a_step + row, M = s.M, Nn = s.N;  // fields in registers before the stores
    const long long l = ld;
    float* dst = part + (long long)z * zstride + g;
#pragma unroll 1
    for (int ch = 0; ch < BN / 16; ++ch) {
      float v[16];
      src.load16(ch * 16, v);
      if (g >= M) continue;
      const int n0 = nti * s.b_step + ch * 16;
#pragma unroll
      for (int i = 0; i < 16; ++i)
        if (n0 + i < Nn) dst[(long long)(n0 + i) * l] = v[i];
    }
  }
};

struct VhsEpiU {
  bf16* vp[3];
  int npc, N;
  long long ld, wstride;
  template <int BN>
  __device__ void tile(int, int mti, int nti, int row, const AccSrc& src, const UmmaShape& s,
                       uint8_t*) const {
    // fields in registers before the bf16 stores
    const int n_ = N, np = npc, M = s.M, Nn = s.N;
    const long long l = ld, ws = wstride;
    const int q = mti * s.a_step + row;  // q = p*N + r
    const int p = q / n_, r = q - (q / n_) * n_;
    bf16* const v0 = vp[0] + (long long)p * l + r;
    bf16* const v1 = vp[1] + (long long)p * l + r;
    bf16* const v2 = np > 2 ? vp[2] + (long long)p * l + r : nullptr;
#pragma unroll 1
    for (int ch = 0; ch < BN / 16; ++ch) {
      float v[16];
      src.load16(ch * 16, v);
      if (q >= M) continue;
      const int n0 = nti * s.b_step + ch * 16;
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int n = n0 + i;
        if (n < Nn) {
          const long long off = (long long)(n >> 1) * ws + (n & 1) * n_;
          const float x = v[i];
          const bf16 h = __float2bfloat16_rn(x);
          v0[off] = h;
          const float rr = x - __bfloat162float(h);
          const bf16 lo = __float2bfloat16_rn(rr);
          v1[off] = lo;
          if (np > 2) v2[off] = __float2bfloat16_rn(rr - __bfloat162float(lo));
        }
      }
    }
  }
};

// Modes of the propagator GEMMs.  The one-body factor is applied as
// w + (e^{-dt h/2} - I) w: the tensor cores see only the small correction D
// and the identity part is added exactly from the FP32 accumulator.
// The Taylor series of e^{VHS} y runs in Horner form, z_T = y,
// z_{n-1} = y + VHS z_n / n, down to z_0 = sum_{n <= T} VHS^n y / n!: every
// term reads y from the FP32 accumulator and only the last one writes it back,
// where the forward sum (acc += VHS^n y / n!) read and wrote it in each term.
//   PM_Y     v = D w      : acc = w + v = y ; next B <- [y^T | (i y)^T]
//   PM_H     v = VHS z_n  : z = acc + v/n   ; next B <- [z^T | (i z)^T]
//   PM_HLAST v = VHS z_1  : z_0 = acc + v   ; acc = z_0 ; next B <- z_0^T
//   PM_OUT   v = D acc    : walker = acc + v  (FP64 walker state)
enum { PM_Y = 0, PM_H = 1, PM_HLAST = 2, PM_OUT = 3 };

struct PropEpiU {
  int mode, npc, N, nc;
  float scale;
  float* acc;           // (W, nc, N) fp32, transposed so that a warp's lanes (rows p) are contiguous
  long long acc_bs;
  bf16* bt[3];          // next B operand: (W, nc rows, ld) pieces
  long long bt_ld, bt_bs;
  double* wout;         // (W, N, nc) doubles
  template <int BN>
  __device__ void tile(int b, int mti, int nti, int row, const AccSrc& src, const UmmaShape& s,
                       uint8_t*) const {
    // every field in a register first: the stores below go through float and
    // bf16 pointers that the compiler cannot prove leave this struct alone
    const int md = mode, np = npc, n_ = N, ncol = nc;
    const float sc = scale;
    const long long ld = bt_ld;
    const int p = mti * s.a_step + row;
    const bool ok = p < n_;
    float* const acol = acc + (long long)b * acc_bs + p;  // element (n, p) at acol[n * N]
    const long long bb = (long long)b * bt_bs + p;
    bf16* const q0 = bt[0] + bb;
    bf16* const q1 = bt[1] + bb;
    bf16* const q2 = np > 2 ? bt[2] + bb : nullptr;
    double* const wo = md == PM_OUT ? wout + (long long)b * n_ * ncol + (long long)p * ncol : nullptr;
    // split-BF16 pieces of x at offset `off` of this row's operand column
    auto put = [&](float x, long long off) {
      const bf16 h = __float2bfloat16_rn(x);
      q0[off] = h;
      const float r = x - __bfloat162float(h);
      const bf16 l = __float2bfloat16_rn(r);
      q1[off] = l;
      if (np > 2) q2[off] = __float2bfloat16_rn(r - __bfloat162float(l));
    };
#pragma unroll 1
    for (int ch = 0; ch < BN / 16; ++ch) {
      float v[16];
      src.load16(ch * 16, v);
      const int n0 = nti * BN + ch * 16;  // column tiles of BN when 2 No > BN
      if (!ok || n0 >= ncol) continue;
      // all accumulator loads of the chunk first (independent, in flight together)
      float av[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) av[i] = (n0 + i < ncol) ? acol[(long long)(n0 + i) * n_] : 0.f;
#pragma unroll
      for (int i = 0; i < 16; i += 2) {
        const int n = n0 + i;  // (re, im) pair of orbital j = n/2
        if (n >= ncol) break;
        float* a0 = acol + (long long)n * n_;
        float* a1 = a0 + n_;
        float tr = v[i], ti = v[i + 1];
        if (md == PM_OUT) {
          wo[n] = (double)(av[i] + tr);
          wo[n + 1] = (double)(av[i + 1] + ti);
          continue;
        }
        if (md == PM_Y) {
          tr += av[i];
          ti += av[i + 1];
          *a0 = tr;
          *a1 = ti;
        } else {  // Horner step z = y + v / n, y in the accumulator
          tr = av[i] + tr * sc;
          ti = av[i + 1] + ti * sc;
          if (md == PM_HLAST) {  // hand the finished sum to the closing half-step
            *a0 = tr;
            *a1 = ti;
          }
        }
        // rows n (re) and n+1 (im) of the next B operand; columns [0,N): x, [N,2N): i*x
        const long long o0 = (long long)n * ld, o1 = o0 + ld;
        put(tr, o0);
        put(ti, o1);
        if (md != PM_HLAST) {
          put(-ti, o0 + n_);
          put(tr, o1 + n_);
        }
      }
    }
  }
};

struct ExchEpiU {
  int G, no, W, gpt, wpt;
  double* cout;    // (W, G) complex
  double* excout;  // (mt, W) complex
  // Per walker of the tile: stage f (gcount*No rows x 2No floats) in shared
  // memory as (re, im) pairs, row stride exch_fs2(No) pairs (odd: 64-bit
  // accesses by consecutive rows or consecutive pairs are bank-conflict free).
  // Row (g, i) forms sum_j f[i][j] f[j][i] in four FP32 chains combined in
  // FP64; the rows of one Cholesky vector are summed by a segmented shuffle
  // reduction inside each warp plus at most three cross-warp partials, then
  // the Cholesky vectors of the tile by a shuffle reduction in the first
  // warp.  Every sum has a fixed order, so results are reproducible.
  template <int BN>
  __device__ void tile(int, int mti, int nti, int row, const AccSrc& src, const UmmaShape& s,
                       uint8_t* smem) const {
    const int nc = 2 * no, fs2 = exch_fs2(no);
    float2* Fs = reinterpret_cast<float2*>(smem);
    double4* pr = reinterpret_cast<double4*>(smem + exch_fs_bytes(no));
    double2* ge = reinterpret_cast<double2*>(pr + 128);
    const int g0 = mti * gpt, w0 = nti * wpt;
    const int gcount = min(gpt, G - g0), wcount = min(wpt, W - w0);
    const bool valid = row < gcount * no;
    const int gl = row / no, i = row - (row / no) * no;
    const int lane = row & 31;
    const int seg = valid ? gl : -1;
    for (int wl = 0; wl < wcount; ++wl) {
      const int cb = wl * nc;  // even; chunk starts are multiples of 16, so pairs stay aligned
      const int c_lo = cb & ~15, c_hi = (cb + nc + 15) & ~15;
      for (int c = c_lo; c < c_hi; c += 16) {
        float v[16];
        src.load16(c, v);
#pragma unroll
        for (int k = 0; k < 16; k += 2) {
          const int col = c + k - cb;
          if (col >= 0 && col < nc) Fs[row * fs2 + (col >> 1)] = make_float2(v[k], v[k + 1]);
        }
      }
      named_sync_epi();
      double4 q = make_double4(0.0, 0.0, 0.0, 0.0);
      if (valid) {
        const float2* fr = Fs + row * fs2;
        const float2* fc = Fs + (gl * no) * fs2 + i;
        float ar[4] = {0.f, 0.f, 0.f, 0.f}, ai[4] = {0.f, 0.f, 0.f, 0.f};
        int j = 0;
        for (; j + 4 <= no; j += 4) {
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const float2 a = fr[j + u];
            const float2 b = fc[(j + u) * fs2];
            ar[u] = fmaf(a.x, b.x, fmaf(-a.y, b.y, ar[u]));
            ai[u] = fmaf(a.x, b.y, fmaf(a.y, b.x, ai[u]));
          }
        }
        for (; j < no; ++j) {
          const float2 a = fr[j];
          const float2 b = fc[j * fs2];
          ar[0] = fmaf(a.x, b.x, fmaf(-a.y, b.y, ar[0]));
          ai[0] = fmaf(a.x, b.y, fmaf(a.y, b.x, ai[0]));
        }
        const float2 d = fr[i];
        q = make_double4(((double)ar[0] + (double)ar[1]) + ((double)ar[2] + (double)ar[3]),
                         ((double)ai[0] + (double)ai[1]) + ((double)ai[2] + (double)ai[3]),
                         (double)d.x, (double)d.y);
      }
      // suffix sums inside each run of equal `seg` within the warp
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const double tx = __shfl_down_sync(0xffffffffu, q.x, off);
        const double ty = __shfl_down_sync(0xffffffffu, q.y, off);
        const double tz = __shfl_down_sync(0xffffffffu, q.z, off);
        const double tw = __shfl_down_sync(0xffffffffu, q.w, off);
        const int st = __shfl_down_sync(0xffffffffu, seg, off);
        if (lane + off < 32 && st == seg) {
          q.x += tx;
          q.y += ty;
          q.z += tz;
          q.w += tw;
        }
      }
      const int sp = __shfl_up_sync(0xffffffffu, seg, 1);
      if (valid && (lane == 0 || sp != seg)) pr[row] = q;  // run heads
      named_sync_epi();
      if (gcount <= 32) {
        if (row < 32) {
          double sr = 0.0, si = 0.0;
          if (row < gcount) {
            const int h = row * no;
            double4 a = pr[h];
            for (int r = (h / 32 + 1) * 32; r < h + no; r += 32) {
              const double4 b = pr[r];
              a.x += b.x;
              a.y += b.y;
              a.z += b.z;
              a.w += b.w;
            }
            const long long co = 2 * ((long long)(w0 + wl) * G + g0 + row);
            cout[co] = a.z;
            cout[co + 1] = a.w;
            sr = a.x;
            si = a.y;
          }
#pragma unroll
          for (int off = 16; off > 0; off >>= 1) {
            sr += __shfl_down_sync(0xffffffffu, sr, off);
            si += __shfl_down_sync(0xffffffffu, si, off);
          }
          if (row == 0) {
            excout[2 * ((long long)mti * W + w0 + wl)] = sr;
            excout[2 * ((long long)mti * W + w0 + wl) + 1] = si;
          }
        }
      } else {  // more than 32 Cholesky vectors per tile (No < 4)
        if (row < gcount) {
          const int h = row * no;
          double4 a = pr[h];
          for (int r = (h / 32 + 1) * 32; r < h + no; r += 32) {
            const double4 b = pr[r];
            a.x += b.x;
            a.y += b.y;
            a.z += b.z;
            a.w += b.w;
          }
          const long long co = 2 * ((long long)(w0 + wl) * G + g0 + row);
          cout[co] = a.z;
          cout[co + 1] = a.w;
          ge[row] = make_double2(a.x, a.y);
        }
        named_sync_epi();
        if (row == 0) {
          double sx = 0, sy = 0;
          for (int g = 0; g < gcount; ++g) {
            sx += ge[g].x;
            sy += ge[g].y;
          }
          excout[2 * ((long long)mti * W + w0 + wl)] = sx;
          excout[2 * ((long long)mti * W + w0 + wl) + 1] = sy;
        }
      }
    }
  }
  static size_t smem_extra(int no) { return exch_epi_extra(no); }
};

// ---------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------
template <class Epi>
int setup_maps(UmmaParams<Epi>& P, bf16* const a[3], int npa, long long aK, long long arows,
               long long abatch, long long ald, long long abs, bf16* const b[3], int npb,
               long long bK, long long brows, long long bbatch, long long bld, long long bbs,
               int bn) {
  for (int i = 0; i < npa; ++i) {
    int rc = make_tmap_bf16(&P.ta[i], a[i], aK, arows, abatch, ald, abs, kUBM);
    if (rc != AFQ_OK) return rc;
  }
  for (int j = 0; j < npb; ++j) {
    int rc = make_tmap_bf16(&P.tb[j], b[j], bK, brows, bbatch, bld, bbs, bn);
    if (rc != AFQ_OK) return rc;
  }
  return AFQ_OK;
}

template <class Epi>
void base_shape(UmmaParams<Epi>& P, int npc, int M, int N, int K, int batch, int bn, int* err) {
  P.s.npa = P.s.npb = npc;
  P.s.npairs = pairs_for(npc, P.s.pa, P.s.pb);
  P.s.M = M;
  P.s.N = N;
  P.s.K = K;
  P.s.batch = batch;
  P.s.a_batched = 1;
  P.s.a_step = kUBM;
  P.s.b_step = bn;
  P.s.mt = (M + kUBM - 1) / kUBM;
  P.s.nt = (N + bn - 1) / bn;
  P.s.ksplit = 1;
  P.s.kchunk = (K + kUBK - 1) / kUBK * kUBK;
  P.s.ngroups = 1;
  P.s.kc = 0;
  P.s.err = err;
}

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// While a batch is built, the GEMMs of one solve are recorded here (final
// parameters, tile width, epilogue warpgroups) instead of launched.
struct SinkRec {
  int prof, bn, eg;
  UmmaShape shape;
  std::vector<unsigned char> bytes;  // the UmmaParams<Epi> block
};
thread_local std::vector<SinkRec>* g_sink = nullptr;

// `extra`: epilogue scratch bytes per epilogue warpgroup
template <int BN, int EG = 1, class Epi>
int run(UmmaParams<Epi>& P, size_t extra, cudaStream_t st, int prof_id, const afq_tuning& T) {
  P.s.epi_bytes = (int)align256(extra);
  P.s.stages = umma_pick_stages(BN, P.s.npa, P.s.npb, size_t(EG) * P.s.epi_bytes);
  if (P.s.stages < 2 && P.s.kc > 0 && extra == umma_chunk_stage_bytes(BN)) {
    // no room for the chunk staging next to two stages: accumulate in one chunk
    P.s.kc = 0;
    P.s.epi_bytes = 0;
    P.s.stages = umma_pick_stages(BN, P.s.npa, P.s.npb, 0);
  }
  if (P.s.stages < 2) return AFQ_ERR_SHAPE;
  if (T.max_stages >= 2 && P.s.stages > T.max_stages)
    P.s.stages = T.max_stages;
  else if (T.max_stages == 0 && prof_id == K_PROP && P.s.stages > 3)
    P.s.stages = 3;  // the propagator streams VHS from HBM: three stages measured ~1 % faster than four
  if (g_sink) {
    SinkRec r;
    r.prof = prof_id;
    r.bn = BN;
    r.eg = EG;
    r.shape = P.s;
    r.bytes.resize(sizeof(P));
    std::memcpy(r.bytes.data(), &P, sizeof(P));
    g_sink->push_back(std::move(r));
    return AFQ_OK;
  }
  int ctas = sm_count();
  if (T.grid_cap > 0 && T.grid_cap < ctas) ctas = T.grid_cap;
  ProfScope ps(prof_id, st);
  return launch_umma<BN, EG>(P, ctas, st) == cudaSuccess ? AFQ_OK : AFQ_ERR_CUDA;
}

int* err_flag(const Layout& L, double* work) {
  return reinterpret_cast<int*>(work + L.w_misc);
}

template <int BN>
int prop_launch(const Layout& L, const double* prep, double* work, int s, int nc, int mode,
                float scale, bf16* const a[3], long long aK, long long ald, long long abs,
                int a_batched, bf16* const bsrc[3], bf16* const bdst[3], double* wout,
                int seq, cudaStream_t st) {
  UmmaParams<PropEpiU> P{};
  const int N = L.N;
  const long long btbs = 2LL * L.nomax * L.Kv;
  int rc = setup_maps(P, a, L.npc, aK, N, a_batched ? L.W : 1, ald, abs, bsrc, L.npc, aK, nc, L.W,
                      L.Kv, btbs, BN);
  if (rc != AFQ_OK) return rc;
  base_shape(P, L.npc, N, nc, (int)aK, L.W, BN, err_flag(L, work));
  P.s.a_batched = a_batched;
  // consecutive launches of one step walk the walkers in opposite directions, so
  // each starts on the walkers whose VHS, operand pieces and accumulator rows the
  // previous launch touched last (still in L2)
  P.s.reverse = (L.tune.prop_order == 0) && (seq & 1);
  P.epi.mode = mode;
  P.epi.npc = L.npc;
  P.epi.N = N;
  P.epi.nc = nc;
  P.epi.scale = scale;
  P.epi.acc = reinterpret_cast<float*>(work + L.v_acc);
  P.epi.acc_bs = (long long)N * nc;
  for (int i = 0; i < 3; ++i) P.epi.bt[i] = bdst ? bdst[i] : nullptr;
  P.epi.bt_ld = L.Kv;
  P.epi.bt_bs = btbs;
  P.epi.wout = wout;
  P.s.ngroups = 2;
  // The whole K (2N) in one TMEM chain, which leaves the shared memory to the
  // operand pipeline (four stages at N = 200: 87 -> 79 us per launch, and
  // 469 -> 335 us at N = 300; block energies within 2e-5 Ha of FP64 either
  // way), or (prop_chunk = 2) chunks of four 64-wide K blocks summed in FP32
  // round-to-nearest through a shared-memory row per TMEM lane
  const bool one_chain = L.tune.prop_chunk != 2;
  P.s.kc = one_chain ? 0 : 4;
  const size_t ex = one_chain ? 0 : umma_chunk_stage_bytes(BN);
  // the propagator's epilogue (FP32 accumulator update, next operand pieces)
  // outlasts its MMAs: as many epilogue warpgroups (up to three) as their
  // staging, two pipeline stages and one TMEM buffer per group allow
  const size_t cs = align256(ex);
  const int want = L.tune.prop_epi_groups ? L.tune.prop_epi_groups : 3;
  if (want >= 3 && 3 * 2 * BN <= 512 && umma_pick_stages(BN, L.npc, L.npc, 3 * cs) >= 2)
    return run<BN, 3>(P, ex, st, K_PROP, L.tune);
  if (want >= 2 && umma_pick_stages(BN, L.npc, L.npc, 2 * cs) >= 2)
    return run<BN, 2>(P, ex, st, K_PROP, L.tune);
  return run<BN, 1>(P, ex, st, K_PROP, L.tune);
}

template <int BN>
int exch_launch(const Layout& L, const double* prep, double* work, int s, cudaStream_t st) {
  const UExchTile& X = L.uex[s];
  const int no = L.no[s];
  UmmaParams<ExchEpiU> P{};
  bf16* a[3];
  bf16* b[3];
  piece_ptrs(const_cast<double*>(prep), L.q_rc[s], L.q_rc_ps[s], L.npc, a);
  piece_ptrs(work, L.v_gt[s], L.v_gt_ps[s], L.npc, b);
  const long long arows = (long long)L.G * no, brows = (long long)L.W * 2 * no;
  int rc = setup_maps(P, a, L.npc, L.N, arows, 1, L.Nb, arows * L.Nb, b, L.npc, L.N, brows, 1,
                      L.Nb, brows * L.Nb, BN);
  if (rc != AFQ_OK) return rc;
  base_shape(P, L.npc, (int)arows, (int)brows, L.N, 1, BN, err_flag(L, work));
  P.s.ngroups = 2;  // hi x hi products apart from the cross terms: shorter rounding chains
  P.s.a_step = X.gpt * no;
  P.s.b_step = X.wpt * 2 * no;
  P.s.mt = X.mt;
  P.s.nt = (L.W + X.wpt - 1) / X.wpt;
  P.epi.G = L.G;
  P.epi.no = no;
  P.epi.W = L.W;
  P.epi.gpt = X.gpt;
  P.epi.wpt = X.wpt;
  P.epi.cout = work + L.w_c[s];
  P.epi.excout = work + L.w_exc[s];
  return run<BN>(P, ExchEpiU::smem_extra(no), st, K_EXCH, L.tune);
}

}  // namespace

int mixed_prepare(const Layout& L, double* P, cudaStream_t st) {
  ProfScope ps(K_MISC, st);
  bf16* q[3];
  // force-bias operand: rot_chol concatenated over spins (G x Kfb)
  piece_ptrs(P, L.q_rccat, L.q_rccat_ps, L.npc, q);
  split2d_kernel<<<1184, 256, 0, st>>>(P + L.p_rccat, L.G, L.Kfb_used, L.Kfb, L.npc, q[0], q[1],
                                       q[2], L.Kb, 0);
  // VHS operand: chol transposed to (N^2 x G)
  piece_ptrs(P, L.q_cholT, L.q_cholT_ps, L.npc, q);
  {
    const long long NN = (long long)L.N * L.N;
    dim3 grid((unsigned)((NN + 31) / 32), (unsigned)((L.G + 31) / 32));
    transpose_split_kernel<<<grid, dim3(32, 8), 0, st>>>(P + L.p_chol, L.G, NN, L.N2pad, L.npc,
                                                         q[0], q[1], q[2], L.Gb);
  }
  for (int s = 0; s < L.np; ++s) {
    piece_ptrs(P, L.q_exph1[s], L.q_exph1_ps, L.npc, q);
    // the propagator applies e^{-dt h/2} as w + (e^{-dt h/2} - I) w
    split2d_kernel<<<296, 256, 0, st>>>(P + L.p_exph1[s], L.N, L.N, L.Npad, L.npc, q[0], q[1],
                                        q[2], L.Nb, 1);
  }
  const int ntr = L.uhf_trial ? 2 : 1;
  for (int s = 0; s < ntr; ++s) {
    piece_ptrs(P, L.q_rc[s], L.q_rc_ps[s], L.npc, q);
    split2d_kernel<<<1184, 256, 0, st>>>(P + L.p_rc[s], (long long)L.G * L.no[s], L.N, L.Npad,
                                         L.npc, q[0], q[1], q[2], L.Nb, 0);
  }
  return cudaGetLastError() == cudaSuccess ? AFQ_OK : AFQ_ERR_CUDA;
}

template <int BN>
int fb_launch(const Layout& L, const double* prep, double* work, cudaStream_t st) {
  UmmaParams<FbEpiU> P{};
  bf16* a[3];
  bf16* b[3];
  piece_ptrs(const_cast<double*>(prep), L.q_rccat, L.q_rccat_ps, L.npc, a);
  piece_ptrs(work, L.v_gpl, L.v_gpl_ps, L.npc, b);
  const long long K = L.Kfb_used, N2 = 2LL * L.W;
  int rc = setup_maps(P, a, L.npc, K, L.G, 1, L.Kb, (long long)L.G * L.Kb, b, L.npc, K, N2, 1,
                      L.Kb, N2 * L.Kb, BN);
  if (rc != AFQ_OK) return rc;
  base_shape(P, L.npc, L.G, (int)N2, (int)K, 1, BN, err_flag(L, work));
  // every split owns at least one K block; partial buffers beyond the last
  // split are zeroed so that the consumer's fixed-order sum stays exact
  const long long kblocks = (K + kUBK - 1) / kUBK;
  const long long per = (kblocks + L.splitk - 1) / L.splitk;
  const int ks = (int)((kblocks + per - 1) / per);
  P.s.ksplit = ks;
  P.s.kchunk = (int)(per * kUBK);
  float* part = reinterpret_cast<float*>(work + L.w_fbpart);
  for (int z = ks; z < L.splitk; ++z)
    if (cudaMemsetAsync(part + z * 2LL * L.W * L.Gpad, 0, sizeof(float) * 2LL * L.W * L.Gpad, st) !=
        cudaSuccess)
      return AFQ_ERR_CUDA;  // (while recording a batch: once, on the legacy stream, at build time)
  P.epi.part = part;
  P.epi.ld = L.Gpad;
  P.epi.zstride = 2LL * L.W * L.Gpad;
  P.s.ngroups = 2;
  P.s.kc = 4;
  return run<BN>(P, umma_chunk_stage_bytes(BN), st, K_FB, L.tune);
}

int mixed_fb_gemm(const Layout& L, const double* prep, double* work, cudaStream_t st) {
  return L.fb_bn == 64 ? fb_launch<64>(L, prep, work, st) : fb_launch<128>(L, prep, work, st);
}

template <int BN>
int vhs_launch(const Layout& L, const double* prep, double* work, cudaStream_t st) {
  UmmaParams<VhsEpiU> P{};
  bf16* a[3];
  bf16* b[3];
  piece_ptrs(const_cast<double*>(prep), L.q_cholT, L.q_cholT_ps, L.npc, a);
  piece_ptrs(work, L.v_xt, L.v_xt_ps, L.npc, b);
  const long long NN = (long long)L.N * L.N, M2 = 2LL * L.W;
  int rc = setup_maps(P, a, L.npc, L.G, NN, 1, L.Gb, NN * L.Gb, b, L.npc, L.G, M2, 1, L.Gb,
                      M2 * L.Gb, BN);
  if (rc != AFQ_OK) return rc;
  base_shape(P, L.npc, (int)NN, (int)M2, L.G, 1, BN, err_flag(L, work));
  piece_ptrs(work, L.v_vhs, L.v_vhs_ps, L.npc, P.epi.vp);
  P.epi.npc = L.npc;
  P.epi.N = L.N;
  P.epi.ld = L.Kv;
  P.epi.wstride = (long long)L.N * L.Kv;
  // K = G in one TMEM chain per accumulator group (the hi x hi product apart),
  // which leaves the shared memory to four operand stages (364 -> 276 us per
  // launch at N = 200, G = 1000, W = 512; block energies 7.8e-6 Ha from FP64),
  // or (vhs_chunk = 2) in chunks of four 64-wide K blocks summed in FP32
  // round-to-nearest through a shared-memory row per TMEM lane (5.0e-6 Ha)
  P.s.ngroups = 2;
  const bool one_chain = L.tune.vhs_chunk != 2;
  P.s.kc = one_chain ? 0 : 4;
  return run<BN>(P, one_chain ? 0 : umma_chunk_stage_bytes(BN), st, K_VHS, L.tune);
}

int mixed_vhs_gemm(const Layout& L, const double* prep, double* work, cudaStream_t st) {
  // default: two pieces 128-wide tiles, three pieces 64-wide (both keep chunked accumulation)
  return L.vhs_bn == 128 ? vhs_launch<128>(L, prep, work, st) : vhs_launch<64>(L, prep, work, st);
}

template <int BN>
static int propagate_one(const Layout& L, const double* prep, double* work, double* wk, int s,
                         int n_exp_terms, cudaStream_t st) {
  const int N = L.N, nc = 2 * L.no[s];
  bf16 *e[3], *v[3], *b0[3], *b1[3];
  piece_ptrs(const_cast<double*>(prep), L.q_exph1[s], L.q_exph1_ps, L.npc, e);
  piece_ptrs(work, L.v_vhs, L.v_vhs_ps, L.npc, v);
  piece_ptrs(work, L.v_bt[0], L.v_bt_ps, L.npc, b0);
  piece_ptrs(work, L.v_bt[1], L.v_bt_ps, L.npc, b1);
  const long long btbs = 2LL * L.nomax * L.Kv;
  if (!g_sink) {  // a batch launches the operand preparation of all its solves together
    ProfScope ps(K_MISC, st);
    dim3 grid((N + 31) / 32, (nc + 31) / 32, L.W);
    walker_t_kernel<<<grid, dim3(32, 8), 0, st>>>(wk, N, nc, L.npc, b0[0], b0[1], b0[2], L.Kv,
                                                  btbs, reinterpret_cast<float*>(work + L.v_acc));
    if (cudaGetLastError() != cudaSuccess) return AFQ_ERR_CUDA;
  }
  const long long vbs = (long long)N * L.Kv;
  if (n_exp_terms <= 1) {
    int rc = prop_launch<BN>(L, prep, work, s, nc, PM_Y, 1.f, e, N, L.Nb, N * L.Nb, 0, b0, b1,
                             nullptr, 0, st);
    if (rc != AFQ_OK) return rc;
    return prop_launch<BN>(L, prep, work, s, nc, PM_OUT, 1.f, e, N, L.Nb, N * L.Nb, 0, b1, nullptr,
                           wk, 1, st);
  }
  // y = e^{-dt h/2} w  -> acc, and [y^T | (i y)^T] into b1
  int rc = prop_launch<BN>(L, prep, work, s, nc, PM_Y, 1.f, e, N, L.Nb, N * L.Nb, 0, b0, b1,
                           nullptr, 0, st);
  if (rc != AFQ_OK) return rc;
  bf16** src = b1;
  bf16** dst = b0;
  // Horner: z_{n-1} = y + VHS z_n / n for n = T .. 1 (T = n_exp_terms - 1)
  for (int n = n_exp_terms - 1; n >= 1; --n) {
    const int mode = (n == 1) ? PM_HLAST : PM_H;
    rc = prop_launch<BN>(L, prep, work, s, nc, mode, 1.f / n, v, 2LL * N, L.Kv, vbs, 1, src, dst,
                         nullptr, n_exp_terms - n, st);
    if (rc != AFQ_OK) return rc;
    bf16** t = src;
    src = dst;
    dst = t;
  }
  // w' = e^{-dt h/2} (y + sum t_n): B operand holds the finished sum
  return prop_launch<BN>(L, prep, work, s, nc, PM_OUT, 1.f, e, N, L.Nb, N * L.Nb, 0, src, nullptr,
                         wk, n_exp_terms, st);
}

int mixed_propagate_walkers(const Layout& L, const double* prep, double* work,
                            double* const walkers[2], int n_exp_terms, cudaStream_t st) {
  for (int s = 0; s < L.np; ++s) {
    const int nc = 2 * L.no[s];
    const int bn = L.tune.prop_bn;  // tuning: a narrower column tile (several per walker)
    int rc;
    if (bn == 16)
      rc = propagate_one<16>(L, prep, work, walkers[s], s, n_exp_terms, st);
    else if (bn == 32)
      rc = propagate_one<32>(L, prep, work, walkers[s], s, n_exp_terms, st);
    else if (bn == 48)
      rc = propagate_one<48>(L, prep, work, walkers[s], s, n_exp_terms, st);
    else if (bn == 64)
      rc = propagate_one<64>(L, prep, work, walkers[s], s, n_exp_terms, st);
    else if (bn == 80)
      rc = propagate_one<80>(L, prep, work, walkers[s], s, n_exp_terms, st);
    else if (bn == 96)
      rc = propagate_one<96>(L, prep, work, walkers[s], s, n_exp_terms, st);
    else if (bn == 128)
      rc = propagate_one<128>(L, prep, work, walkers[s], s, n_exp_terms, st);
    else if (nc <= 16)
      rc = propagate_one<16>(L, prep, work, walkers[s], s, n_exp_terms, st);
    else if (nc <= 32)
      rc = propagate_one<32>(L, prep, work, walkers[s], s, n_exp_terms, st);
    else if (nc <= 48)
      rc = propagate_one<48>(L, prep, work, walkers[s], s, n_exp_terms, st);
    else if (nc <= 64)
      rc = propagate_one<64>(L, prep, work, walkers[s], s, n_exp_terms, st);
    else if (nc <= 80)
      rc = propagate_one<80>(L, prep, work, walkers[s], s, n_exp_terms, st);
    else if (nc <= 96)
      rc = propagate_one<96>(L, prep, work, walkers[s], s, n_exp_terms, st);
    else
      rc = propagate_one<128>(L, prep, work, walkers[s], s, n_exp_terms, st);
    if (rc != AFQ_OK) return rc;
  }
  return AFQ_OK;
}

int mixed_exchange(const Layout& L, const double* prep, double* work, int s, cudaStream_t st) {
  switch (L.uex[s].bn) {
    case 128: return exch_launch<128>(L, prep, work, s, st);
    case 96: return exch_launch<96>(L, prep, work, s, st);
    case 80: return exch_launch<80>(L, prep, work, s, st);
    case 64: return exch_launch<64>(L, prep, work, s, st);
    default: return exch_launch<32>(L, prep, work, s, st);
  }
}

cudaError_t launch_walker_t_grouped(const WalkerTArgs* args, const BlockMap& m, cudaStream_t st) {
  ProfScope ps(K_MISC, st);
  walker_t_grouped<<<m.start[m.n], dim3(32, 8), 0, st>>>(args, m);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// batches: the step's GEMMs of many solves, one persistent launch per group
// ---------------------------------------------------------------------------
namespace {

// one grouped launch: entries of the same kind, tile width, epilogue
// warpgroups, ring depth and operand/epilogue layout
struct GroupLaunch {
  int prof, bn, eg;
  UmmaShape shape0;
  const void* entries;  // device
  int n, stages;
  int start[kUmmaMaxGroup + 1];
};

template <int BN, int EG, class Epi>
int launch_group_as(const GroupLaunch& g, cudaStream_t st) {
  UmmaGroup<Epi> G;
  G.entries = static_cast<const UmmaParams<Epi>*>(g.entries);
  G.n = g.n;
  G.stages = g.stages;
  for (int i = 0; i <= g.n; ++i) G.start[i] = g.start[i];
  ProfScope ps(g.prof, st);
  return launch_umma_group<BN, EG>(G, g.shape0, sm_count(), st) == cudaSuccess ? AFQ_OK : AFQ_ERR_CUDA;
}

template <class Epi, int EG>
int launch_group_bn(const GroupLaunch& g, cudaStream_t st) {
  switch (g.bn) {
    case 16: return launch_group_as<16, EG, Epi>(g, st);
    case 32: return launch_group_as<32, EG, Epi>(g, st);
    case 48: return launch_group_as<48, EG, Epi>(g, st);
    case 64: return launch_group_as<64, EG, Epi>(g, st);
    case 80: return launch_group_as<80, EG, Epi>(g, st);
    case 96: return launch_group_as<96, EG, Epi>(g, st);
    case 128: return launch_group_as<128, EG, Epi>(g, st);
    default: return AFQ_ERR_SHAPE;
  }
}

int launch_group(const GroupLaunch& g, cudaStream_t st) {
  if (g.prof == K_FB) {
    if (g.eg != 1 || (g.bn != 64 && g.bn != 128)) return AFQ_ERR_SHAPE;
    return g.bn == 64 ? launch_group_as<64, 1, FbEpiU>(g, st) : launch_group_as<128, 1, FbEpiU>(g, st);
  }
  if (g.prof == K_VHS) {
    if (g.eg != 1 || (g.bn != 64 && g.bn != 128)) return AFQ_ERR_SHAPE;
    return g.bn == 64 ? launch_group_as<64, 1, VhsEpiU>(g, st) : launch_group_as<128, 1, VhsEpiU>(g, st);
  }
  if (g.prof == K_PROP) {
    if (g.eg == 1) return launch_group_bn<PropEpiU, 1>(g, st);
    if (g.eg == 2) return launch_group_bn<PropEpiU, 2>(g, st);
    if (g.eg == 3) return launch_group_bn<PropEpiU, 3>(g, st);
  }
  return AFQ_ERR_SHAPE;
}

constexpr int kMaxPropLaunches = 34;  // n_exp_terms (<= 32) + 1, per spin sector

size_t rec_bytes_max() {
  size_t b = sizeof(UmmaParams<FbEpiU>);
  if (sizeof(UmmaParams<VhsEpiU>) > b) b = sizeof(UmmaParams<VhsEpiU>);
  if (sizeof(UmmaParams<PropEpiU>) > b) b = sizeof(UmmaParams<PropEpiU>);
  return (b + 255) & ~size_t(255);
}

}  // namespace

struct UmmaBatch {
  std::vector<GroupLaunch> fb, vhs;
  std::vector<GroupLaunch> prop[2][kMaxPropLaunches];
  int nprop = 0;
};

size_t umma_batch_table_bytes(int n, const Layout* L, int n_exp_terms) {
  size_t cnt = 0;
  for (int f = 0; f < n; ++f) cnt += 2 + (size_t)L[f].np * (n_exp_terms + 1);
  return cnt * rec_bytes_max() + 4096;
}

int umma_batch_create(int n, const Layout* L, const double* const* prep, double* const* work,
                      double* const* walkers0, double* const* walkers1, int n_exp_terms,
                      void* table, size_t table_bytes, UmmaBatch** out) {
  if (n < 1 || n > kMaxBatch || n_exp_terms + 1 > kMaxPropLaunches) return AFQ_ERR_SHAPE;
  // record every solve's GEMMs with the solo code path
  std::vector<std::vector<SinkRec>> recs(n);
  for (int f = 0; f < n; ++f) {
    std::vector<SinkRec> sink;
    g_sink = &sink;
    double* wk[2] = {walkers0[f], walkers1[f]};
    int rc = mixed_fb_gemm(L[f], prep[f], work[f], 0);
    if (rc == AFQ_OK) rc = mixed_vhs_gemm(L[f], prep[f], work[f], 0);
    if (rc == AFQ_OK) rc = mixed_propagate_walkers(L[f], prep[f], work[f], wk, n_exp_terms, 0);
    g_sink = nullptr;
    if (rc != AFQ_OK) return rc;
    recs[f] = std::move(sink);
  }
  if (cudaStreamSynchronize(0) != cudaSuccess) return AFQ_ERR_CUDA;  // the split-K zero fills
  // slot of record r of solve f: 0 fb, 1 vhs, 2 + s*(n_exp_terms+1) + i propagator i of sector s
  const int nprop = n_exp_terms <= 1 ? 2 : n_exp_terms + 1;
  for (int f = 0; f < n; ++f)
    if ((int)recs[f].size() != 2 + L[f].np * nprop) return AFQ_ERR_SHAPE;
  std::vector<unsigned char> host(table_bytes, 0);
  size_t off = 0;
  UmmaBatch* b = new UmmaBatch();
  b->nprop = nprop;
  // group the records of one slot across solves
  auto group_slot = [&](int slot_kind, int sector, int index, std::vector<GroupLaunch>& dst) -> int {
    std::vector<std::pair<const SinkRec*, int>> items;  // (record, solve)
    for (int f = 0; f < n; ++f) {
      int r;
      if (slot_kind == 0) r = 0;
      else if (slot_kind == 1) r = 1;
      else {
        if (sector >= L[f].np) continue;
        r = 2 + sector * nprop + index;
      }
      items.push_back({&recs[f][r], f});
    }
    std::vector<bool> done(items.size(), false);
    for (size_t i = 0; i < items.size(); ++i) {
      if (done[i]) continue;
      const SinkRec& k = *items[i].first;
      GroupLaunch g{};
      g.prof = k.prof;
      g.bn = k.bn;
      g.eg = k.eg;
      g.shape0 = k.shape;
      g.stages = k.shape.stages;
      g.n = 0;
      g.start[0] = 0;
      off = (off + 255) & ~size_t(255);
      const size_t first = off;
      for (size_t j = i; j < items.size(); ++j) {
        if (done[j]) continue;
        const SinkRec& r = *items[j].first;
        if (r.prof != k.prof || r.bn != k.bn || r.eg != k.eg || r.shape.stages != k.shape.stages ||
            r.shape.npa != k.shape.npa || r.shape.npb != k.shape.npb ||
            r.shape.ngroups != k.shape.ngroups || r.shape.epi_bytes != k.shape.epi_bytes ||
            r.bytes.size() != k.bytes.size())
          continue;
        if (off + r.bytes.size() > table_bytes) return AFQ_ERR_WORKSPACE;
        std::memcpy(host.data() + off, r.bytes.data(), r.bytes.size());
        off += r.bytes.size();
        const UmmaShape& S = r.shape;
        g.start[g.n + 1] = g.start[g.n] + S.batch * S.ksplit * S.mt * S.nt;
        ++g.n;
        done[j] = true;
      }
      g.entries = static_cast<unsigned char*>(table) + first;
      dst.push_back(g);
    }
    return AFQ_OK;
  };
  int rc = group_slot(0, 0, 0, b->fb);
  if (rc == AFQ_OK) rc = group_slot(1, 0, 0, b->vhs);
  for (int sct = 0; sct < 2 && rc == AFQ_OK; ++sct)
    for (int i = 0; i < nprop && rc == AFQ_OK; ++i) rc = group_slot(2, sct, i, b->prop[sct][i]);
  if (rc == AFQ_OK && cudaMemcpy(table, host.data(), off, cudaMemcpyHostToDevice) != cudaSuccess)
    rc = AFQ_ERR_CUDA;
  if (rc != AFQ_OK) {
    delete b;
    return rc;
  }
  *out = b;
  return AFQ_OK;
}

int umma_batch_fb(const UmmaBatch* b, cudaStream_t st) {
  for (const GroupLaunch& g : b->fb) {
    const int rc = launch_group(g, st);
    if (rc != AFQ_OK) return rc;
  }
  return AFQ_OK;
}

int umma_batch_vhs(const UmmaBatch* b, cudaStream_t st) {
  for (const GroupLaunch& g : b->vhs) {
    const int rc = launch_group(g, st);
    if (rc != AFQ_OK) return rc;
  }
  return AFQ_OK;
}

int umma_batch_prop(const UmmaBatch* b, int sector, int index, cudaStream_t st) {
  if (sector < 0 || sector > 1 || index < 0 || index >= b->nprop) return AFQ_ERR_ARG;
  for (const GroupLaunch& g : b->prop[sector][index]) {
    const int rc = launch_group(g, st);
    if (rc != AFQ_OK) return rc;
  }
  return AFQ_OK;
}

int umma_batch_nprop(const UmmaBatch* b) { return b->nprop; }

void umma_batch_destroy(UmmaBatch* b) { delete b; }

}  // namespace afq
