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

// asynchronous global -> shared copies (Ampere-style cp.async): the next
// chunk of walker rows streams in while the current one is multiplied
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                   static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(
                   static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// wait until at most one group (the newest) of this thread's copies is in flight
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// Gauss-Jordan inverse with partial pivoting of the No x No complex S in
// shared memory, in place, by the whole CTA (T threads); returns det S in
// thread 0.
template <int T>
__device__ double2 gauss_jordan_cta(double2* S, double2* colk, int* perm, double2* ipk_s, int no) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr int Q = 4096 / T;  // elements of a 64 x 64 S per thread
  const int npairs = no * no;
  // Each elimination step: warp 0 alone finds the pivot (first max of
  // |re|+|im| in column k, as LAPACK izamax), swaps it into row k, keeps
  // column k and scales row k by 1/p (= conj(p)/|p|^2); then every thread
  // updates its fixed elements.  Two block barriers per step.
  int my_i[Q], my_j[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int e = tid + q * T;
    my_i[q] = e < npairs ? e / no : -1;
    my_j[q] = e < npairs ? e - (e / no) * no : 0;
  }
  double2 det = make_double2(1.0, 0.0);
  for (int k = 0; k < no; ++k) {
    if (warp == 0) {
      double best = -1.0;
      int bi = k;
      for (int r = k + lane; r < no; r += 32) {
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
      const int pv = bi;
      if (pv != k)
        for (int j = lane; j < no; j += 32) {
          const double2 t0 = S[k * no + j];
          S[k * no + j] = S[pv * no + j];
          S[pv * no + j] = t0;
        }
      __syncwarp();
      const double2 pk = S[k * no + k];
      const double inv = 1.0 / (pk.x * pk.x + pk.y * pk.y);
      const double2 ipk = make_double2(pk.x * inv, -pk.y * inv);
      for (int i = lane; i < no; i += 32) colk[i] = S[i * no + k];
      __syncwarp();
      for (int j = lane; j < no; j += 32) S[k * no + j] = (j == k) ? ipk : cmul(S[k * no + j], ipk);
      if (lane == 0) {
        perm[k] = pv;
        *ipk_s = ipk;
        det = cmul(det, pk);
        if (pv != k) det = make_double2(-det.x, -det.y);
      }
    }
    __syncthreads();
    const double2 ipk = *ipk_s;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int i = my_i[q], j = my_j[q];
      if (i < 0 || i == k) continue;
      const double2 f = colk[i];
      if (j == k) {
        const double2 t0 = cmul(f, ipk);
        S[i * no + j] = make_double2(-t0.x, -t0.y);
      } else {
        S[i * no + j] = csub(S[i * no + j], cmul(f, S[k * no + j]));
      }
    }
    __syncthreads();
  }
  // undo the row interchanges as column interchanges, last first (rows independent)
  for (int i = tid; i < no; i += T)
    for (int k = no - 1; k >= 0; --k) {
      const int pv = perm[k];
      if (pv != k) {
        const double2 t0 = S[i * no + k];
        S[i * no + k] = S[i * no + pv];
        S[i * no + pv] = t0;
      }
    }
  __syncthreads();
  return det;
}

// mode 0: the whole computation; 1: S = C^T W only, into a.sbuf; 2: Theta
// and its outputs from S^-1 in a.sbuf (the inverse and det by gj_kernel).
// T threads: 256, or 512 where the staging allows one CTA per SM only (each
// warp then owns one column tile instead of up to two).
template <int T>
__device__ __forceinline__ void green_body(const GreenArgs& a, int mode, int w, int sct) {
  extern __shared__ double2 sm[];
  const GreenSector& S_ = a.sec[sct];
  const int N = a.N, no = S_.no, tid = threadIdx.x;
  constexpr int NW = T / 32;                 // warps
  constexpr int SL = (16 + NW - 1) / NW;     // column tiles per warp (2 No <= 128: 16 tiles)

  double2* S = sm;                          // no*no
  double2* colk = S + no * no;              // 64
  // two buffers each of walker rows and trial rows (chunk c in buffer c & 1);
  // walker rows at a stride of sd doubles, sd = 4 (mod 16): the 8-byte
  // fragment loads of a warp (8 rows x 4 columns, or 4 rows x 8 columns) then
  // take the minimum two shared-memory wavefronts
  const int nc2_ = 2 * no;
  const int sd = nc2_ + ((20 - nc2_ % 16) % 16);
  const int sbuf_ = kRowChunk * (sd / 2);  // double2 per buffer
  double2* stage = colk + 64;                                            // 2 x sbuf_
  double* moc = reinterpret_cast<double*>(stage + 2 * sbuf_);             // 2 x kRowChunk*no
  double2* tstage = reinterpret_cast<double2*>(moc + 2 * kRowChunk * no);
  const int ts = no + 1;  // padded row stride of tstage (conflict-free column reads)
  __shared__ double red[2 * (T / 32)];
  __shared__ int perm[64];

  const double2* Wg =
      reinterpret_cast<const double2*>(S_.walk) + (long long)w * N * no;

  // ---- S = C^T W on the FP64 tensor cores ----------------------------------
  // As real matrices: S (No x 2No, (re, im) interleaved) = C^T (No x N) times
  // W (N x 2No, the complex walker viewed as doubles).  mma.m8n8k4 tiles: warp
  // w owns column tiles w and w + 8 and every row tile, so each B fragment is
  // loaded once per k-step.  Rows of W and C are staged 32 at a time.
  const int warp = tid >> 5, lane = tid & 31;
  const int nc2 = 2 * no;
  const int mtiles = (no + 7) >> 3, ntiles = (nc2 + 7) >> 3;  // <= 8, <= 16
  const int nchunks = (N + kRowChunk - 1) / kRowChunk;
  // chunk c of the walker rows (and, with_mo, of the trial rows) into buffer c & 1
  auto load_chunk = [&](int c, bool with_mo) {
    const int p0 = c * kRowChunk, rows = min(kRowChunk, N - p0);
    double2* st = stage + (c & 1) * sbuf_;
    double* mc = moc + (c & 1) * kRowChunk * no;
    for (int e = tid; e < rows * no; e += T) {
      const int r = e / no;
      cp_async16(&st[r * (sd / 2) + (e - r * no)], &Wg[(long long)p0 * no + e]);
      if (with_mo) cp_async8(&mc[e], &S_.mo[(long long)p0 * no + e]);
    }
    cp_async_commit();
  };
  double2* sg = a.sbuf ? reinterpret_cast<double2*>(a.sbuf) + ((long long)sct * a.W + w) * a.sstride
                       : nullptr;
  const int npairs = no * no;
  if (mode != 2) {
  double sacc[SL][8][2];
#pragma unroll
  for (int sl = 0; sl < SL; ++sl)
#pragma unroll
    for (int mi = 0; mi < 8; ++mi) sacc[sl][mi][0] = sacc[sl][mi][1] = 0.0;
  load_chunk(0, true);
  for (int c = 0; c < nchunks; ++c) {
    const int p0 = c * kRowChunk, rows = min(kRowChunk, N - p0);
    if (c + 1 < nchunks) load_chunk(c + 1, true);
    else cp_async_commit();  // an empty group keeps the wait count uniform
    cp_async_wait1();
    __syncthreads();
    const double* stageD = reinterpret_cast<const double*>(stage + (c & 1) * sbuf_);
    const double* mocc = moc + (c & 1) * kRowChunk * no;
    for (int kk = 0; kk < rows; kk += 4) {
      const int kr = kk + (lane & 3);
      const bool kin = kr < rows;
      double afr[8];
#pragma unroll
      for (int mi = 0; mi < 8; ++mi) {
        const int m = mi * 8 + (lane >> 2);
        afr[mi] = (mi < mtiles && kin && m < no) ? mocc[kr * no + m] : 0.0;
      }
#pragma unroll
      for (int sl = 0; sl < SL; ++sl) {
        const int ni = warp + sl * NW;
        if (ni < ntiles) {  // warp-uniform
          const int n = ni * 8 + (lane >> 2);
          const double b = (kin && n < nc2) ? stageD[kr * sd + n] : 0.0;
#pragma unroll
          for (int mi = 0; mi < 8; ++mi)
            if (mi < mtiles) dmma_8x8x4(sacc[sl][mi][0], sacc[sl][mi][1], afr[mi], b);
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int sl = 0; sl < SL; ++sl) {
    const int ni = warp + sl * NW;
    if (ni < ntiles) {
#pragma unroll
      for (int mi = 0; mi < 8; ++mi) {
        const int i = mi * 8 + (lane >> 2), j = ni * 4 + (lane & 3);
        if (mi < mtiles && i < no && j < no) {
          const double2 v = make_double2(sacc[sl][mi][0], sacc[sl][mi][1]);
          if (mode == 1)
            sg[i * no + j] = v;
          else
            S[i * no + j] = v;
        }
      }
    }
  }
  if (mode == 1) return;
  __syncthreads();
  }  // mode != 2
  if (mode == 2) {  // S^-1 from gj_kernel
    for (int e = tid; e < npairs; e += T) S[e] = sg[e];
    __syncthreads();
  } else {

  // ---- Gauss-Jordan inverse with partial pivoting, det ----------------------
  __shared__ double2 ipk_s;
  const double2 det = gauss_jordan_cta<T>(S, colk, perm, &ipk_s, no);
  if (tid == 0 && a.wscal) {
    a.wscal[(long long)w * 16 + 4 + 2 * sct] = det.x;
    a.wscal[(long long)w * 16 + 5 + 2 * sct] = det.y;
  }
  }  // mode 0: inverse in this CTA

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
  load_chunk(0, false);
  for (int c = 0; c < nchunks; ++c) {
    const int p0 = c * kRowChunk, rows = min(kRowChunk, N - p0);
    // walker rows of the next chunk stream in while this one is processed
    if (c + 1 < nchunks) load_chunk(c + 1, false);
    else cp_async_commit();
    cp_async_wait1();
    __syncthreads();
    const double* stageD = reinterpret_cast<const double*>(stage + (c & 1) * sbuf_);
    // Theta rows (N x 2No real) = W rows (N x 2No) times the real form of
    // S^-1: R[2i][2j] = R[2i+1][2j+1] = Re s_ij, R[2i][2j+1] = Im s_ij,
    // R[2i+1][2j] = -Im s_ij, generated in the B fragments
    {
      const int rtiles = (rows + 7) >> 3;  // <= 4
      double tacc[SL][4][2];
#pragma unroll
      for (int sl = 0; sl < SL; ++sl)
#pragma unroll
        for (int ri = 0; ri < 4; ++ri) tacc[sl][ri][0] = tacc[sl][ri][1] = 0.0;
      for (int kk = 0; kk < nc2; kk += 4) {
        const int k = kk + (lane & 3);
        const bool kin = k < nc2;
        double afr[4];
#pragma unroll
        for (int ri = 0; ri < 4; ++ri) {
          const int r = ri * 8 + (lane >> 2);
          afr[ri] = (ri < rtiles && kin && r < rows) ? stageD[r * sd + k] : 0.0;
        }
#pragma unroll
        for (int sl = 0; sl < SL; ++sl) {
          const int ni = warp + sl * NW;
          if (ni < ntiles) {  // warp-uniform
            const int n = ni * 8 + (lane >> 2);
            double b = 0.0;
            if (kin && n < nc2) {
              const double2 sv = S[(k >> 1) * no + (n >> 1)];
              b = (k & 1) == 0 ? ((n & 1) == 0 ? sv.x : sv.y) : ((n & 1) == 0 ? -sv.y : sv.x);
            }
#pragma unroll
            for (int ri = 0; ri < 4; ++ri)
              if (ri < rtiles) dmma_8x8x4(tacc[sl][ri][0], tacc[sl][ri][1], afr[ri], b);
          }
        }
      }
#pragma unroll
      for (int sl = 0; sl < SL; ++sl) {
        const int ni = warp + sl * NW;
        if (ni >= ntiles) continue;
#pragma unroll
        for (int ri = 0; ri < 4; ++ri) {
          const int r = ri * 8 + (lane >> 2), j = ni * 4 + (lane & 3);
          if (ri < rtiles && r < rows && j < no) {
            const double2 sv = make_double2(tacc[sl][ri][0], tacc[sl][ri][1]);
            tstage[r * ts + j] = sv;
            if (th) th[(long long)(p0 + r) * no + j] = sv;
            if (S_.rh1) {
              const double h = S_.rh1[(long long)j * N + p0 + r];
              e1.x = fma(sv.x, h, e1.x);
              e1.y = fma(sv.y, h, e1.y);
            }
          }
        }
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

// Warp 0 of gj_kernel: the pivot among this lane's two candidate rows (lane,
// lane + 32) and the other lanes': the largest |re|+|im|, the lowest row
// among equal values (LAPACK izamax).  One 64-bit max-reduction over keys
// that hold the magnitude's bits above the row number: a non-negative
// double's bit pattern orders like its value, so the key order is the
// magnitude order except between values within 128 ulps of each other,
// which go to the lower row.  Non-candidates have key 0.
__device__ __forceinline__ int gj_pivot(double2 v0, double2 v1, bool ok0, bool ok1, int lane) {
  auto key = [](double2 v, int row) -> unsigned long long {
    const unsigned long long b = (unsigned long long)__double_as_longlong(fabs(v.x) + fabs(v.y));
    return (b & ~127ull) | 64ull | (unsigned long long)(63 - row);
  };
  unsigned long long k = ok0 ? key(v0, lane) : 0ull;
  const unsigned long long k1 = ok1 ? key(v1, lane + 32) : 0ull;
  k = k1 > k ? k1 : k;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long ok = __shfl_xor_sync(0xffffffffu, k, o);
    k = ok > k ? ok : k;
  }
  return 63 - (int)(k & 63ull);
}

// Gauss-Jordan inverse and det of S = C^T W held in sbuf, one CTA per
// (walker, sector), in place in one shared-memory copy of S, with one block
// barrier per elimination step (partial pivoting, pivot = largest |re|+|im|
// in the column).
//  * Rows are never swapped: the pivot row r_k of step k stays in place and
//    the inverse is unscrambled once at the end, S^-1[i][r_k] = X[r_i][k].
//  * Pivot rows are scaled lazily: row r_k keeps its unscaled values U (the
//    true row is U / p_k).  Every later update of that row has the same form
//    on U (the update is linear in the row), so no thread writes row r_k
//    during step k, and each thread reads the pivot row straight from S and
//    scales the elements it needs.  The row scales are applied when the
//    inverse is unscrambled.
//  * The multipliers of step k (column k before the step) come from a copy
//    that warp 0 wrote during step k-1, when it computed that column, so the
//    owners of column k may overwrite it during step k.
//  * Warp 0 computes the new column k+1, its pivot (over the rows not yet
//    used) and the reciprocal; warps 1..7 update every other column, each
//    thread one column and a stride of rows.  Rows are stored with an odd
//    stride (ld = no | 1 double2), so a warp reading a column hits distinct
//    banks.  det = product of the pivots times the permutation's sign.
// At most 64 rows (no <= 64, checked by the caller).
__device__ __forceinline__ void gj_body(int W, int no0, int no1, double* sbuf, long long sstride,
                                        int bstride, double* wscal, int w, int sct) {
  extern __shared__ double2 gsm[];
  const int no = sct ? no1 : no0;
  const int ld = no | 1;
  const int nn = no * no;
  double2* const A = gsm;
  double2* const pcol = gsm + bstride;  // [2][64]: multipliers of the step, by parity
  __shared__ double2 ipks[64];          // 1 / pivot of each step (the lazy row scales)
  __shared__ int piv[64];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  double2* g = reinterpret_cast<double2*>(sbuf) + ((long long)sct * W + w) * sstride;
  for (int e = tid; e < nn; e += kGreenThreads) {
    const int i = e / no;
    A[i * ld + (e - i * no)] = g[e];
  }
  __syncthreads();

  const double2 zero = make_double2(0.0, 0.0);
  const bool in0 = lane < no, in1 = lane + 32 < no;
  bool used0 = false, used1 = false;  // warp 0: rows lane, lane + 32 already pivots
  double2 det = make_double2(1.0, 0.0);
  // warp 0: the pivot of column 0 and its value, from the column in registers
  auto pivot = [&](double2 v0, double2 v1, int col) {
    const int rn = gj_pivot(v0, v1, in0 && !used0, in1 && !used1, lane);
    const double2 sel = rn < 32 ? v0 : v1;
    const double2 p = make_double2(__shfl_sync(0xffffffffu, sel.x, rn & 31),
                                   __shfl_sync(0xffffffffu, sel.y, rn & 31));
    const double inv = 1.0 / (p.x * p.x + p.y * p.y);
    if (lane == (rn & 31)) (rn < 32 ? used0 : used1) = true;
    if (lane == 0) {
      piv[col] = rn;
      ipks[col] = make_double2(p.x * inv, -p.y * inv);
      det = cmul(det, p);
    }
  };
  if (warp == 0) {
    const double2 v0 = in0 ? A[lane * ld] : zero, v1 = in1 ? A[(lane + 32) * ld] : zero;
    if (in0) pcol[lane] = v0;
    if (in1) pcol[lane + 32] = v1;
    pivot(v0, v1, 0);
  }
  __syncthreads();

  // warps 1..7: thread tid - 32 = g * no + j owns column j, rows g, g + G, ...
  // (G = 224 / no row groups; threads beyond G * no idle)
  constexpr int TW = kGreenThreads - 32;
  const int nd = no > 0 ? no : 1;
  const int G = TW / nd;
  const int tu = tid - 32;
  const int jc = tu % nd, g0 = tu / nd;
  const bool upd = warp > 0 && g0 < G;
  for (int k = 0; k < no; ++k) {
    const int cur = k & 1;
    const double2* pc = pcol + cur * 64;
    const int r = piv[k];
    const double2 ipk = ipks[k];
    const int c = k + 1;
    if (warp == 0) {
      if (c < no) {
        // the new column c (row r keeps its unscaled values), the next step's
        // multipliers, then the pivot among the unused rows
        const double2 prc = cmul(A[r * ld + c], ipk);
        double2 v0 = zero, v1 = zero;
        if (in0) {
          const int i = lane;
          v0 = A[i * ld + c];
          if (i != r) {
            v0 = csub(v0, cmul(pc[i], prc));
            A[i * ld + c] = v0;
          }
          pcol[(cur ^ 1) * 64 + i] = v0;
        }
        if (in1) {
          const int i = lane + 32;
          v1 = A[i * ld + c];
          if (i != r) {
            v1 = csub(v1, cmul(pc[i], prc));
            A[i * ld + c] = v1;
          }
          pcol[(cur ^ 1) * 64 + i] = v1;
        }
        pivot(v0, v1, c);
      }
    } else if (upd && jc != c) {
      const int j = jc;
      if (j == k) {  // the pivot column: -(multiplier) / p, and 1 in the (lazy) pivot row
        for (int i = g0; i < no; i += G) {
          const double2 t0 = cmul(pc[i], ipk);
          A[i * ld + j] = (i == r) ? make_double2(1.0, 0.0) : make_double2(-t0.x, -t0.y);
        }
      } else {
        const double2 prj = cmul(A[r * ld + j], ipk);
        for (int i = g0; i < no; i += G)
          if (i != r) A[i * ld + j] = csub(A[i * ld + j], cmul(pc[i], prj));
      }
    }
    __syncthreads();
  }
  // unscramble with the row scales: S^-1[i][r_k] = X[r_i][k] = A[r_i][k] / p_i
  for (int e = tid; e < nn; e += kGreenThreads) {
    const int i = e / no, k = e - (e / no) * no;
    g[i * no + piv[k]] = cmul(A[piv[i] * ld + k], ipks[i]);
  }
  if (tid == 0) {
    // sign of the permutation k -> r_k: (-1)^(no - cycles)
    unsigned long long seen = 0ull;
    int cycles = 0;
    for (int s0 = 0; s0 < no; ++s0) {
      if (seen >> s0 & 1ull) continue;
      ++cycles;
      for (int t = s0; !(seen >> t & 1ull); t = piv[t]) seen |= 1ull << t;
    }
    if ((no - cycles) & 1) det = make_double2(-det.x, -det.y);
    if (wscal) {
      wscal[(long long)w * 16 + 4 + 2 * sct] = det.x;
      wscal[(long long)w * 16 + 5 + 2 * sct] = det.y;
    }
  }
}

template <int T>
__global__ void __launch_bounds__(T) green_kernel(GreenArgs a, int mode) {
  green_body<T>(a, mode, blockIdx.x, blockIdx.y);
}

__global__ void __launch_bounds__(kGreenThreads) green_kernel_grouped(const GreenArgs* A, BlockMap m,
                                                                      int mode) {
  int local;
  const GreenArgs& a = A[block_owner(m, blockIdx.x, local)];
  green_body<kGreenThreads>(a, mode, local % a.W, local / a.W);
}

__global__ void __launch_bounds__(kGreenThreads, 4)
    gj_kernel(int W, int no0, int no1, double* sbuf, long long sstride, int bstride, double* wscal) {
  gj_body(W, no0, no1, sbuf, sstride, bstride, wscal, blockIdx.x, blockIdx.y);
}

__global__ void __launch_bounds__(kGreenThreads, 4) gj_kernel_grouped(const GjArgs* A, BlockMap m) {
  int local;
  const GjArgs& a = A[block_owner(m, blockIdx.x, local)];
  gj_body(a.W, a.no0, a.no1, a.sbuf, a.sstride, a.bstride, a.wscal, local % a.W, local / a.W);
}

// one compiled copy for the solo and the grouped kernel (identical rounding)
__device__ __noinline__ void ovlp_body(int W, int ns, int mult, const double* wscal, double* out,
                                          int out_stride, int w) {
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

__global__ void ovlp_combine_kernel(int W, int ns, int mult, const double* wscal, double* out,
                                    int out_stride) {
  ovlp_body(W, ns, mult, wscal, out, out_stride, blockIdx.x * blockDim.x + threadIdx.x);
}

__global__ void ovlp_combine_grouped(const OvlpArgs* A, BlockMap m) {
  int local;
  const OvlpArgs& a = A[block_owner(m, blockIdx.x, local)];
  ovlp_body(a.W, a.ns, a.mult, a.wscal, a.out, a.out_stride, local * blockDim.x + threadIdx.x);
}

}  // namespace

size_t green_smem_bytes(int nomax) {
  const int sdmax = 2 * nomax + ((20 - (2 * nomax) % 16) % 16);  // padded walker-row stride (doubles)
  return (size_t(nomax) * nomax + 64) * sizeof(double2) + 2 * size_t(kRowChunk) * sdmax * sizeof(double) +
         2 * size_t(kRowChunk) * nomax * sizeof(double) + size_t(kRowChunk) * (nomax + 1) * sizeof(double2);
}

// S with row stride nomax | 1 and two columns of multipliers
size_t gj_smem_bytes(int nomax) { return (size_t(nomax) * (nomax | 1) + 128) * sizeof(double2); }

cudaError_t launch_green_grouped(const GreenArgs* args, const BlockMap& m, int mode, size_t smem,
                                 cudaStream_t st) {
  ProfScope ps(K_GREEN, st);
  cudaError_t e = cudaFuncSetAttribute(green_kernel_grouped, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  green_kernel_grouped<<<m.start[m.n], kGreenThreads, smem, st>>>(args, m, mode);
  return cudaGetLastError();
}

cudaError_t launch_gj_grouped(const GjArgs* args, const BlockMap& m, size_t smem, cudaStream_t st) {
  cudaError_t e = cudaFuncSetAttribute(gj_kernel_grouped, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  ProfScope ps(K_GREEN, st);
  gj_kernel_grouped<<<m.start[m.n], kGreenThreads, smem, st>>>(args, m);
  return cudaGetLastError();
}

cudaError_t launch_ovlp_grouped(const OvlpArgs* args, const BlockMap& m, cudaStream_t st) {
  ProfScope ps(K_MISC, st);
  ovlp_combine_grouped<<<m.start[m.n], 256, 0, st>>>(args, m);
  return cudaGetLastError();
}

cudaError_t launch_green(const GreenArgs& a, cudaStream_t st) {
  int nomax = 0;
  for (int s = 0; s < a.ns; ++s) nomax = a.sec[s].no > nomax ? a.sec[s].no : nomax;
  const size_t smem = green_smem_bytes(nomax);
  // staging above ~113 KB leaves one CTA per SM: 16 warps instead of 8 then
  const bool wide = smem > 113 * 1024;
  auto kernel = wide ? green_kernel<2 * kGreenThreads> : green_kernel<kGreenThreads>;
  const int threads = wide ? 2 * kGreenThreads : kGreenThreads;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid(a.W, a.ns);
  ProfScope ps(K_GREEN, st);
  bool need_theta = a.gpl || a.gplb[0];
  for (int s = 0; s < a.ns; ++s)
    need_theta = need_theta || a.sec[s].theta || a.sec[s].gout || a.sec[s].rh1 || a.sec[s].gtb[0];
  if (!a.sbuf || !need_theta) {  // one kernel: S, its inverse and det, Theta and outputs
    kernel<<<grid, threads, smem, st>>>(a, 0);
    return cudaGetLastError();
  }
  // S into a.sbuf; warp-level inverse and det; Theta and its outputs
  kernel<<<grid, threads, smem, st>>>(a, 1);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  const int bstride = nomax * (nomax | 1);
  const size_t gsmem = gj_smem_bytes(nomax);
  if ((e = cudaFuncSetAttribute(gj_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gsmem)) !=
      cudaSuccess)
    return e;
  gj_kernel<<<grid, kGreenThreads, gsmem, st>>>(a.W, a.sec[0].no, a.ns > 1 ? a.sec[1].no : 0,
                                                a.sbuf, a.sstride, bstride, a.wscal);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  kernel<<<grid, threads, smem, st>>>(a, 2);
  return cudaGetLastError();
}

cudaError_t launch_ovlp_combine(int W, int ns, int mult, const double* wscal, double* out,
                                int out_stride, cudaStream_t st) {
  ProfScope ps(K_MISC, st);
  ovlp_combine_kernel<<<(W + 255) / 256, 256, 0, st>>>(W, ns, mult, wscal, out, out_stride);
  return cudaGetLastError();
}

}  // namespace afq
