// Persistent tcgen05 GEMM with split-BF16 operands (sm_100a).
//
//   C[b] (M x N, fp32 in TMEM) = sum_{p in pairs} A_{pa[p]}[b] (M x K) * B_{pb[p]}[b]^T (N x K)
//
// A value x is stored as bf16 pieces x = x_0 + x_1 (+ x_2); the pair list
// {(0,0),(0,1),(1,0)} is the "BF16x3" product (about 16 significant bits),
// {(0,0),(0,1),(1,0),(0,2),(1,1),(2,0)} with three pieces about 24 bits.
//
// Roles (64 + 128*EG threads, one CTA per SM, persistent over tiles):
//   warp 0      TMA producer: 128-byte-swizzled K-major tiles into a STAGES ring
//   warp 1      TMEM allocator; lane 0 issues tcgen05.mma into one of two
//               accumulators and commits stage/accumulator barriers
//   warps 2..5  epilogue: tcgen05.ld rows of the finished accumulator (one TMEM
//               lane per thread) and hand 32 columns at a time to the functor
//   warps 6..   (EG = 2, 3) more epilogue warpgroups.  The CTA's tiles then
//               rotate over the groups, tile t in accumulator t % EG for all its
//               K chunks, so a long epilogue of one tile runs while the other
//               groups drain and process the next tiles
// All waits are bounded; on timeout the CTA records an error and unwinds.
#pragma once

#include "common.cuh"
#include "umma.cuh"

namespace afq {

constexpr int kUBM = 128;  // UMMA M
constexpr int kUBK = 64;   // K per stage (128 bytes of bf16: one swizzle row)

struct UmmaShape {
  int stages;        // depth of the shared-memory ring (host-chosen)
  int a_batched;     // 0: A is shared by every batch (tensor map batch extent 1)
  int M, N, K;       // per batch
  int batch;
  int mt, nt;        // tiles along M and N
  int a_step, b_step;  // rows of A / B advanced per tile (<= 128 / BN)
  int ksplit, kchunk;  // K split into ksplit chunks of kchunk (multiple of 64)
  int npa, npb;      // pieces of A and B
  int npairs;
  int pa[6], pb[6];
  int ngroups;       // 1, or 2: pair 0 (the hi x hi product) accumulates apart from the rest
  int kc;            // K blocks per accumulator chunk (0: the whole K of a tile in one chunk)
  int epi_bytes;     // epilogue scratch per epilogue warpgroup (bytes, multiple of 256)
  int reverse;       // 1: tiles in reverse order (the last batch first)
  int* err;          // device error flag (set to 1 on a timed-out wait)
};

// Where an epilogue reads the finished accumulator of its row: straight from
// TMEM (one chunk; two groups summed) or from the FP32 shared-memory row that
// summed the chunks with round-to-nearest adds.
struct AccSrc {
  uint32_t taddr;
  int ngroups, bn;
  const float* srow;  // nullptr: read TMEM
  __device__ __forceinline__ void load16(int col, float (&v)[16]) const {
    if (srow) {
#pragma unroll
      for (int i = 0; i < 16; ++i) v[i] = srow[col + i];
    } else {
      acc_ld16(taddr + col, ngroups, bn, v);
    }
  }
};

// FP32 staging for chunked accumulation: one (BN+1)-float row per TMEM lane
__host__ __device__ inline size_t umma_chunk_stage_bytes(int bn) {
  return size_t(128) * (bn + 1) * sizeof(float);
}

template <class Epi>
struct UmmaParams {
  CUtensorMap ta[3];
  CUtensorMap tb[3];
  UmmaShape s;
  Epi epi;
};

// TMEM columns for nbuf (two, or one per epilogue warpgroup) accumulator
// buffers of ngroups x bn fp32 columns
__host__ __device__ constexpr int umma_tmem_cols(int bn, int ngroups = 1, int nbuf = 2) {
  int c = 32;
  while (c < nbuf * ngroups * bn) c <<= 1;
  return c;
}

constexpr size_t kUmmaSmemBudget = 227 * 1024;

__host__ __device__ inline size_t umma_stage_bytes(int bn, int npa, int npb) {
  return size_t(npa) * kUBM * 128 + size_t(npb) * bn * 128;
}
__host__ __device__ inline size_t umma_smem_bytes(int bn, int stages, int npa, int npb,
                                                  size_t extra) {
  return 1024 /*alignment slack*/ + size_t(stages) * umma_stage_bytes(bn, npa, npb) +
         256 /*barriers*/ + extra;
}
// deepest ring (<= 8) that fits next to `extra` bytes of epilogue scratch
inline int umma_pick_stages(int bn, int npa, int npb, size_t extra) {
  for (int st = 8; st >= 2; --st)
    if (umma_smem_bytes(bn, st, npa, npb, extra) <= kUmmaSmemBudget) return st;
  return 0;
}

// Several independent GEMMs of one kind (one per fragment of a batch) in one
// persistent launch: entry e owns global tiles [start[e], start[e+1]).  The
// entries share BN, the number of bf16 pieces, the accumulator groups, the
// epilogue scratch and the ring depth; everything else (tensor maps, sizes,
// epilogue pointers, error flag) is per entry.  The entries live in device
// memory (their tensor maps are read by TMA from global memory).
constexpr int kUmmaMaxGroup = 64;

template <class Epi>
struct UmmaGroup {
  const UmmaParams<Epi>* entries;
  int n;
  int stages;
  int start[kUmmaMaxGroup + 1];
};

// Tile sources of the kernel body: one GEMM from the kernel parameter, or a
// group of GEMMs from device memory (entry found by binary search).
template <class Epi>
struct UmmaOne {
  const UmmaParams<Epi>& P;
  __device__ int stages() const { return P.s.stages; }
  __device__ int tiles() const { return P.s.batch * P.s.ksplit * P.s.mt * P.s.nt; }
  __device__ const UmmaParams<Epi>& first() const { return P; }
  __device__ const UmmaParams<Epi>& entry(int it, int& local) const {
    local = it;
    return P;
  }
};

template <class Epi>
struct UmmaMany {
  const UmmaGroup<Epi>& G;
  __device__ int stages() const { return G.stages; }
  __device__ int tiles() const { return G.start[G.n]; }
  __device__ const UmmaParams<Epi>& first() const { return G.entries[0]; }
  __device__ const UmmaParams<Epi>& entry(int it, int& local) const {
    int lo = 0, hi = G.n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (G.start[mid] <= it) lo = mid;
      else hi = mid - 1;
    }
    local = it - G.start[lo];
    return G.entries[lo];
  }
};

template <int BN, class Epi, int EG, class Src>
__device__ __forceinline__ void umma_body(const Src& src) {
  static_assert(EG >= 1 && EG <= 3, "one to three epilogue warpgroups");
  constexpr int NBUF = EG > 2 ? EG : 2;  // accumulator buffers
  static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "UMMA N for M=128");
  static_assert(umma_tmem_cols(BN) <= 512, "two accumulators must fit in TMEM");
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const UmmaParams<Epi>& P0 = src.first();
  const int ST = src.stages();
  const int npa = P0.s.npa, npb = P0.s.npb, ngrp = P0.s.ngroups, epi_bytes = P0.s.epi_bytes;
  const uint32_t a_bytes = kUBM * 128, b_bytes = BN * 128;
  const uint32_t stage_bytes = npa * a_bytes + npb * b_bytes;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + ST * stage_bytes);
  uint64_t* empty = full + ST;
  uint64_t* accf = empty + ST;
  uint64_t* acce = accf + NBUF;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acce + NBUF);
  volatile int* abort_s = reinterpret_cast<volatile int*>(tmem_slot + 1);
  uint8_t* epi_smem = reinterpret_cast<uint8_t*>(full) + 256;  // epilogue scratch
  const uint32_t kCols = umma_tmem_cols(BN, ngrp, NBUF);
  const uint32_t acc_stride = (uint32_t)(ngrp * BN);  // columns per accumulator buffer

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < ST; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < NBUF; ++b) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], 4);
    }
    *abort_s = 0;
    fence_barrier_init();
  }
  if (warp == 0 && lane == 0) {
    for (int i = 0; i < npa; ++i) prefetch_tmap(&P0.ta[i]);
    for (int i = 0; i < npb; ++i) prefetch_tmap(&P0.tb[i]);
  }
  if (warp == 1) tmem_alloc(tmem_slot, kCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tmem_slot;

  const int tiles = src.tiles();
  auto fail = [&](int* err) {
    atomicExch(err, 1);
    *abort_s = 1;
  };
  // (global iteration) -> entry, tile of the entry, and its coordinates
  struct TileAt {
    int z, mti, nti, b, k0, KB;
  };
  auto locate = [&](const UmmaShape& S, int local) {
    const int etiles = S.batch * S.ksplit * S.mt * S.nt;
    const int tile = S.reverse ? etiles - 1 - local : local;
    TileAt t;
#ifdef AFQ_CHECKS
    // debug builds: a tile outside its GEMM (a corrupt work list) is reported
    // (flag value 2) and skipped by every role alike (KB = 0)
    if (local < 0 || local >= etiles) {
      atomicExch(S.err, 2);
      t.z = t.mti = t.nti = t.b = t.k0 = t.KB = 0;
      return t;
    }
#endif
    t.nti = tile % S.nt;
    const int rest = tile / S.nt;
    t.mti = rest % S.mt;
    t.z = rest / S.mt;
    t.b = t.z / S.ksplit;
    t.k0 = (t.z % S.ksplit) * S.kchunk;
    t.KB = (min(S.kchunk, S.K - t.k0) + kUBK - 1) / kUBK;
    return t;
  };

  if (warp == 0) {
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      for (int it_ = blockIdx.x; it_ < tiles && !*abort_s; it_ += gridDim.x) {
        int local;
        const UmmaParams<Epi>& P = src.entry(it_, local);
        const UmmaShape& S = P.s;
        const TileAt t = locate(S, local);
        bool ok = true;
        for (int kb = 0; kb < t.KB; ++kb) {
          if (!mbar_wait(&empty[stage], phase ^ 1)) { fail(S.err); ok = false; break; }
          mbar_arrive_expect_tx(&full[stage], stage_bytes);
          uint8_t* sa = smem + stage * stage_bytes;
          uint8_t* sb = sa + npa * a_bytes;
          for (int i = 0; i < npa; ++i)
            tma_load_3d(sa + i * a_bytes, &P.ta[i], &full[stage], t.k0 + kb * kUBK,
                        t.mti * S.a_step, S.a_batched ? t.b : 0);
          for (int j = 0; j < npb; ++j)
            tma_load_3d(sb + j * b_bytes, &P.tb[j], &full[stage], t.k0 + kb * kUBK,
                        t.nti * S.b_step, t.b);
          if (++stage == ST) { stage = 0; phase ^= 1; }
        }
        if (!ok) break;
      }
      // drain: wait (bounded) until the MMA side released every stage we filled
      for (int s = 0; s < ST; ++s) {
        if (!mbar_wait(&empty[stage], phase ^ 1)) { fail(P0.s.err); break; }
        if (++stage == ST) { stage = 0; phase ^= 1; }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t idesc = instr_desc(kUBM, BN, 1);
      int stage = 0;
      uint32_t phase = 0;
      int it = 0, t = 0;
      uint32_t uses[NBUF] = {};  // EG > 1: chunks accumulated so far in each buffer
      for (int it_ = blockIdx.x; it_ < tiles && !*abort_s; it_ += gridDim.x, ++t) {
        int local;
        const UmmaParams<Epi>& P = src.entry(it_, local);
        const UmmaShape& S = P.s;
        const TileAt tl = locate(S, local);
        const int KB = tl.KB;
        if (KB == 0) continue;  // (debug builds: a tile skipped by every role)
        const int kc = S.kc > 0 ? S.kc : KB;
        bool ok = true;
        for (int c0 = 0; c0 < KB && ok; c0 += kc, ++it) {
          const int buf = EG > 1 ? (t % EG) : (it & 1);
          const uint32_t use = EG > 1 ? uses[buf]++ : (uint32_t)(it >> 1);
          if (!mbar_wait(&acce[buf], (use & 1) ^ 1)) { fail(S.err); ok = false; break; }
          tc_fence_after();
          const uint32_t dt = tbase + buf * acc_stride;
          const int c1 = min(KB, c0 + kc);
          for (int kb = c0; kb < c1; ++kb) {
            if (!mbar_wait(&full[stage], phase)) { fail(S.err); ok = false; break; }
            tc_fence_after();
            const uint8_t* sa = smem + stage * stage_bytes;
            const uint8_t* sb = sa + npa * a_bytes;
            for (int p = 0; p < S.npairs; ++p) {
              const uint64_t ad = smem_desc_sw128(sa + S.pa[p] * a_bytes);
              const uint64_t bd = smem_desc_sw128(sb + S.pb[p] * b_bytes);
              // group 0: pair 0 alone; group 1 (if any): the remaining pairs
              const int grp = (ngrp == 2 && p > 0) ? 1 : 0;
              const int first = (p == 0) || (ngrp == 2 && p == 1);
#pragma unroll
              for (int ks = 0; ks < kUBK / 16; ++ks)
                umma_bf16(dt + grp * BN, ad + 2 * ks, bd + 2 * ks, idesc,
                          (kb - c0) != 0 || ks != 0 || !first);
            }
            umma_commit(&empty[stage]);
            if (++stage == ST) { stage = 0; phase ^= 1; }
          }
          if (!ok) break;
          umma_commit(&accf[buf]);
        }
        if (!ok) break;
      }
    }
  } else {
    const int sub = warp & 3;
    const int eg = (warp - 2) >> 2;  // epilogue warpgroup
    const int row = sub * 32 + lane;
    uint8_t* escr = epi_smem + eg * epi_bytes;
    float* srow = reinterpret_cast<float*>(escr) + row * (BN + 1);
    int it = 0, t = 0;
    uint32_t uses = 0;  // EG = 2: chunks drained from this group's buffer so far
    bool ok = true;
    for (int it_ = blockIdx.x; it_ < tiles && ok; it_ += gridDim.x, ++t) {
      if (EG > 1 && (t % EG) != eg) continue;
      int local;
      const UmmaParams<Epi>& P = src.entry(it_, local);
      const UmmaShape& S = P.s;
      const TileAt tl = locate(S, local);
      const int KB = tl.KB;
      if (KB == 0) continue;
      const int kc = S.kc > 0 ? S.kc : KB;
      const int nch = (KB + kc - 1) / kc;
      for (int ch = 0; ch < nch; ++ch, ++it) {
        const int buf = EG > 1 ? eg : (it & 1);
        const uint32_t use = EG > 1 ? uses++ : (uint32_t)(it >> 1);
        if (!mbar_wait_abortable(&accf[buf], use & 1, abort_s)) { fail(S.err); ok = false; break; }
        tc_fence_after();
        const uint32_t taddr = tbase + ((uint32_t)(sub * 32) << 16) + buf * acc_stride;
        if (nch == 1) {
          // z = batch * ksplit + split
          P.epi.template tile<BN>(tl.z, tl.mti, tl.nti, row, AccSrc{taddr, ngrp, BN, nullptr}, S,
                                  escr);
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&acce[buf]);
        } else {
#pragma unroll 1
          for (int c = 0; c < BN / 16; ++c) {
            float v[16];
            acc_ld16(taddr + c * 16, ngrp, BN, v);
#pragma unroll
            for (int i = 0; i < 16; ++i)
              srow[c * 16 + i] = (ch == 0) ? v[i] : srow[c * 16 + i] + v[i];
          }
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&acce[buf]);
          if (ch == nch - 1)
            P.epi.template tile<BN>(tl.z, tl.mti, tl.nti, row, AccSrc{0u, 1, BN, srow}, S, escr);
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tbase, kCols);
  }
}

template <int BN, class Epi, int EG>
__global__ void __launch_bounds__(64 + 128 * EG, 1)
    umma_gemm_kernel(const __grid_constant__ UmmaParams<Epi> P) {
  umma_body<BN, Epi, EG>(UmmaOne<Epi>{P});
}

template <int BN, class Epi, int EG>
__global__ void __launch_bounds__(64 + 128 * EG, 1)
    umma_group_kernel(const __grid_constant__ UmmaGroup<Epi> G) {
  umma_body<BN, Epi, EG>(UmmaMany<Epi>{G});
}

// ---------------------------------------------------------------------------
// host side: tensor maps and launch
// ---------------------------------------------------------------------------
// 3-D bf16 tensor map: dims {K, rows, batch}; box {64, box_rows, 1}; SW128.
int make_tmap_bf16(CUtensorMap* map, const void* base, long long K, long long rows,
                   long long batch, long long row_stride_elems, long long batch_stride_elems,
                   int box_rows);

// P.s.stages must come from umma_pick_stages(BN, npa, npb, EG * P.s.epi_bytes).
template <int BN, int EG = 1, class Epi>
cudaError_t launch_umma(const UmmaParams<Epi>& P, int num_sms, cudaStream_t st) {
  const size_t smem = umma_smem_bytes(BN, P.s.stages, P.s.npa, P.s.npb, size_t(EG) * P.s.epi_bytes);
  if (P.s.stages < 2 || smem > kUmmaSmemBudget || (P.s.epi_bytes & 255) ||
      (EG > 2 ? EG : 2) * P.s.ngroups * BN > 512)
    return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(umma_gemm_kernel<BN, Epi, EG>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int tiles = P.s.batch * P.s.ksplit * P.s.mt * P.s.nt;
  const int grid = tiles < num_sms ? tiles : num_sms;
  umma_gemm_kernel<BN, Epi, EG><<<grid, 64 + 128 * EG, smem, st>>>(P);
  return cudaGetLastError();
}

// A group of GEMMs in one launch.  `shape0` is any entry's shape (host copy):
// pieces, accumulator groups and epilogue scratch are the same for all.
template <int BN, int EG = 1, class Epi>
cudaError_t launch_umma_group(const UmmaGroup<Epi>& G, const UmmaShape& shape0, int num_sms,
                              cudaStream_t st) {
  const size_t smem = umma_smem_bytes(BN, G.stages, shape0.npa, shape0.npb, size_t(EG) * shape0.epi_bytes);
  if (G.n < 1 || G.n > kUmmaMaxGroup || G.stages < 2 || smem > kUmmaSmemBudget ||
      (shape0.epi_bytes & 255) || (EG > 2 ? EG : 2) * shape0.ngroups * BN > 512)
    return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(umma_group_kernel<BN, Epi, EG>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int tiles = G.start[G.n];
  const int grid = tiles < num_sms ? tiles : num_sms;
  umma_group_kernel<BN, Epi, EG><<<grid, 64 + 128 * EG, smem, st>>>(G);
  return cudaGetLastError();
}

}  // namespace afq
