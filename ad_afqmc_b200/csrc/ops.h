// Internal launch wrappers shared by the C-ABI translation unit.
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"
#include "layout.cuh"

namespace afq {

// ---- Green's function / overlap (green.cu) --------------------------------
struct GreenSector {
  const double* walk;   // (W, N, no) complex
  const double* mo;     // (N, no)
  const double* rh1;    // (no, N) or nullptr
  int no;
  long long koff;       // offset of this sector inside a G-planar row
  double* theta;        // (W, N, no) complex or nullptr
  double* gout;         // (W, no, N) complex or nullptr
  bf16* gtb[3];         // exchange operand pieces: rows (w, j, re/im), row stride ldtb, or nullptr
  long long ldtb;
};
struct GreenArgs {
  int N, W, ns;
  GreenSector sec[2];
  double* wscal;        // per-walker scalars (16 doubles) or nullptr
  double* gpl;          // (2W, ldg) planar G or nullptr
  long long ldg;
  int npc;              // bf16 pieces for the *b outputs
  bf16* gplb[3];        // force-bias operand pieces (2W, ldgb) or nullptr
  long long ldgb;
  double* sbuf;         // (ns, W, sstride) complex scratch for S and S^-1, or nullptr (one kernel)
  long long sstride;    // complex elements per (sector, walker): No_max^2
};
cudaError_t launch_green(const GreenArgs& a, cudaStream_t st);
// overlaps from per-sector determinants in wscal: out[w] = det0^mult (or det0*det1)
cudaError_t launch_ovlp_combine(int W, int ns, int mult, const double* wscal, double* out,
                                int out_stride, cudaStream_t st);

// ---- dense contractions (gemm_ops.cu) --------------------------------------
cudaError_t launch_fb_gemm(const Layout& L, const double* prepared, double* work,
                           cudaStream_t st);
cudaError_t launch_prep(const Layout& L, const double* prepared, double* work,
                        const double* fields, double dt, double* fb_out, cudaStream_t st);
cudaError_t launch_free_fields(const Layout& L, double* work, const double* fields, double dt,
                               cudaStream_t st);
cudaError_t launch_vhs_gemm(const Layout& L, const double* prepared, double* work,
                            cudaStream_t st);
cudaError_t launch_propagate_walkers(const Layout& L, const double* prepared, double* work,
                                     double* const walkers[2], int n_exp_terms,
                                     cudaStream_t st);
cudaError_t launch_exchange(const Layout& L, const double* prepared, double* work, int sector,
                            cudaStream_t st);
// LNO orbital energy of restricted walkers from Theta in the workspace
// (overwrites its occupied rows); prj: n_lo x No device doubles, n_lo <= 8
cudaError_t launch_orbenergy(const Layout& L, const double* prepared, double* work,
                             const double* prj, int nlo, double* out, cudaStream_t st);
cudaError_t launch_energy_combine(const Layout& L, const double* prepared, double* work,
                                  double* eout, int eout_stride, cudaStream_t st);

// ---- walker ops (walker_ops.cu) --------------------------------------------
cudaError_t launch_weight_update(const Layout& L, const double* prepared, double* work,
                                 double* weights, double* overlaps, double* scalars, double dt,
                                 cudaStream_t st);
cudaError_t launch_qr(const Layout& L, double* const walkers[2], double* norms, double* work,
                      cudaStream_t st);
// W <= kMaxSrWalkers (cumulative sum kept in shared memory)
constexpr int kMaxSrWalkers = 16384;
cudaError_t launch_sr(int W, int ranks, const double* weights_in, double zeta,
                      const double* zeta_dev, int mode, double* weights_out, int* indices,
                      cudaStream_t st);
cudaError_t launch_gather(int W, long long walker_doubles, const double* in, double* out,
                          const int* indices, cudaStream_t st);
cudaError_t launch_block_end(const Layout& L, double* work, const double* weights,
                             double* scalars, double dt, double* block_out, cudaStream_t st);
cudaError_t launch_normal(double* out, long long n, unsigned long long seed,
                          unsigned long long offset, cudaStream_t st);
cudaError_t launch_normal_dev(double* out, long long n, unsigned long long seed,
                              unsigned long long* counter, cudaStream_t st);
cudaError_t launch_uniform_dev(double* out, unsigned long long seed, unsigned long long* counter,
                               cudaStream_t st);
cudaError_t launch_set_scalars(double* dst, double a, double b, double c, double d,
                               cudaStream_t st);

// ---- tensor-core (mixed precision) path (mixed_ops.cu) ---------------------
int mixed_prepare(const Layout& L, double* prepared, cudaStream_t st);
int mixed_fb_gemm(const Layout& L, const double* prepared, double* work, cudaStream_t st);
int mixed_vhs_gemm(const Layout& L, const double* prepared, double* work, cudaStream_t st);
int mixed_propagate_walkers(const Layout& L, const double* prepared, double* work,
                            double* const walkers[2], int n_exp_terms, cudaStream_t st);
int mixed_exchange(const Layout& L, const double* prepared, double* work, int sector,
                   cudaStream_t st);
// bf16 piece pointers of a buffer at offset `off` (doubles) with piece stride `ps`
inline void piece_ptrs(double* base, long long off, long long ps, int npc, bf16* out[3]) {
  for (int i = 0; i < 3; ++i)
    out[i] = i < npc ? reinterpret_cast<bf16*>(base + off + i * ps) : nullptr;
}

// Green's-function arguments of a walker set with trial orbitals `mo`
// (overlaps, Green's function; no workspace-resident S buffer)
inline GreenArgs green_args_mo(const Layout& L, const double* const mo[2], double* work,
                               const double* const walkers[2]) {
  GreenArgs a{};
  a.N = L.N;
  a.W = L.W;
  a.ns = L.ns;
  a.wscal = work + L.w_wscal;
  a.gpl = nullptr;
  a.ldg = L.Kfb;
  for (int s = 0; s < L.ns; ++s) {
    a.sec[s].walk = walkers[s];
    a.sec[s].mo = mo[L.uhf_trial ? s : 0];
    a.sec[s].rh1 = nullptr;
    a.sec[s].no = L.no[s];
    a.sec[s].koff = L.koff[s];
    a.sec[s].theta = nullptr;
    a.sec[s].gout = nullptr;
    for (int i = 0; i < 3; ++i) a.sec[s].gtb[i] = nullptr;
    a.sec[s].ldtb = L.Nb;
  }
  a.npc = L.npc;
  for (int i = 0; i < 3; ++i) a.gplb[i] = nullptr;
  a.ldgb = L.Kb;
  a.sbuf = nullptr;
  a.sstride = (long long)L.nomax * L.nomax;
  return a;
}

// ... of the engine's walkers with the prepared trial and the full workspace
// (S goes through the separate Gauss-Jordan kernel)
inline GreenArgs green_args(const Layout& L, const double* prep, double* work,
                            const double* const walkers[2]) {
  const double* mo[2] = {prep + L.p_mo[0], prep + L.p_mo[1]};
  GreenArgs a = green_args_mo(L, mo, work, walkers);
  a.sbuf = work + L.w_s;
  return a;
}

// ---- batches of independent solves (batch.cu) --------------------------------
// A grouped launch runs the blocks of up to kMaxBatch solves: solve f owns the
// global blocks [start[f], start[f+1]); every kernel finds its solve by a
// binary search and reads that solve's arguments from device memory.
constexpr int kMaxBatch = 64;
struct BlockMap {
  int n;
  int start[kMaxBatch + 1];
};
__device__ __forceinline__ int block_owner(const BlockMap& m, int b, int& local) {
  int lo = 0, hi = m.n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (m.start[mid] <= b) lo = mid;
    else hi = mid - 1;
  }
  local = b - m.start[lo];
  return lo;
}

struct GjArgs {
  int W, no0, no1, bstride;
  double* sbuf;
  long long sstride;
  double* wscal;
};
struct PrepArgs {
  int W, G, splitk, npc;
  long long Gpad, ldxb, field_step;  // doubles between the fields of consecutive steps
  const void* fbpart;                // FP32 partials (tensor-core force bias)
  int f32;
  double alpha, sdt;
  const double* fields;              // fields of step 0
  const double* mf;
  double* xt;
  double* wscal;
  bf16* xb[3];
};
struct OvlpArgs {
  int W, ns, mult, out_stride;
  const double* wscal;
  double* out;
};
struct WeightArgs {
  int W;
  double dt;
  const double* scal;
  const double* wscal;
  double* weights;
  double* overlaps;
  double* scalars;
};
struct WalkerTArgs {
  const double* wk;
  int N, nc, np, gx, gy;  // gx, gy: 32-wide tiles along N and nc
  bf16* p[3];
  long long ld, bstride;
  float* acc;
};
size_t green_smem_bytes(int nomax);
size_t gj_smem_bytes(int nomax);
cudaError_t launch_green_grouped(const GreenArgs* args, const BlockMap& m, int mode, size_t smem,
                                 cudaStream_t st);
cudaError_t launch_gj_grouped(const GjArgs* args, const BlockMap& m, size_t smem, cudaStream_t st);
cudaError_t launch_ovlp_grouped(const OvlpArgs* args, const BlockMap& m, cudaStream_t st);
cudaError_t launch_prep_grouped(const PrepArgs* args, const BlockMap& m, int step, cudaStream_t st);
cudaError_t launch_weight_grouped(const WeightArgs* args, int n, cudaStream_t st);
cudaError_t launch_walker_t_grouped(const WalkerTArgs* args, const BlockMap& m, cudaStream_t st);

// The tensor-core GEMMs of one mixed-precision step for a batch of solves
// (mixed_ops.cu).  Built from the same per-solve parameters as the solo
// calls (recorded instead of launched), then grouped by tile shape: one
// persistent launch per group.  The per-solve parameter blocks live in the
// caller's device table.
struct UmmaBatch;
size_t umma_batch_table_bytes(int n, const Layout* L, int n_exp_terms);
int umma_batch_create(int n, const Layout* L, const double* const* prep, double* const* work,
                      double* const* walkers0, double* const* walkers1, int n_exp_terms,
                      void* table, size_t table_bytes, UmmaBatch** out);
int umma_batch_fb(const UmmaBatch* b, cudaStream_t st);
int umma_batch_vhs(const UmmaBatch* b, cudaStream_t st);
// propagator GEMM number `index` (0 .. n_exp_terms) of spin sector `sector`
int umma_batch_prop(const UmmaBatch* b, int sector, int index, cudaStream_t st);
int umma_batch_nprop(const UmmaBatch* b);
void umma_batch_destroy(UmmaBatch* b);

}  // namespace afq
