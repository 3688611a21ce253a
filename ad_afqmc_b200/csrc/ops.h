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

}  // namespace afq
