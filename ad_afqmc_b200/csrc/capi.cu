// extern "C" entry points of libafqmc_b200.so (declared in include/afqmc_b200.h).
#include <cuda_runtime.h>

#include "afqmc_b200.h"
#include "layout.cuh"
#include "ops.h"

using namespace afq;

namespace {

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }
inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

#define AFQ_TRY(expr)                          \
  do {                                         \
    cudaError_t _e = (expr);                   \
    if (_e != cudaSuccess) return AFQ_ERR_CUDA; \
  } while (0)

// Debug builds (-DAFQ_CHECKS, libafqmc_b200_checks.so): every pointer an
// entry point dereferences on the device must be device (or managed) memory;
// a host pointer is rejected with AFQ_ERR_ARG before anything is launched.
inline bool device_ptr_ok(const void* p) {
#ifdef AFQ_CHECKS
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
#else
  (void)p;
  return true;
#endif
}

int check_common(const afq_dims* d, Layout& L, const void* prepared, void* work,
                 size_t work_bytes) {
  int rc = make_layout(d, L);
  if (rc != AFQ_OK) return rc;
  if (!prepared || !work) return AFQ_ERR_NULL;
  if (!aligned16(prepared) || !aligned16(work)) return AFQ_ERR_ALIGN;
  if (work_bytes < (size_t)L.work * sizeof(double)) return AFQ_ERR_WORKSPACE;
  if (!device_ptr_ok(prepared) || !device_ptr_ok(work)) return AFQ_ERR_ARG;
  return AFQ_OK;
}

int check_walkers(const Layout& L, const double* const w[2]) {
  if (!w || !w[0]) return AFQ_ERR_NULL;
  if (!aligned16(w[0])) return AFQ_ERR_ALIGN;
  if (!device_ptr_ok(w[0])) return AFQ_ERR_ARG;
  if (L.ns == 2) {
    if (!w[1]) return AFQ_ERR_NULL;
    if (!aligned16(w[1])) return AFQ_ERR_ALIGN;
    if (!device_ptr_ok(w[1])) return AFQ_ERR_ARG;
  }
  return AFQ_OK;
}

int check_small(const afq_dims* d, Layout& L, void* work, size_t work_bytes) {
  int rc = make_layout(d, L);
  if (rc != AFQ_OK) return rc;
  if (!work) return AFQ_ERR_NULL;
  if (!aligned16(work)) return AFQ_ERR_ALIGN;
  if (work_bytes < (size_t)L.W * 16 * sizeof(double)) return AFQ_ERR_WORKSPACE;
  return AFQ_OK;
}

// Green's function of the current walkers and the force-bias contraction
// (split-K partial sums in the workspace, consumed by the field preparation).
int force_bias_impl(const Layout& L, const double* prep, double* work, GreenArgs& a,
                    cudaStream_t st) {
  if (L.mixed)
    piece_ptrs(work, L.v_gpl, L.v_gpl_ps, L.npc, a.gplb);
  else
    a.gpl = work + L.w_gpl;
  AFQ_TRY(launch_green(a, st));
  if (L.mixed) return mixed_fb_gemm(L, prep, work, st);
  AFQ_TRY(launch_fb_gemm(L, prep, work, st));
  return AFQ_OK;
}

// energy of the current walkers into wscal[.,14..15] and optionally eout
int energy_impl(const Layout& L, const double* prep, double* work, const double* const walkers[2],
                double* eout, int eout_stride, cudaStream_t st) {
  GreenArgs a = green_args(L, prep, work, walkers);
  for (int s = 0; s < L.ns; ++s) {
    a.sec[s].rh1 = prep + L.p_rh1[s];
    if (L.exch_f64[s])
      a.sec[s].theta = work + L.w_theta[s];
    else
      piece_ptrs(work, L.v_gt[s], L.v_gt_ps[s], L.npc, a.sec[s].gtb);
  }
  AFQ_TRY(launch_green(a, st));
  for (int s = 0; s < L.ns; ++s) {
    if (L.exch_f64[s]) {
      AFQ_TRY(launch_exchange(L, prep, work, s, st));
    } else {
      const int rc = mixed_exchange(L, prep, work, s, st);
      if (rc != AFQ_OK) return rc;
    }
  }
  AFQ_TRY(launch_energy_combine(L, prep, work, eout, eout_stride, st));
  return AFQ_OK;
}

}  // namespace

extern "C" {

int afq_version(void) { return 100; }

const char* afq_status_string(int status) {
  switch (status) {
    case AFQ_OK: return "ok";
    case AFQ_ERR_SHAPE: return "unsupported or inconsistent sizes";
    case AFQ_ERR_NULL: return "a required pointer is NULL";
    case AFQ_ERR_CUDA: return "CUDA runtime error";
    case AFQ_ERR_WORKSPACE: return "prepared/workspace buffer too small";
    case AFQ_ERR_ALIGN: return "pointer not 16-byte aligned";
    case AFQ_ERR_ARG: return "argument out of range";
    case AFQ_ERR_LIMIT: return "size exceeds the fixed static scratch capacity";
    case AFQ_ERR_TIMEOUT: return "a device-side wait timed out; results since the last check are invalid";
    case AFQ_ERR_BOUNDS: return "a device-side bounds check failed (debug build); results are invalid";
    default: return "unknown status";
  }
}

int afq_set_tuning(const afq_dims* d, const afq_tuning* t) {
  if (!d) return AFQ_ERR_NULL;
  if (t) {
    Layout L;
    const int rc = make_layout(d, L, t);
    if (rc != AFQ_OK) return rc;
  }
  tuning_store(*d, t);
  return AFQ_OK;
}

int afq_get_tuning(const afq_dims* d, afq_tuning* out) {
  if (!out) return AFQ_ERR_NULL;
  Layout L;
  const int rc = make_layout(d, L);
  if (rc != AFQ_OK) return rc;
  *out = L.tune;
  out->fb_splitk = L.splitk;
  out->fb_bn = L.fb_bn;
  out->vhs_bn = L.vhs_bn;
  out->exch_bn = L.mixed && !L.exch_f64[0] ? L.uex[0].bn : 0;
  out->f64_exch_bn = L.ex[0].bn;
  out->max_stages = L.tune.max_stages;  // 0: as many as fit, per GEMM
  out->grid_cap = L.tune.grid_cap;      // 0: one CTA per SM
  return AFQ_OK;
}

int afq_prepared_size(const afq_dims* d, size_t* bytes) {
  Layout L;
  int rc = make_layout(d, L);
  if (rc != AFQ_OK) return rc;
  if (!bytes) return AFQ_ERR_NULL;
  *bytes = (size_t)L.prepared * sizeof(double);
  return AFQ_OK;
}

int afq_workspace_size(const afq_dims* d, size_t* bytes) {
  Layout L;
  int rc = make_layout(d, L);
  if (rc != AFQ_OK) return rc;
  if (!bytes) return AFQ_ERR_NULL;
  *bytes = (size_t)L.work * sizeof(double);
  return AFQ_OK;
}

int afq_prepare(const afq_dims* d, const afq_ham* h, void* prepared, size_t prepared_bytes,
                void* stream) {
  Layout L;
  int rc = make_layout(d, L);
  if (rc != AFQ_OK) return rc;
  if (!h || !prepared) return AFQ_ERR_NULL;
  if (!aligned16(prepared)) return AFQ_ERR_ALIGN;
  if (prepared_bytes < (size_t)L.prepared * sizeof(double)) return AFQ_ERR_WORKSPACE;
  const int ntr = L.uhf_trial ? 2 : 1;
  for (int s = 0; s < ntr; ++s)
    if (!h->mo[s] || !h->rot_h1[s] || !h->rot_chol[s]) return AFQ_ERR_NULL;
  if (!h->chol) return AFQ_ERR_NULL;
  cudaStream_t st = as_stream(stream);
  double* P = static_cast<double*>(prepared);
  const size_t D = sizeof(double);
  AFQ_TRY(cudaMemsetAsync(P, 0, (size_t)L.prepared * D, st));
  const int N = L.N;
  for (int s = 0; s < ntr; ++s) {
    const int no = L.no[s];
    AFQ_TRY(cudaMemcpyAsync(P + L.p_mo[s], h->mo[s], (size_t)N * no * D, cudaMemcpyDeviceToDevice,
                            st));
    AFQ_TRY(cudaMemcpyAsync(P + L.p_rh1[s], h->rot_h1[s], (size_t)no * N * D,
                            cudaMemcpyDeviceToDevice, st));
    AFQ_TRY(cudaMemcpy2DAsync(P + L.p_rc[s], (size_t)L.Npad * D, h->rot_chol[s], (size_t)N * D,
                              (size_t)N * D, (size_t)L.G * no, cudaMemcpyDeviceToDevice, st));
  }
  for (int s = 0; s < L.ns; ++s) {
    const int ts = L.uhf_trial ? s : 0;
    const size_t row = (size_t)L.no[s] * N * D;
    AFQ_TRY(cudaMemcpy2DAsync(P + L.p_rccat + L.koff[s], (size_t)L.Kfb * D, h->rot_chol[ts], row,
                              row, (size_t)L.G, cudaMemcpyDeviceToDevice, st));
  }
  AFQ_TRY(cudaMemcpy2DAsync(P + L.p_chol, (size_t)L.N2pad * D, h->chol, (size_t)N * N * D,
                            (size_t)N * N * D, (size_t)L.G, cudaMemcpyDeviceToDevice, st));
  for (int s = 0; s < L.np; ++s)
    if (h->exp_h1[s])
      AFQ_TRY(cudaMemcpy2DAsync(P + L.p_exph1[s], (size_t)L.Npad * D, h->exp_h1[s], (size_t)N * D,
                              (size_t)N * D, (size_t)N, cudaMemcpyDeviceToDevice, st));
  if (h->mf_shifts)
    AFQ_TRY(cudaMemcpyAsync(P + L.p_mf, h->mf_shifts, (size_t)L.G * 2 * D, cudaMemcpyDeviceToDevice,
                          st));
  AFQ_TRY(launch_set_scalars(P + L.p_scal, h->h0, h->h0_prop[0], h->h0_prop[1], 0.0, st));
  if (L.mixed) return mixed_prepare(L, P, st);
  return AFQ_OK;
}

int afq_small_workspace_size(const afq_dims* d, size_t* bytes) {
  Layout L;
  int rc = make_layout(d, L);
  if (rc != AFQ_OK) return rc;
  if (!bytes) return AFQ_ERR_NULL;
  *bytes = (size_t)L.W * 16 * sizeof(double);
  return AFQ_OK;
}

int afq_calc_overlap(const afq_dims* d, const double* const mo[2], const double* const walkers[2],
                     double* overlaps, void* work, size_t work_bytes, void* stream) {
  Layout L;
  int rc = check_small(d, L, work, work_bytes);
  if (rc != AFQ_OK) return rc;
  if ((rc = check_walkers(L, walkers)) != AFQ_OK) return rc;
  if (!overlaps || !mo || !mo[0] || (L.uhf_trial && !mo[1])) return AFQ_ERR_NULL;
  double* Wk = static_cast<double*>(work);
  cudaStream_t st = as_stream(stream);
  GreenArgs a = green_args_mo(L, mo, Wk, walkers);
  a.wscal = Wk;
  AFQ_TRY(launch_green(a, st));
  AFQ_TRY(launch_ovlp_combine(L.W, L.ns, L.mult, Wk, overlaps, 2, st));
  return AFQ_OK;
}

int afq_calc_green(const afq_dims* d, const double* const mo[2], const double* const walkers[2],
                   double* const green[2], void* work, size_t work_bytes, void* stream) {
  Layout L;
  int rc = check_small(d, L, work, work_bytes);
  if (rc != AFQ_OK) return rc;
  if ((rc = check_walkers(L, walkers)) != AFQ_OK) return rc;
  if (!green || !green[0] || (L.ns == 2 && !green[1])) return AFQ_ERR_NULL;
  if (!mo || !mo[0] || (L.uhf_trial && !mo[1])) return AFQ_ERR_NULL;
  double* Wk = static_cast<double*>(work);
  GreenArgs a = green_args_mo(L, mo, Wk, walkers);
  a.wscal = Wk;
  for (int s = 0; s < L.ns; ++s) a.sec[s].gout = green[s];
  AFQ_TRY(launch_green(a, as_stream(stream)));
  return AFQ_OK;
}

int afq_calc_force_bias(const afq_dims* d, const void* prepared, const double* const walkers[2],
                        double* force_bias, void* work, size_t work_bytes, void* stream) {
  Layout L;
  int rc = check_common(d, L, prepared, work, work_bytes);
  if (rc != AFQ_OK) return rc;
  if ((rc = check_walkers(L, walkers)) != AFQ_OK) return rc;
  if (!force_bias) return AFQ_ERR_NULL;
  const double* P = static_cast<const double*>(prepared);
  double* Wk = static_cast<double*>(work);
  cudaStream_t st = as_stream(stream);
  GreenArgs a = green_args(L, P, Wk, walkers);
  rc = force_bias_impl(L, P, Wk, a, st);
  if (rc != AFQ_OK) return rc;
  AFQ_TRY(launch_prep(L, P, Wk, nullptr, d->dt, force_bias, st));
  return AFQ_OK;
}

int afq_calc_energy(const afq_dims* d, const void* prepared, const double* const walkers[2],
                    double* energies, void* work, size_t work_bytes, void* stream) {
  Layout L;
  int rc = check_common(d, L, prepared, work, work_bytes);
  if (rc != AFQ_OK) return rc;
  if ((rc = check_walkers(L, walkers)) != AFQ_OK) return rc;
  if (!energies) return AFQ_ERR_NULL;
  return energy_impl(L, static_cast<const double*>(prepared), static_cast<double*>(work), walkers,
                     energies, 2, as_stream(stream));
}

int afq_propagate_constrained(const afq_dims* d, const void* prepared, afq_state* s,
                              const double* fields, void* work, size_t work_bytes,
                              void* stream) {
  Layout L;
  int rc = check_common(d, L, prepared, work, work_bytes);
  if (rc != AFQ_OK) return rc;
  if (!s || !fields || !s->weights || !s->overlaps || !s->scalars) return AFQ_ERR_NULL;
  const double* const wc[2] = {s->walkers[0], s->walkers[1]};
  if ((rc = check_walkers(L, wc)) != AFQ_OK) return rc;
  if (!device_ptr_ok(fields) || !device_ptr_ok(s->weights) || !device_ptr_ok(s->overlaps) ||
      !device_ptr_ok(s->scalars))
    return AFQ_ERR_ARG;
  const double* P = static_cast<const double*>(prepared);
  double* Wk = static_cast<double*>(work);
  cudaStream_t st = as_stream(stream);
  // force bias of the current walkers (the Green's function is reused when the
  // previous step on this workspace already computed it for these walkers)
  GreenArgs a = green_args(L, P, Wk, wc);
  if (s->flags & AFQ_STATE_GREEN_CURRENT) {
    if (L.mixed) {
      if ((rc = mixed_fb_gemm(L, P, Wk, st)) != AFQ_OK) return rc;
    } else {
      AFQ_TRY(launch_fb_gemm(L, P, Wk, st));
    }
  } else {
    rc = force_bias_impl(L, P, Wk, a, st);
    if (rc != AFQ_OK) return rc;
  }
  s->flags &= ~AFQ_STATE_GREEN_CURRENT;
  AFQ_TRY(launch_prep(L, P, Wk, fields, d->dt, nullptr, st));
  // VHS and the Trotterized propagator
  if (L.mixed) {
    if ((rc = mixed_vhs_gemm(L, P, Wk, st)) != AFQ_OK) return rc;
    if ((rc = mixed_propagate_walkers(L, P, Wk, s->walkers, d->n_exp_terms, st)) != AFQ_OK)
      return rc;
  } else {
    AFQ_TRY(launch_vhs_gemm(L, P, Wk, st));
    AFQ_TRY(launch_propagate_walkers(L, P, Wk, s->walkers, d->n_exp_terms, st));
  }
  // new overlaps (and the next step's force-bias operand) and the weight update
  GreenArgs b = green_args(L, P, Wk, wc);
  if (L.mixed)
    piece_ptrs(Wk, L.v_gpl, L.v_gpl_ps, L.npc, b.gplb);
  else
    b.gpl = Wk + L.w_gpl;
  AFQ_TRY(launch_green(b, st));
  s->flags |= AFQ_STATE_GREEN_CURRENT;
  AFQ_TRY(launch_ovlp_combine(L.W, L.ns, L.mult, Wk + L.w_wscal, Wk + L.w_wscal + 12, 16, st));
  AFQ_TRY(launch_weight_update(L, P, Wk, s->weights, s->overlaps, s->scalars, d->dt, st));
  return AFQ_OK;
}

int afq_apply_trotprop(const afq_dims* d, const void* prepared, double* const walkers[2],
                       const double* fields, void* work, size_t work_bytes, void* stream) {
  Layout L;
  int rc = check_common(d, L, prepared, work, work_bytes);
  if (rc != AFQ_OK) return rc;
  if (!walkers || !fields) return AFQ_ERR_NULL;
  const double* const wc[2] = {walkers[0], walkers[1]};
  if ((rc = check_walkers(L, wc)) != AFQ_OK) return rc;
  const double* P = static_cast<const double*>(prepared);
  double* Wk = static_cast<double*>(work);
  cudaStream_t st = as_stream(stream);
  AFQ_TRY(launch_free_fields(L, Wk, fields, d->dt, st));
  if (L.mixed) {
    if ((rc = mixed_vhs_gemm(L, P, Wk, st)) != AFQ_OK) return rc;
    return mixed_propagate_walkers(L, P, Wk, walkers, d->n_exp_terms, st);
  }
  AFQ_TRY(launch_vhs_gemm(L, P, Wk, st));
  AFQ_TRY(launch_propagate_walkers(L, P, Wk, walkers, d->n_exp_terms, st));
  return AFQ_OK;
}

int afq_orthonormalize(const afq_dims* d, double* const walkers[2], double* norms, void* work,
                       size_t work_bytes, void* stream) {
  Layout L;
  int rc = make_layout(d, L);
  if (rc != AFQ_OK) return rc;
  if (!work) return AFQ_ERR_NULL;
  if (!aligned16(work)) return AFQ_ERR_ALIGN;
  if (work_bytes < (size_t)L.W * 16 * sizeof(double)) return AFQ_ERR_WORKSPACE;
  const double* const wc[2] = {walkers ? walkers[0] : nullptr, walkers ? walkers[1] : nullptr};
  if ((rc = check_walkers(L, wc)) != AFQ_OK) return rc;
  AFQ_TRY(launch_qr(L, walkers, norms, static_cast<double*>(work), as_stream(stream)));
  return AFQ_OK;
}

static int sr_impl(const afq_dims* d, const double* weights_in, double zeta, const double* zeta_dev,
                   int mode, const double* const walkers_in[2], double* const walkers_out[2],
                   double* weights_out, int32_t* indices, void* stream) {
  Layout L;
  int rc = make_layout(d, L);
  if (rc != AFQ_OK) return rc;
  if (mode != AFQ_SR_LOCAL && mode != AFQ_SR_GLOBAL) return AFQ_ERR_ARG;
  if (!weights_in || !weights_out || !indices) return AFQ_ERR_NULL;
  if (L.W > kMaxSrWalkers) return AFQ_ERR_SHAPE;
  if (weights_out == weights_in) return AFQ_ERR_ARG;
  cudaStream_t st = as_stream(stream);
  AFQ_TRY(launch_sr(L.W, 1, weights_in, zeta, zeta_dev, mode, weights_out, indices, st));
  if (walkers_in && walkers_out) {
    for (int s = 0; s < L.ns; ++s) {
      if (!walkers_in[s] || !walkers_out[s]) return AFQ_ERR_NULL;
      if (walkers_in[s] == walkers_out[s]) return AFQ_ERR_ARG;
      AFQ_TRY(launch_gather(L.W, (long long)L.N * 2 * L.no[s], walkers_in[s], walkers_out[s],
                            indices, st));
    }
  }
  return AFQ_OK;
}

int afq_stochastic_reconfiguration(const afq_dims* d, const double* weights_in, double zeta,
                                   int mode, const double* const walkers_in[2],
                                   double* const walkers_out[2], double* weights_out,
                                   int32_t* indices, void* stream) {
  return sr_impl(d, weights_in, zeta, nullptr, mode, walkers_in, walkers_out, weights_out, indices,
                 stream);
}

int afq_stochastic_reconfiguration_dev(const afq_dims* d, const double* weights_in,
                                       const double* zeta_dev, int mode,
                                       const double* const walkers_in[2],
                                       double* const walkers_out[2], double* weights_out,
                                       int32_t* indices, void* stream) {
  if (!zeta_dev) return AFQ_ERR_NULL;
  return sr_impl(d, weights_in, 0.0, zeta_dev, mode, walkers_in, walkers_out, weights_out,
                 indices, stream);
}

int afq_calc_orbenergy(const afq_dims* d, const void* prepared, const double* const walkers[2],
                       const double* prjlo, int32_t n_lo, double* orbe, void* work,
                       size_t work_bytes, void* stream) {
  Layout L;
  int rc = check_common(d, L, prepared, work, work_bytes);
  if (rc != AFQ_OK) return rc;
  if (!walkers || !walkers[0] || !prjlo || !orbe) return AFQ_ERR_NULL;
  if (!L.restricted || L.uhf_trial) return AFQ_ERR_ARG;  // rhf_lno with restricted walkers
  if (n_lo < 1 || n_lo > 8) return AFQ_ERR_ARG;
  const double* prep = static_cast<const double*>(prepared);
  double* wk = static_cast<double*>(work);
  cudaStream_t st = as_stream(stream);
  GreenArgs a = green_args(L, prep, wk, walkers);
  a.sec[0].theta = wk + L.w_theta[0];
  AFQ_TRY(launch_green(a, st));
  AFQ_TRY(launch_orbenergy(L, prep, wk, prjlo, n_lo, orbe, st));
  return AFQ_OK;
}

int afq_comb_indices_ranks(const double* weights_all, int32_t n_per_rank, int32_t n_ranks,
                           double zeta, double* weights_out, int32_t* indices, void* stream) {
  if (!weights_all || !weights_out || !indices) return AFQ_ERR_NULL;
  if (n_per_rank <= 0 || n_ranks <= 0) return AFQ_ERR_SHAPE;
  const long long W = (long long)n_per_rank * n_ranks;
  if (W > kMaxSrWalkers) return AFQ_ERR_SHAPE;
  if (weights_out == weights_all) return AFQ_ERR_ARG;
  AFQ_TRY(launch_sr((int)W, n_ranks, weights_all, zeta, nullptr, AFQ_SR_GLOBAL, weights_out,
                    indices, as_stream(stream)));
  return AFQ_OK;
}

int afq_block_end(const afq_dims* d, const void* prepared, afq_state* s, double* block_out,
                  void* work, size_t work_bytes, void* stream) {
  Layout L;
  int rc = check_common(d, L, prepared, work, work_bytes);
  if (rc != AFQ_OK) return rc;
  if (!s || !s->weights || !s->overlaps || !s->scalars || !block_out) return AFQ_ERR_NULL;
  const double* const wc[2] = {s->walkers[0], s->walkers[1]};
  if ((rc = check_walkers(L, wc)) != AFQ_OK) return rc;
  const double* P = static_cast<const double*>(prepared);
  double* Wk = static_cast<double*>(work);
  cudaStream_t st = as_stream(stream);
  AFQ_TRY(launch_qr(L, s->walkers, nullptr, Wk, st));
  rc = energy_impl(L, P, Wk, wc, Wk + L.w_wscal + 14, 16, st);
  if (rc != AFQ_OK) return rc;
  AFQ_TRY(launch_ovlp_combine(L.W, L.ns, L.mult, Wk + L.w_wscal, s->overlaps, 2, st));
  AFQ_TRY(launch_block_end(L, Wk, s->weights, s->scalars, d->dt, block_out, st));
  return AFQ_OK;
}

int afq_normal_fields_dev(double* out, int64_t n, uint64_t seed, uint64_t* counter,
                          void* stream) {
  if (!out || !counter) return AFQ_ERR_NULL;
  if (n <= 0) return AFQ_ERR_ARG;
  AFQ_TRY(launch_normal_dev(out, n, seed, reinterpret_cast<unsigned long long*>(counter),
                            as_stream(stream)));
  return AFQ_OK;
}

int afq_uniform_dev(double* out, uint64_t seed, uint64_t* counter, void* stream) {
  if (!out || !counter) return AFQ_ERR_NULL;
  AFQ_TRY(launch_uniform_dev(out, seed, reinterpret_cast<unsigned long long*>(counter),
                             as_stream(stream)));
  return AFQ_OK;
}

int afq_normal_fields(double* out, int64_t n, uint64_t seed, uint64_t offset, void* stream) {
  if (!out) return AFQ_ERR_NULL;
  if (n < 0) return AFQ_ERR_ARG;
  if (n == 0) return AFQ_OK;
  AFQ_TRY(launch_normal(out, n, seed, offset, as_stream(stream)));
  return AFQ_OK;
}

}  // extern "C"
