// Device-memory layout of the prepared Hamiltonian and of the workspace.
//
// All leading dimensions are padded to an even number of doubles so that
// every row starts on a 16-byte boundary (cp.async / vector loads).
#pragma once

#include <stddef.h>

#include "afqmc_b200.h"

namespace afq {

constexpr int kMaxOcc = 64;  // largest occupied block per spin accepted by the kernels

// registry of afq_tuning records (tuning.cu)
bool tuning_lookup(const afq_dims& d, afq_tuning& out);
void tuning_store(const afq_dims& d, const afq_tuning* t);

inline long long round_even(long long x) { return (x + 1) & ~1LL; }
inline long long align_up(long long x, long long a) { return (x + a - 1) / a * a; }

// Exchange-energy tile choice (see exchange kernel): gpt Cholesky vectors
// per BM-row tile and wpt walkers per BN-column tile.
struct ExchTile {
  int bm;   // 120 or 128
  int bn;   // 80, 120 or 160
  int gpt;  // Cholesky vectors per tile
  int wpt;  // walkers per tile
  int mt;   // number of row tiles = ceil(G / gpt)
};

// Shared memory of the tensor-core exchange epilogue: the f block as
// (re, im) float pairs with an odd row stride in pairs, per-row partials
// (double4) and per-Cholesky-vector sums (double2) for 128 rows.
__host__ __device__ inline int exch_fs2(int no) { return (no + 1) | 1; }
__host__ __device__ inline long long exch_fs_bytes(int no) {
  return (128LL * exch_fs2(no) * 8 + 31) & ~31LL;
}
__host__ __device__ inline long long exch_epi_extra(int no) {
  return exch_fs_bytes(no) + 128 * 32 + 128 * 16;
}

// Exchange tile of the tensor-core path: 128 rows hold gpt Cholesky
// vectors, BN columns hold wpt walkers.
struct UExchTile {
  int bn, gpt, wpt, mt;
};

// Column tile of the exchange (two accumulator groups, double buffered:
// BN <= 128) holding whole walkers with the least padding, with room for two
// pipeline stages plus the epilogue's staging of one walker's f block.
inline UExchTile choose_uexch_tile(int no, int G, int npc) {
  UExchTile t;
  const int bns[5] = {128, 96, 80, 64, 32};
  const long long budget = 227 * 1024 - 1024 - 256;
  const long long extra = exch_epi_extra(no);
  t.bn = 0;
  double best = -1.0;
  for (int i = 0; i < 5; ++i) {
    const int bn = bns[i];
    if (((2 * no + 15) & ~15) > bn) continue;
    const long long stage = (long long)npc * (128 * 128 + bn * 128);
    if (2 * stage + extra > budget) continue;
    const int wpt = bn / (2 * no);
    const double eff = double(wpt * 2 * no) / bn;
    if (eff > best + 1e-9) { best = eff; t.bn = bn; }
  }
  t.gpt = 128 / no;
  t.wpt = t.bn ? t.bn / (2 * no) : 0;
  t.mt = (G + t.gpt - 1) / t.gpt;
  return t;
}

// The exchange tile of one column width, or bn = 0 when it cannot hold a
// walker or does not fit shared memory (same rules as choose_uexch_tile).
inline UExchTile uexch_tile_for(int no, int G, int npc, int bn) {
  UExchTile t{0, 128 / no, 0, 0};
  const long long budget = 227 * 1024 - 1024 - 256;
  const long long extra = exch_epi_extra(no);
  const long long stage = (long long)npc * (128 * 128 + bn * 128);
  if (((2 * no + 15) & ~15) <= bn && 2 * stage + extra <= budget) {
    t.bn = bn;
    t.wpt = bn / (2 * no);
  }
  t.mt = (G + t.gpt - 1) / t.gpt;
  return t;
}

inline long long round8(long long x) { return (x + 7) & ~7LL; }

struct Layout {
  // sizes
  int N, G, W, no[2], ns, np, mult, restricted, uhf_trial, nomax;
  int mixed, npc;      // tensor-core path and bf16 pieces per operand (2 or 3)
  long long Kb, Gb, Nb, Kv;  // bf16 row strides (multiples of 8 elements)
  UExchTile uex[2];
  int exch_f64[2];     // exchange of this spin on the FP64 kernel (always when !mixed)
  afq_tuning tune;     // registered record for this shape (zeros: heuristics)
  int fb_bn, vhs_bn;   // tensor-core column tiles of the force bias and VHS
  // bf16 buffers, offsets in doubles (4 bf16 per double); [piece] stride given by *_ps
  long long q_rccat, q_cholT, q_exph1[2], q_rc[2];
  long long q_rccat_ps, q_cholT_ps, q_exph1_ps, q_rc_ps[2];
  long long v_gpl, v_xt, v_vhs, v_bt[2], v_acc, v_gt[2];
  long long v_gpl_ps, v_xt_ps, v_vhs_ps, v_bt_ps, v_gt_ps[2];
  long long Npad, N2pad, Gpad, Kfb, Kfb_used, koff[2];
  int splitk;
  ExchTile ex[2];
  // prepared buffer offsets (doubles)
  long long p_mo[2], p_rh1[2], p_rc[2], p_rccat, p_chol, p_exph1[2], p_mf, p_scal, prepared;
  // workspace offsets (doubles)
  long long w_gpl, w_theta[2], w_fbpart, w_xt, w_wscal, w_vhs, w_y, w_acc, w_ta, w_tb;
  long long w_c[2], w_exc[2], w_orb, w_s, w_cum, w_idx, w_misc, work;
};

inline ExchTile choose_exch_tile(int no, int G, int W) {
  // (BM, BN) of the FP64 exchange kernels: 120 x 80, 120 x 120, 128 x 160
  const int bms[3] = {120, 120, 128}, bns[3] = {80, 120, 160};
  ExchTile best{0, 0, 0, 0, 0};
  double best_eff = -1.0;
  for (int i = 0; i < 3; ++i) {
    const int bm = bms[i], bn = bns[i];
    if (2 * no > bn || no > bm) continue;
    const int gpt = bm / no, wpt = bn / (2 * no);
    const double eff = double(gpt * no) / bm * double(wpt * 2 * no) / double(bn);
    if (eff > best_eff + 1e-9) {
      best_eff = eff;
      best = ExchTile{bm, bn, gpt, wpt, (G + gpt - 1) / gpt};
    }
  }
  (void)W;
  return best;
}

inline ExchTile exch_tile_for(int no, int G, int bn) {
  const int bm = bn == 160 ? 128 : 120;
  if ((bn != 80 && bn != 120 && bn != 160) || 2 * no > bn || no > bm) return ExchTile{0, 0, 0, 0, 0};
  const int gpt = bm / no;
  return ExchTile{bm, bn, gpt, bn / (2 * no), (G + gpt - 1) / gpt};
}

// Returns AFQ_OK and fills L, or a shape error.
// `record` (optional) replaces the registered tuning record of this shape.
inline int make_layout(const afq_dims* d, Layout& L, const afq_tuning* record = nullptr) {
  if (!d) return AFQ_ERR_NULL;
  if (d->norb <= 0 || d->nchol <= 0 || d->nwalkers <= 0) return AFQ_ERR_SHAPE;
  if (d->walker_type != AFQ_RESTRICTED && d->walker_type != AFQ_UNRESTRICTED) return AFQ_ERR_ARG;
  if (d->trial_type != AFQ_TRIAL_RHF && d->trial_type != AFQ_TRIAL_UHF) return AFQ_ERR_ARG;
  if (d->precision != AFQ_FP64 && d->precision != AFQ_MIXED && d->precision != AFQ_MIXED_HI)
    return AFQ_ERR_ARG;
  if (d->n_exp_terms < 1 || d->n_exp_terms > 32) return AFQ_ERR_ARG;
  L.N = d->norb;
  L.G = d->nchol;
  L.W = d->nwalkers;
  L.restricted = d->walker_type == AFQ_RESTRICTED;
  L.uhf_trial = d->trial_type == AFQ_TRIAL_UHF;
  if (L.restricted && L.uhf_trial) return AFQ_ERR_SHAPE;  // uhf trial needs unrestricted walkers
  L.no[0] = d->nocc[0];
  L.no[1] = L.restricted ? d->nocc[0] : d->nocc[1];
  if (!L.uhf_trial && L.no[0] != L.no[1]) return AFQ_ERR_SHAPE;  // rhf requires Na == Nb
  L.ns = L.restricted ? 1 : 2;
  L.np = L.ns;
  L.mult = L.restricted ? 2 : 1;
  // the exchange tile holds one walker's 2*No columns in at most 120
  for (int s = 0; s < L.ns; ++s)
    if (L.no[s] <= 0 || L.no[s] > kMaxOcc || L.no[s] > L.N) return AFQ_ERR_SHAPE;
  if (L.W > (1 << 16)) return AFQ_ERR_SHAPE;
  L.nomax = L.no[0] > L.no[1] ? L.no[0] : L.no[1];
  L.Npad = round_even(L.N);
  L.N2pad = round_even((long long)L.N * L.N);
  L.Gpad = round_even(L.G);
  L.koff[0] = 0;
  L.koff[1] = (long long)L.no[0] * L.N;
  long long kfb = 0;
  for (int s = 0; s < L.ns; ++s) kfb += (long long)L.no[s] * L.N;
  L.Kfb_used = kfb;  // columns actually written; the padding is never read
  L.Kfb = round_even(kfb);
  // split-K for the force-bias GEMM so that the grid covers the SMs twice
  {
    const long long tiles = ((2LL * L.W + 127) / 128) * ((L.G + 127) / 128);
    int sk = 1;
    while (tiles * sk < 296 && sk < 8 && L.Kfb / (sk * 2) >= 256) sk *= 2;
    L.splitk = sk;
  }
  if (record)
    L.tune = *record;
  else if (!tuning_lookup(*d, L.tune))
    L.tune = afq_tuning{};
  const afq_tuning& T = L.tune;
  if (T.fb_splitk < 0 || T.fb_splitk > 8 || T.max_stages < 0 || T.max_stages == 1 ||
      T.max_stages > 8 || T.grid_cap < 0)
    return AFQ_ERR_ARG;
  if (T.fb_bn != 0 && T.fb_bn != 64 && T.fb_bn != 128) return AFQ_ERR_ARG;
  if (T.prop_epi_groups < 0 || T.prop_epi_groups > 3) return AFQ_ERR_ARG;
  if (T.prop_order < 0 || T.prop_order > 1) return AFQ_ERR_ARG;
  if (T.prop_chunk < 0 || T.prop_chunk > 2) return AFQ_ERR_ARG;
  if (T.qr_mode < 0 || T.qr_mode > 2) return AFQ_ERR_ARG;
  if (T.vhs_chunk < 0 || T.vhs_chunk > 2) return AFQ_ERR_ARG;
  if (T.prop_bn != 0 && T.prop_bn != 16 && T.prop_bn != 32 && T.prop_bn != 48 && T.prop_bn != 64 &&
      T.prop_bn != 80 && T.prop_bn != 96 && T.prop_bn != 128)
    return AFQ_ERR_ARG;
  if (T.vhs_bn != 0 && T.vhs_bn != 64 && T.vhs_bn != 128) return AFQ_ERR_ARG;
  if (T.fb_splitk > 0) L.splitk = T.fb_splitk;
  for (int s = 0; s < 2; ++s) {
    L.ex[s] = T.f64_exch_bn ? exch_tile_for(L.no[s], L.G, T.f64_exch_bn)
                            : choose_exch_tile(L.no[s], L.G, L.W);
    if (T.f64_exch_bn && L.ex[s].bn == 0 && s < L.ns) return AFQ_ERR_ARG;
  }
  L.mixed = d->precision != AFQ_FP64;
  L.npc = d->precision == AFQ_MIXED_HI ? 3 : 2;
  L.Kb = round8(L.Kfb_used);
  L.Gb = round8(L.G);
  L.Nb = round8(L.N);
  L.Kv = round8(2LL * L.N);
  L.fb_bn = T.fb_bn ? T.fb_bn : 128;
  L.vhs_bn = T.vhs_bn ? T.vhs_bn : (L.npc == 2 ? 128 : 64);
  for (int s = 0; s < 2; ++s) {
    L.uex[s] = choose_uexch_tile(L.no[s], L.G, L.npc);
    if (T.exch_bn && L.mixed && s < L.ns) {
      L.uex[s] = uexch_tile_for(L.no[s], L.G, L.npc, T.exch_bn);
      if (L.uex[s].bn == 0) return AFQ_ERR_ARG;
    }
  }
  for (int s = 0; s < 2; ++s) {
    if (L.ex[s].bn == 0 && s < L.ns) return AFQ_ERR_SHAPE;
    // three-piece operands of a large occupied block leave no room for two
    // pipeline stages of the tensor-core exchange: that spin's exchange runs
    // on the FP64 kernel (exact) instead
    L.exch_f64[s] = !L.mixed || L.uex[s].bn == 0;
    if (!L.exch_f64[s]) L.ex[s].mt = L.uex[s].mt;  // partial sums follow the tensor-core tiling
  }

  // ---- prepared buffer
  long long o = 0;
  auto take = [&](long long n) {
    long long r = o;
    o += align_up(n, 32);  // 256-byte aligned sub-buffers
    return r;
  };
  const int ntr = L.uhf_trial ? 2 : 1;
  for (int s = 0; s < 2; ++s) {
    L.p_mo[s] = L.p_rh1[s] = L.p_rc[s] = -1;
    L.p_exph1[s] = -1;
  }
  for (int s = 0; s < ntr; ++s) {
    L.p_mo[s] = take((long long)L.N * L.no[s]);
    L.p_rh1[s] = take((long long)L.no[s] * L.N);
    L.p_rc[s] = take((long long)L.G * L.no[s] * L.Npad);
  }
  if (!L.uhf_trial) {
    L.p_mo[1] = L.p_mo[0];
    L.p_rh1[1] = L.p_rh1[0];
    L.p_rc[1] = L.p_rc[0];
  }
  L.p_rccat = take((long long)L.G * L.Kfb);
  L.p_chol = take((long long)L.G * L.N2pad);
  for (int s = 0; s < L.np; ++s) L.p_exph1[s] = take((long long)L.N * L.Npad);
  L.p_mf = take(2LL * L.G);
  L.p_scal = take(8);
  // bf16 operand pieces of the tensor-core path (n bf16 = n/4 doubles)
  auto takeb = [&](long long nbf16, long long& ps) {
    ps = align_up((nbf16 + 3) / 4, 32);
    return take(ps * L.npc);
  };
  for (int s = 0; s < 2; ++s) L.q_exph1[s] = L.q_rc[s] = -1;
  if (L.mixed) {
    L.q_rccat = takeb((long long)L.G * L.Kb, L.q_rccat_ps);
    L.q_cholT = takeb((long long)L.N * L.N * L.Gb, L.q_cholT_ps);
    for (int s = 0; s < L.np; ++s) L.q_exph1[s] = takeb((long long)L.N * L.Nb, L.q_exph1_ps);
    for (int s = 0; s < ntr; ++s) L.q_rc[s] = takeb((long long)L.G * L.no[s] * L.Nb, L.q_rc_ps[s]);
    if (!L.uhf_trial) {
      L.q_rc[1] = L.q_rc[0];
      L.q_rc_ps[1] = L.q_rc_ps[0];
    }
  }
  L.prepared = o;

  // ---- workspace
  o = 0;
  const long long W = L.W, N = L.N;
  L.w_gpl = take(W * 2 * L.Kfb);
  for (int s = 0; s < 2; ++s) L.w_theta[s] = -1;
  for (int s = 0; s < L.ns; ++s) L.w_theta[s] = take(W * N * 2 * L.no[s]);
  L.w_xt = take(2 * W * L.Gpad);
  L.w_wscal = take(W * 16);
  L.w_vhs = take(W * N * 2 * L.Npad);
  const long long pb = W * N * 2 * L.nomax;  // (fp64 path) y / acc / t buffers
  L.w_y = take(pb);
  L.w_acc = take(pb);
  L.w_ta = take(pb);
  L.w_tb = take(pb);
  for (int s = 0; s < 2; ++s) L.w_c[s] = L.w_exc[s] = -1;
  for (int s = 0; s < L.ns; ++s) L.w_c[s] = take(W * L.G * 2);
  L.w_cum = take(W);
  L.w_idx = take(W);  // int32 indices stored in double slots
  L.w_misc = take(64);
  for (int s = 0; s < 2; ++s) L.v_gt[s] = -1;
  if (L.mixed) {
    L.v_gpl = takeb(2 * W * L.Kb, L.v_gpl_ps);
    L.v_xt = takeb(2 * W * L.Gb, L.v_xt_ps);
    L.v_vhs = takeb(W * N * L.Kv, L.v_vhs_ps);
    L.v_bt[0] = takeb(W * 2 * L.nomax * L.Kv, L.v_bt_ps);
    L.v_bt[1] = takeb(W * 2 * L.nomax * L.Kv, L.v_bt_ps);
    L.v_acc = take((W * N * 2 * L.nomax + 1) / 2);  // fp32
    for (int s = 0; s < L.ns; ++s) L.v_gt[s] = takeb(W * 2 * L.no[s] * L.Nb, L.v_gt_ps[s]);
  }
  // scratch whose size follows the tuning record last, so that every buffer
  // above keeps its offset when the record changes
  L.w_fbpart = take((long long)L.splitk * 2 * W * L.Gpad);
  for (int s = 0; s < L.ns; ++s) L.w_exc[s] = take((long long)L.ex[s].mt * W * 2);
  // LNO orbital-energy partials per FP64 exchange row tile (restricted walkers)
  L.w_orb = take((long long)((L.G + L.ex[0].gpt - 1) / L.ex[0].gpt) * W * 2);
  // S and S^-1 of the Green's function per (sector, walker), No_max^2 complex each
  L.w_s = take((long long)L.ns * W * L.nomax * L.nomax * 2);
  L.work = o;
  return AFQ_OK;
}

}  // namespace afq
