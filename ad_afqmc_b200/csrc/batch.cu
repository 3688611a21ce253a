// Batches of independent solves (fragments of different sizes) advanced by
// grouped launches: each kernel of the mixed-precision phaseless step runs
// once for the whole batch over a device table of per-solve arguments, the
// tensor-core GEMMs as persistent grouped kernels over (solve, tile) work
// lists (mixed_ops.cu).  Every solve gets exactly the arithmetic of its solo
// afq_propagate_constrained call (same kernels, tiles and summation orders),
// so its results are bit-identical to the solve run alone.
#include <cuda_runtime.h>

#include <algorithm>
#include <math.h>
#include <vector>

#include "afqmc_b200.h"
#include "layout.cuh"
#include "ops.h"

using namespace afq;

struct afq_batch {
  int n = 0, ns_max = 0, nprop = 0;
  UmmaBatch* umma = nullptr;
  GreenArgs* green = nullptr;
  GjArgs* gj = nullptr;
  PrepArgs* prep = nullptr;
  WalkerTArgs* wt[2] = {nullptr, nullptr};
  OvlpArgs* ovlp = nullptr;
  WeightArgs* weight = nullptr;
  BlockMap m_green{}, m_prep{}, m_wt[2]{}, m_ovlp{};
  size_t green_smem = 0, gj_smem = 0;
};

namespace {

size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

struct TableLayout {
  size_t green, gj, prep, wt0, wt1, ovlp, weight, umma, total;
};

TableLayout table_layout(int n, const Layout* L, int n_exp_terms) {
  TableLayout t{};
  size_t o = 0;
  t.green = o;
  o = al256(o + n * sizeof(GreenArgs));
  t.gj = o;
  o = al256(o + n * sizeof(GjArgs));
  t.prep = o;
  o = al256(o + n * sizeof(PrepArgs));
  t.wt0 = o;
  o = al256(o + n * sizeof(WalkerTArgs));
  t.wt1 = o;
  o = al256(o + n * sizeof(WalkerTArgs));
  t.ovlp = o;
  o = al256(o + n * sizeof(OvlpArgs));
  t.weight = o;
  o = al256(o + n * sizeof(WeightArgs));
  t.umma = o;
  o += umma_batch_table_bytes(n, L, n_exp_terms);
  t.total = al256(o);
  return t;
}

int layouts(int n, const afq_dims* dims, std::vector<Layout>& L) {
  if (n < 1 || n > kMaxBatch) return AFQ_ERR_SHAPE;
  if (!dims) return AFQ_ERR_NULL;
  L.resize(n);
  for (int f = 0; f < n; ++f) {
    const int rc = make_layout(&dims[f], L[f]);
    if (rc != AFQ_OK) return rc;
    if (!L[f].mixed) return AFQ_ERR_ARG;  // the FP64 path runs solve by solve
    if (dims[f].n_exp_terms != dims[0].n_exp_terms) return AFQ_ERR_ARG;
  }
  return AFQ_OK;
}

}  // namespace

extern "C" {

int afq_batch_table_size(int32_t n, const afq_dims* dims, size_t* bytes) {
  if (!bytes) return AFQ_ERR_NULL;
  std::vector<Layout> L;
  const int rc = layouts(n, dims, L);
  if (rc != AFQ_OK) return rc;
  *bytes = table_layout(n, L.data(), dims[0].n_exp_terms).total;
  return AFQ_OK;
}

int afq_batch_create(int32_t n, const afq_dims* dims, const void* const* prepared, void* const* work,
                     const size_t* work_bytes, const afq_state* states, const double* const* fields,
                     void* table, size_t table_bytes, afq_batch** out) {
  if (!prepared || !work || !work_bytes || !states || !fields || !table || !out) return AFQ_ERR_NULL;
  std::vector<Layout> L;
  int rc = layouts(n, dims, L);
  if (rc != AFQ_OK) return rc;
  const int nexp = dims[0].n_exp_terms;
  const TableLayout T = table_layout(n, L.data(), nexp);
  if (table_bytes < T.total) return AFQ_ERR_WORKSPACE;
  if ((reinterpret_cast<uintptr_t>(table) & 255u) != 0) return AFQ_ERR_ALIGN;
  for (int f = 0; f < n; ++f) {
    if (!prepared[f] || !work[f] || !fields[f] || !states[f].weights || !states[f].overlaps ||
        !states[f].scalars || !states[f].walkers[0] || (L[f].ns == 2 && !states[f].walkers[1]))
      return AFQ_ERR_NULL;
    if (work_bytes[f] < (size_t)L[f].work * sizeof(double)) return AFQ_ERR_WORKSPACE;
  }
  afq_batch* b = new afq_batch();
  b->n = n;
  std::vector<GreenArgs> green(n);
  std::vector<GjArgs> gj(n);
  std::vector<PrepArgs> prep(n);
  std::vector<WalkerTArgs> wt[2];
  std::vector<OvlpArgs> ovlp(n);
  std::vector<WeightArgs> weight(n);
  std::vector<const double*> P(n);
  std::vector<double*> Wk(n), w0(n), w1(n);
  int gb = 0, pb = 0, ob = 0, wb[2] = {0, 0}, nw[2] = {0, 0};
  b->m_green.n = b->m_prep.n = b->m_ovlp.n = n;
  for (int f = 0; f < n; ++f) {
    const Layout& l = L[f];
    P[f] = static_cast<const double*>(prepared[f]);
    Wk[f] = static_cast<double*>(work[f]);
    w0[f] = states[f].walkers[0];
    w1[f] = states[f].walkers[1];
    const double* const wc[2] = {w0[f], w1[f]};
    GreenArgs a = green_args(l, P[f], Wk[f], wc);
    piece_ptrs(Wk[f], l.v_gpl, l.v_gpl_ps, l.npc, a.gplb);
    green[f] = a;
    b->m_green.start[f] = gb;
    gb += l.W * l.ns;
    b->green_smem = std::max(b->green_smem, green_smem_bytes(l.nomax));
    b->gj_smem = std::max(b->gj_smem, gj_smem_bytes(l.nomax));
    gj[f] = GjArgs{l.W, l.no[0], l.ns > 1 ? l.no[1] : 0, l.nomax * (l.nomax | 1), Wk[f] + l.w_s,
                   (long long)l.nomax * l.nomax, Wk[f] + l.w_wscal};
    PrepArgs p{};
    p.W = l.W;
    p.G = l.G;
    p.splitk = l.splitk;
    p.npc = l.npc;
    p.Gpad = l.Gpad;
    p.ldxb = l.Gb;
    p.field_step = (long long)l.W * l.G;
    p.fbpart = Wk[f] + l.w_fbpart;
    p.f32 = 1;  // batches are mixed precision: FP32 partials
    p.alpha = (double)l.mult;
    p.sdt = sqrt(dims[f].dt);
    p.fields = fields[f];
    p.mf = P[f] + l.p_mf;
    p.xt = Wk[f] + l.w_xt;
    p.wscal = Wk[f] + l.w_wscal;
    piece_ptrs(Wk[f], l.v_xt, l.v_xt_ps, l.npc, p.xb);
    prep[f] = p;
    b->m_prep.start[f] = pb;
    pb += l.W;
    for (int s = 0; s < l.np; ++s) {
      WalkerTArgs t{};
      t.wk = s == 0 ? w0[f] : w1[f];
      t.N = l.N;
      t.nc = 2 * l.no[s];
      t.np = l.npc;
      t.gx = (l.N + 31) / 32;
      t.gy = (t.nc + 31) / 32;
      piece_ptrs(Wk[f], l.v_bt[0], l.v_bt_ps, l.npc, t.p);
      t.ld = l.Kv;
      t.bstride = 2LL * l.nomax * l.Kv;
      t.acc = reinterpret_cast<float*>(Wk[f] + l.v_acc);
      b->m_wt[s].start[nw[s]] = wb[s];
      wb[s] += t.gx * t.gy * l.W;
      wt[s].push_back(t);
      ++nw[s];
    }
    ovlp[f] = OvlpArgs{l.W, l.ns, l.mult, 16, Wk[f] + l.w_wscal, Wk[f] + l.w_wscal + 12};
    b->m_ovlp.start[f] = ob;
    ob += (l.W + 255) / 256;
    weight[f] = WeightArgs{l.W, dims[f].dt, P[f] + l.p_scal, Wk[f] + l.w_wscal, states[f].weights,
                           states[f].overlaps, states[f].scalars};
    b->ns_max = std::max(b->ns_max, l.np);
  }
  b->m_green.start[n] = gb;
  b->m_prep.start[n] = pb;
  b->m_ovlp.start[n] = ob;
  for (int s = 0; s < 2; ++s) {
    b->m_wt[s].n = nw[s];
    b->m_wt[s].start[nw[s]] = wb[s];
  }
  unsigned char* base = static_cast<unsigned char*>(table);
  b->green = reinterpret_cast<GreenArgs*>(base + T.green);
  b->gj = reinterpret_cast<GjArgs*>(base + T.gj);
  b->prep = reinterpret_cast<PrepArgs*>(base + T.prep);
  b->wt[0] = reinterpret_cast<WalkerTArgs*>(base + T.wt0);
  b->wt[1] = reinterpret_cast<WalkerTArgs*>(base + T.wt1);
  b->ovlp = reinterpret_cast<OvlpArgs*>(base + T.ovlp);
  b->weight = reinterpret_cast<WeightArgs*>(base + T.weight);
  bool ok = cudaMemcpy(b->green, green.data(), n * sizeof(GreenArgs), cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemcpy(b->gj, gj.data(), n * sizeof(GjArgs), cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemcpy(b->prep, prep.data(), n * sizeof(PrepArgs), cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemcpy(b->ovlp, ovlp.data(), n * sizeof(OvlpArgs), cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemcpy(b->weight, weight.data(), n * sizeof(WeightArgs), cudaMemcpyHostToDevice) == cudaSuccess;
  for (int s = 0; s < 2 && ok; ++s)
    if (nw[s] > 0)
      ok = cudaMemcpy(b->wt[s], wt[s].data(), nw[s] * sizeof(WalkerTArgs), cudaMemcpyHostToDevice) ==
           cudaSuccess;
  if (!ok) {
    delete b;
    return AFQ_ERR_CUDA;
  }
  rc = umma_batch_create(n, L.data(), P.data(), Wk.data(), w0.data(), w1.data(), nexp, base + T.umma,
                         table_bytes - T.umma, &b->umma);
  if (rc != AFQ_OK) {
    delete b;
    return rc;
  }
  b->nprop = umma_batch_nprop(b->umma);
  *out = b;
  return AFQ_OK;
}

int afq_batch_propagate_constrained(afq_batch* b, int32_t step, int32_t green_current, void* stream) {
  if (!b) return AFQ_ERR_NULL;
  if (step < 0) return AFQ_ERR_ARG;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
#define AFQ_B(expr)                             \
  do {                                          \
    if ((expr) != cudaSuccess) return AFQ_ERR_CUDA; \
  } while (0)
  // force bias of the current walkers (Green's function unless already current)
  if (!green_current) {
    AFQ_B(launch_green_grouped(b->green, b->m_green, 1, b->green_smem, st));
    AFQ_B(launch_gj_grouped(b->gj, b->m_green, b->gj_smem, st));
    AFQ_B(launch_green_grouped(b->green, b->m_green, 2, b->green_smem, st));
  }
  int rc = umma_batch_fb(b->umma, st);
  if (rc != AFQ_OK) return rc;
  AFQ_B(launch_prep_grouped(b->prep, b->m_prep, step, st));
  // VHS and the Trotterized propagator, spin sector by spin sector
  if ((rc = umma_batch_vhs(b->umma, st)) != AFQ_OK) return rc;
  for (int s = 0; s < b->ns_max; ++s) {
    AFQ_B(launch_walker_t_grouped(b->wt[s], b->m_wt[s], st));
    for (int i = 0; i < b->nprop; ++i)
      if ((rc = umma_batch_prop(b->umma, s, i, st)) != AFQ_OK) return rc;
  }
  // new overlaps, the next step's force-bias operand, weights
  AFQ_B(launch_green_grouped(b->green, b->m_green, 1, b->green_smem, st));
  AFQ_B(launch_gj_grouped(b->gj, b->m_green, b->gj_smem, st));
  AFQ_B(launch_green_grouped(b->green, b->m_green, 2, b->green_smem, st));
  AFQ_B(launch_ovlp_grouped(b->ovlp, b->m_ovlp, st));
  AFQ_B(launch_weight_grouped(b->weight, b->n, st));
#undef AFQ_B
  return AFQ_OK;
}

int afq_batch_destroy(afq_batch* b) {
  if (!b) return AFQ_ERR_NULL;
  umma_batch_destroy(b->umma);
  delete b;
  return AFQ_OK;
}

}  // extern "C"
