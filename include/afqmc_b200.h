/*
 * afqmc_b200.h -- C ABI of the B200 (sm_100a) phaseless-AFQMC walker path.
 *
 * One shared library, libafqmc_b200.so, exports the walker-path operations
 * of ad_afqmc as plain C functions on raw device pointers.  The reference is
 * pure Python/JAX and has no FFI of its own; each entry point below names the
 * reference function (file:line inside the ad_afqmc project) whose behaviour
 * it replaces, and the Python layer in ad_afqmc_b200/ binds them with ctypes
 * behind the reference's method names.
 *
 * Conventions
 *  - All array arguments are device pointers (CUDA global memory), 16-byte
 *    aligned, C-contiguous.  complex128 data are interleaved (re, im) doubles.
 *  - Walkers: restricted (W, N, No) complex128; unrestricted two arrays
 *    (W, N, Na) and (W, N, Nb).
 *  - exp_h1 and mf_shifts may be NULL in afq_prepare() when only
 *    measurements (force bias, energy) are needed.
 *  - Every function is asynchronous on the given stream (cudaStream_t passed
 *    as void*; NULL = legacy default stream) and returns an afq_status.
 *  - The library never allocates device memory.  Hamiltonian data are laid
 *    out once by afq_prepare() into a caller-owned "prepared" buffer, and
 *    every operation takes a caller-owned workspace; their sizes come from
 *    afq_prepared_size() and afq_workspace_size().
 *  - Calls on one workspace must not overlap on the device; distinct
 *    (prepared, workspace) pairs are independent.
 */
#ifndef AFQMC_B200_H
#define AFQMC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum afq_status {
  AFQ_OK = 0,
  AFQ_ERR_SHAPE = 1,      /* unsupported or inconsistent sizes            */
  AFQ_ERR_NULL = 2,       /* a required pointer is NULL                   */
  AFQ_ERR_CUDA = 3,       /* CUDA runtime error during launch             */
  AFQ_ERR_WORKSPACE = 4,  /* prepared/workspace buffer too small          */
  AFQ_ERR_ALIGN = 5,      /* a pointer is not 16-byte aligned             */
  AFQ_ERR_ARG = 6,        /* an enum/flag argument is out of range        */
  AFQ_ERR_LIMIT = 7,      /* size beyond a fixed (static) scratch capacity */
  AFQ_ERR_TIMEOUT = 8,    /* a bounded device-side wait ran out (afq_check_status) */
  AFQ_ERR_BOUNDS = 9      /* debug builds: a device-side bounds check failed */
} afq_status;

enum { AFQ_RESTRICTED = 0, AFQ_UNRESTRICTED = 1 };      /* walker_type  */
enum { AFQ_TRIAL_RHF = 0, AFQ_TRIAL_UHF = 1 };          /* trial_type   */
/* precision: AFQ_FP64 everywhere; AFQ_MIXED: force bias, VHS, propagator
 * and exchange contractions on tcgen05 tensor cores with operands split into
 * two bfloat16 pieces (three products, FP32 accumulation); AFQ_MIXED_HI: three
 * pieces, six products.  Green's functions, determinants, QR, weights and
 * energy accumulation stay FP64 in every mode. */
enum { AFQ_FP64 = 0, AFQ_MIXED = 1, AFQ_MIXED_HI = 2 };
enum { AFQ_SR_LOCAL = 0, AFQ_SR_GLOBAL = 1 };           /* sr z-formula */

/* Problem sizes and method switches (fixed for one prepared buffer). */
typedef struct afq_dims {
  int32_t norb;        /* N: orbitals                                        */
  int32_t nocc[2];     /* electrons per spin (restricted walkers use nocc[0]), */
                       /* 1..64 (AFQ_ERR_SHAPE above: the Green's-function   */
                       /* and exchange kernels keep No x No blocks in shared  */
                       /* memory; the reference has no such limit)            */
  int32_t nchol;       /* G: Cholesky vectors                                */
  int32_t nwalkers;    /* W                                                  */
  int32_t walker_type; /* AFQ_RESTRICTED / AFQ_UNRESTRICTED                  */
  int32_t trial_type;  /* AFQ_TRIAL_RHF / AFQ_TRIAL_UHF                      */
  int32_t n_exp_terms; /* Taylor terms incl. identity (reference default 6)  */
  int32_t precision;   /* AFQ_FP64 / AFQ_MIXED                               */
  int32_t reserved;    /* must be 0                                          */
  double dt;           /* imaginary time step                                */
} afq_dims;

/* Trial and Hamiltonian inputs of afq_prepare() (device pointers). */
typedef struct afq_ham {
  const double* mo[2];       /* trial orbitals (N, nocc[s]) float64; [1] unused for RHF   */
  const double* rot_h1[2];   /* (nocc[s], N) float64; RHF: [0] only                       */
  const double* rot_chol[2]; /* (G, nocc[s], N) float64; RHF: [0] only                    */
  const double* chol;        /* (G, N*N) float64                                          */
  const double* exp_h1[2];   /* (N, N) float64; restricted walkers: [0] only              */
  const double* mf_shifts;   /* (G,) complex128                                           */
  double h0;                 /* constant energy                                           */
  double h0_prop[2];         /* complex h0_prop (re, im)                                  */
} afq_ham;

/* Per-walker propagation state (device pointers, updated in place). */
typedef struct afq_state {
  double* walkers[2];  /* restricted: [0] (W,N,No); unrestricted: [0] up, [1] down  */
  double* weights;     /* (W,) float64                                               */
  double* overlaps;    /* (W,) complex128                                            */
  double* scalars;     /* device doubles: [0] e_estimate, [1] pop_control_ene_shift,
                          [2] n_killed_walkers (accumulated), [3..7] reserved       */
  int32_t flags;       /* host-side; AFQ_STATE_GREEN_CURRENT: the workspace already
                          holds the force-bias operand (Green's function) of these
                          walkers, left there by the previous afq_propagate_constrained
                          on the same workspace.  Set on return by that function;
                          the caller clears it whenever the walkers change otherwise. */
  int32_t reserved;
} afq_state;

enum { AFQ_STATE_GREEN_CURRENT = 1 };

/* Library version (major*10000 + minor*100 + patch). */
int afq_version(void);
/* Human-readable status text. */
const char* afq_status_string(int status);

/* Bytes of the prepared Hamiltonian buffer / of the workspace. */
int afq_prepared_size(const afq_dims* d, size_t* bytes);
int afq_workspace_size(const afq_dims* d, size_t* bytes);

/* Lay out trial + Hamiltonian intermediates for the kernels.
 * Replaces the consumer side of rhf._build_measurement_intermediates
 * (wavefunctions.py:1215-1232), uhf (:1472-1496) and
 * propagator_afqmc._build_propagation_intermediates (propagation.py:378-438):
 * those tensors are computed by the caller and copied here into padded,
 * concatenated device layouts. */
int afq_prepare(const afq_dims* d, const afq_ham* h, void* prepared, size_t prepared_bytes,
                void* stream);

/* Bytes of workspace needed by afq_calc_overlap / afq_calc_green /
 * afq_orthonormalize (16 doubles per walker; no Hamiltonian data needed). */
int afq_small_workspace_size(const afq_dims* d, size_t* bytes);

/* overlap <psi_T|walker>  (W,) complex128.  mo: trial orbitals (N, nocc[s])
 * float64 per spin ([1] ignored for an RHF trial).
 * Replaces wave_function.calc_overlap (wavefunctions.py:93-200) ->
 * rhf._calc_overlap_restricted (:1064-1066) / _unrestricted (:1068-1074),
 * uhf._calc_overlap_unrestricted (:1259-1268). */
int afq_calc_overlap(const afq_dims* d, const double* const mo[2], const double* const walkers[2],
                     double* overlaps, void* work, size_t work_bytes, void* stream);

/* Overlaps like afq_calc_overlap, for callers that cannot allocate device
 * memory: no workspace argument, and nothing is allocated.  No counterpart in
 * the reference.  Host frameworks that own the device memory pool (an XLA
 * custom call inside a JAX program, for one) or code recording into a CUDA
 * graph under a capture mode that forbids allocation cannot pass a workspace;
 * this entry point keeps its per-walker scratch in a fixed 1 MiB array inside
 * the library's device image (held on every GPU that loads the library until
 * the process exits).  Limit: nwalkers <= 8192, else AFQ_ERR_LIMIT.  The
 * first call on a device looks up the array's device address; make it before
 * any stream capture.  Calls share the array, so calls that overlap on the
 * GPU race; nothing in it needs to start at zero. */
int afq_calc_overlap_static(const afq_dims* d, const double* const mo[2],
                            const double* const walkers[2], double* overlaps, void* stream);

/* half-rotated Green's function per spin, (W, nocc[s], N) complex128 each.
 * Replaces rhf._calc_green (wavefunctions.py:1089-1100), uhf._calc_green (:1289-1312). */
int afq_calc_green(const afq_dims* d, const double* const mo[2], const double* const walkers[2],
                   double* const green[2], void* work, size_t work_bytes, void* stream);

/* force bias (W, G) complex128.
 * Replaces wave_function.calc_force_bias (wavefunctions.py:202-262) ->
 * rhf._calc_force_bias_restricted (:1102-1110) / _unrestricted (:1112-1126),
 * uhf._calc_force_bias_unrestricted (:1314-1329). */
int afq_calc_force_bias(const afq_dims* d, const void* prepared, const double* const walkers[2],
                        double* force_bias, void* work, size_t work_bytes, void* stream);

/* local energy (W,) complex128.
 * Replaces wave_function.calc_energy (wavefunctions.py:264-394) ->
 * rhf._calc_energy_restricted (:1128-1141) / _unrestricted (:1143-1174),
 * uhf._calc_energy_unrestricted (:1331-1363).  The exchange term is a fused
 * kernel: the (G, No, No) intermediate is never written. */
int afq_calc_energy(const afq_dims* d, const void* prepared, const double* const walkers[2],
                    double* energies, void* work, size_t work_bytes, void* stream);

/* One phaseless step: force bias, field shifts, VHS, Taylor propagator with
 * one-body half-steps, new overlaps, phaseless weight update and population
 * control shift.  fields: (W, G) float64 (device).
 * Replaces propagator_afqmc.propagate_constrained (propagation.py:274-336)
 * with _apply_trotprop* (:154-272). */
int afq_propagate_constrained(const afq_dims* d, const void* prepared, afq_state* s,
                              const double* fields, void* work, size_t work_bytes, void* stream);

/* Householder QR of every walker in place (LAPACK zgeqrf/zungqr convention);
 * norms (W,) complex128 (prod diag R; unrestricted: |.| per spin multiplied),
 * may be NULL.  work: afq_small_workspace_size() bytes.  Unrestricted walkers get column 0 times sign(prod diag R).
 * Replaces linalg_utils.qr_vmap_restricted / _unrestricted (linalg_utils.py:51-72)
 * via RHFWalkers/UHFWalkers.orthonormalize (walkers.py:155-157, 260-262). */
int afq_orthonormalize(const afq_dims* d, double* const walkers[2], double* norms, void* work,
                       size_t work_bytes, void* stream);

/* walkers <- e^{-dt h/2} Taylor(e^{VHS}) e^{-dt h/2} walkers with VHS = i sqrt(dt)
 * sum_g x[w,g] L_g from the raw fields (W, G) float64, in place: the
 * propagator of free projection, propagator._apply_trotprop
 * (propagation.py:178-229) as called by propagate_free (:338-376).  Needs the
 * propagation intermediates (exp_h1, mf_shifts) in afq_prepare. */
int afq_apply_trotprop(const afq_dims* d, const void* prepared, double* const walkers[2],
                       const double* fields, void* work, size_t work_bytes, void* stream);

/* Comb resampling: indices (W,) int32 and new weights from weights and zeta;
 * the walkers are gathered from walkers_in into walkers_out (distinct buffers).
 * mode AFQ_SR_LOCAL follows sr.py:24-48, AFQ_SR_GLOBAL the single-rank
 * rank-0 arithmetic of sr.py:52-153.  Serial FP64 cumsum: bit-exact indices
 * given identical weights and zeta. */
int afq_stochastic_reconfiguration(const afq_dims* d, const double* weights_in, double zeta,
                                   int mode, const double* const walkers_in[2],
                                   double* const walkers_out[2], double* weights_out,
                                   int32_t* indices, void* stream);

/* Orbital energy of an LNO fragment's localized orbital for restricted
 * walkers and an RHF trial: rhf_lno._calc_orbenergy (wavefunctions.py:
 * 6898-6923), with f_g = rot_chol[g][:, No:] G^T[No:, :] (virtual block),
 * m = prjlo^T prjlo, orbE = 2 sum_g tr(f_g) sum(f_g o m) - sum_g sum((f_g f_g) o m).
 * prjlo: (n_lo, No) device doubles, 1 <= n_lo <= 8.  orbe: (W,) complex128.
 * FP64 whatever the precision of dims; f is never written to memory. */
int afq_calc_orbenergy(const afq_dims* d, const void* prepared, const double* const walkers[2],
                       const double* prjlo, int32_t n_lo, double* orbe, void* work,
                       size_t work_bytes, void* stream);

/* Comb of the reconfiguration across ranks: weights_all holds the weights
 * of n_ranks ranks of n_per_rank walkers each, in rank order (an all-gather).
 * Writes, for every one of the n_ranks * n_per_rank slots, the global index of
 * the walker that fills it and its new weight, with the rank-0 arithmetic of
 * sr.py:52-153 (z = (i + zeta) / n_per_rank / n_ranks * total, serial FP64
 * cumsum, searchsorted left): bit-exact given identical weights and zeta, so
 * every rank can comb the same gathered weights and agree on the plan.  The
 * walkers then move with one all-to-all (ad_afqmc_b200/sr_ranks.py).
 * n_ranks * n_per_rank <= 16384.  Device pointers. */
int afq_comb_indices_ranks(const double* weights_all, int32_t n_per_rank, int32_t n_ranks,
                           double zeta, double* weights_out, int32_t* indices, void* stream);

/* As afq_stochastic_reconfiguration with zeta read from device memory, so
 * that the call can be recorded in a CUDA graph and replayed with fresh
 * uniforms (see afq_uniform_dev). */
int afq_stochastic_reconfiguration_dev(const afq_dims* d, const double* weights_in,
                                       const double* zeta_dev, int mode,
                                       const double* const walkers_in[2],
                                       double* const walkers_out[2], double* weights_out,
                                       int32_t* indices, void* stream);

/* Block end of sampler._block_scan (sampling.py:76-94): killed-walker count,
 * QR, overlaps, local energies with the sqrt(2/dt) clamp, block energy and
 * weight, and the population-control shift update.
 * block_out: device doubles [0] block energy, [1] block weight. */
int afq_block_end(const afq_dims* d, const void* prepared, afq_state* s, double* block_out,
                  void* work, size_t work_bytes, void* stream);

/* Standard-normal auxiliary fields (n, ) float64 from a counter-based
 * Philox4x32-10 generator with Box-Muller; (seed, offset) select the stream.
 * Replaces random.normal(subkey, (S, W, G)) in sampler._block_scan
 * (sampling.py:63-71); the bits differ from JAX threefry by design. */
int afq_normal_fields(double* out, int64_t n, uint64_t seed, uint64_t offset, void* stream);

/* Graph-replayable variants: the Philox counter lives in device memory
 * (*counter) and advances by the draws consumed, so a captured CUDA graph
 * draws fresh fields/uniforms on every replay.  afq_uniform_dev writes one
 * U(0,1) (for the reconfiguration comb) to *out. */
int afq_normal_fields_dev(double* out, int64_t n, uint64_t seed, uint64_t* counter, void* stream);
int afq_uniform_dev(double* out, uint64_t seed, uint64_t* counter, void* stream);

/* Split x (n,) float64 into npieces (1..3) bfloat16 arrays with
 * x ~= p0 + p1 (+ p2), each piece rounded to nearest from the remainder.
 * Operand preparation of the mixed-precision contractions; no counterpart in
 * the reference (which uses float32/complex64 there, launch_script.py:654-657). */
int afq_split_bf16(const double* x, int64_t n, int npieces, void* const pieces[3], void* stream);

/* C[b] (M x N, float32, row stride ldc) = sum over pairs (i,j) of
 * A_i[b] (M x K) * B_j[b]^T (N x K), all pieces bfloat16 K-contiguous with row
 * strides lda/ldb (multiples of 8 elements) and batch strides (0 = packed).
 * pairs: npairs (i,j) index pairs.  tcgen05 tensor cores, FP32 accumulation.
 * err_flag: device int set to 1 if an internal wait timed out.
 * The split-operand GEMM behind the mixed-precision force bias, VHS and
 * exchange contractions (the reference's vhs_mixed_precision switch,
 * propagation.py:196-203); exposed for direct use and testing. */
int afq_gemm_split_bf16(const void* const a_pieces[3], int npa, const void* const b_pieces[3],
                        int npb, int npairs, const int32_t* pairs, int M, int N, int K, int batch,
                        int64_t lda, int64_t a_bstride, int64_t ldb, int64_t b_bstride, float* C,
                        int64_t ldc, int64_t c_bstride, int32_t* err_flag, void* stream);

/* Tile and schedule choices of one problem shape (no counterpart in the
 * reference, where XLA picks its own kernels).  Zero fields keep the built-in
 * heuristic.  afq_set_tuning registers a record for every call whose afq_dims
 * equal *d (process-wide, thread-safe); t == NULL removes it.  The workspace
 * size can depend on the record (split-K partials, exchange partial sums), so
 * query afq_workspace_size after registering; calls with a smaller workspace
 * return AFQ_ERR_WORKSPACE.  Buffers that live across calls (Green's
 * function, per-walker scalars, the error flag) keep their offsets under any
 * record.  A value the shape cannot use returns AFQ_ERR_ARG and registers
 * nothing.  afq_get_tuning reports the values in effect (heuristic ones
 * filled in; max_stages and grid_cap stay 0 when unlimited, and exch_bn is 0
 * when the exchange runs on the FP64 kernel). */
typedef struct afq_tuning {
  int32_t fb_splitk;   /* force-bias GEMM split-K: 1..8                                   */
  int32_t fb_bn;       /* tensor-core force-bias column tile: 64 or 128                  */
  int32_t vhs_bn;      /* tensor-core VHS column tile: 64 or 128                          */
  int32_t exch_bn;     /* tensor-core exchange column tile: 32, 64, 80, 96 or 128         */
  int32_t f64_exch_bn; /* FP64 exchange tile: 80, 120 or 160 (BM 120, 120, 128)           */
  int32_t max_stages;  /* cap on tcgen05 pipeline stages: 2..8                             */
  int32_t grid_cap;    /* CTAs of the persistent tensor-core kernels: 1..number of SMs     */
  int32_t prop_epi_groups; /* epilogue warpgroups of the tensor-core propagator: 1 to 3    */
  int32_t prop_order;  /* propagator tile order: 0 alternate direction per launch (the     */
                       /* walkers last read stay in L2 for the next launch), 1 forward     */
  int32_t prop_chunk;  /* propagator K accumulation: 0 built-in (the whole K in one TMEM  */
                       /* chain), 1 the whole K in one chain, 2 chunks of four 64-wide K   */
                       /* blocks summed in FP32 round-to-nearest (less shared memory left  */
                       /* for the operand pipeline)                                         */
  int32_t qr_mode;     /* QR of the walkers: 0 built-in choice, 1 walker in shared memory   */
                       /* (when it fits), 2 in place in global memory                       */
  int32_t vhs_chunk;   /* VHS GEMM K accumulation: 0 built-in (the whole K in one TMEM      */
                       /* chain per accumulator group), 1 the same, 2 chunks of four        */
                       /* 64-wide K blocks summed in FP32 round-to-nearest (less shared     */
                       /* memory left for the operand pipeline)                             */
  int32_t prop_bn;     /* column tile of the tensor-core propagator: 0 built-in (the        */
                       /* narrowest of 16..128 that holds a walker's 2 No columns), or one  */
                       /* of 16, 32, 48, 64, 80, 96, 128 (several tiles per walker when     */
                       /* 2 No is wider)                                                    */
  int32_t reserved[3];
} afq_tuning;

int afq_set_tuning(const afq_dims* d, const afq_tuning* t);
int afq_get_tuning(const afq_dims* d, afq_tuning* out);

/* ---- Batches of independent solves (uneven fragments) ---------------------
 * No counterpart in the reference, which solves LNO fragments one process at
 * a time (lnoutils.py:175-177).  A batch advances up to 64 solves of
 * different sizes (each with its own afq_dims, prepared buffer, workspace and
 * afq_state, all precision AFQ_MIXED or AFQ_MIXED_HI with the same
 * n_exp_terms) one phaseless step at a time: every kernel of the step runs
 * ONCE for the whole batch over a device table of per-solve arguments, and
 * the force-bias, VHS and propagator contractions run as persistent grouped
 * tcgen05 kernels over (solve, tile) work lists, one launch per tile shape.
 * Each solve gets the arithmetic of its own afq_propagate_constrained call,
 * bit for bit.  The table is caller-owned device memory of
 * afq_batch_table_size() bytes (256-byte aligned), written once by
 * afq_batch_create (synchronously); the buffers it points to must stay put.
 * fields[f]: solve f's fields of step 0, (W_f, G_f) float64; step s reads
 * fields[f] + s * W_f * G_f.  green_current: the workspaces hold the Green's
 * functions of the current walkers (every step of a block but the first). */
typedef struct afq_batch afq_batch;
int afq_batch_table_size(int32_t n, const afq_dims* dims, size_t* bytes);
int afq_batch_create(int32_t n, const afq_dims* dims, const void* const* prepared, void* const* work,
                     const size_t* work_bytes, const afq_state* states, const double* const* fields,
                     void* table, size_t table_bytes, afq_batch** out);
int afq_batch_propagate_constrained(afq_batch* b, int32_t step, int32_t green_current, void* stream);
int afq_batch_destroy(afq_batch* b);

/* ---- Per-solve Hamiltonian intermediates (FP64, device pointers) ----------
 * These replace the set-up half of the walker path, run once per solve:
 * every contraction runs on the FP64 tensor cores of this library.  They
 * take their own scratch `work` of afq_intermediates_workspace_size() bytes
 * (16-byte aligned); nothing is allocated.  Layouts are the reference's:
 * h1 (2, N, N), chol (G, N*N), mo (N, nocc[s]), rdm1 (2, N, N), all row-major. */
int afq_intermediates_workspace_size(int32_t norb, int32_t nchol, size_t* bytes);

/* h1[s] <- (h1[s] + h1[s]^T) / 2 in place for both spins; rot_h1[s] (nocc[s], N)
 * = mo[s]^T h with h = (h1[0] + h1[1]) / 2 for an RHF trial (one sector) and
 * h = h1[s] for a UHF trial (two); rot_chol[s] (G, nocc[s], N) with
 * rot_chol[s][g] = mo[s]^T L_g.  Replaces rhf._build_measurement_intermediates
 * (wavefunctions.py:1215-1232) and uhf._build_measurement_intermediates
 * (:1472-1496). */
int afq_measurement_intermediates(int32_t norb, const int32_t nocc[2], int32_t nchol,
                                  int32_t trial_type, const double* const mo[2], double* h1,
                                  const double* chol, double* const rot_h1[2],
                                  double* const rot_chol[2], void* work, size_t work_bytes,
                                  void* stream);

/* rho = rdm1[0] + rdm1[1]; mf_shifts (G,) complex128 = i sum(L_g o rho);
 * h0_prop (one complex128) = -h0 - sum(mf_shifts^2) / 2; v0 = 1/2 sum_g L_g L_g;
 * v1 = sum_g Re(i mf_g) L_g; exp_h1 = expm(-dt/2 h1_mod) with h1_mod =
 * (h1[0] + h1[1]) / 2 - v0 - v1 for restricted walkers (exp_h1: (N, N)) or
 * h1[s] - v0 - v1 per spin for unrestricted walkers (exp_h1: (2, N, N)).
 * h1 is the symmetrized one (afq_measurement_intermediates).  Synchronizes
 * `stream` once per exponential (the scaling exponent is chosen on the host).
 * Replaces propagator_afqmc._build_propagation_intermediates
 * (propagation.py:378-438); mf_shifts_fp and h0_prop_fp are scalar multiples
 * of these and left to the caller. */
int afq_propagation_intermediates(int32_t norb, int32_t nchol, int32_t walker_type, const double* h1,
                                  const double* rdm1, const double* chol, double h0, double dt,
                                  double* mf_shifts, double* h0_prop, double* exp_h1, void* work,
                                  size_t work_bytes, void* stream);

/* out (n, n) = expm(scale * A) for a real (n, n) matrix A (out must not alias
 * A): scaling and squaring of a truncated Taylor series whose degree follows
 * from the remainder bound for ||scale A / 2^s||_1 <= 1/2.  Synchronizes
 * `stream` once.  Replaces jax.scipy.linalg.expm in propagation.py:422-438.
 * work: 3 n m + 8 doubles with m = n rounded up to even
 * (afq_intermediates_workspace_size(n, 1) bytes cover it). */
int afq_expm(int32_t n, const double* A, double scale, double* out, void* work, size_t work_bytes,
             void* stream);

/* Eigenpairs of a real symmetric (n, n) matrix A, eigenvalues in descending
 * order into evals (n,) and the eigenvectors as the columns of evecs (n, n),
 * in the same order (cyclic Jacobi, n <= 2048).  The natural orbitals of
 * wave_function.get_init_walkers (wavefunctions.py:427-466) are the first
 * nocc columns for rdm1[0] + rdm1[1] (restricted walkers) or rdm1[s]
 * (unrestricted).  Within a degenerate eigenspace the basis may differ from
 * LAPACK's (as it may between LAPACK builds).  work: 2 m + 8 doubles with m =
 * n^2 rounded up to even.  Up to n = 160 the matrix is rotated in shared memory. */
int afq_eigh_desc(int32_t n, const double* A, double* evals, double* evecs, void* work,
                  size_t work_bytes, void* stream);

/* The k natural orbitals of largest occupation of a symmetric density matrix
 * rdm (n, n) (e.g. rdm1[0] + rdm1[1]): orbs (n, k) row-major, occupations
 * occ (k,) descending (may be NULL).  This is what wave_function.get_init_walkers
 * (wavefunctions.py:427-466) takes from eigh.  Subspace iteration on k + 8
 * vectors (orthonormalized by CholeskyQR2) with a Rayleigh-Ritz step (Jacobi
 * on the projected matrix) until every Ritz residual is below 1e-13 of the
 * spectral radius (one iteration for a projector density); when that does not
 * happen within 40 iterations (occupations too close at the cut) the full
 * afq_eigh_desc.  Synchronizes `stream` once per iteration.  k <= 64.
 * work: afq_natural_orbitals_workspace_size() bytes. */
int afq_natural_orbitals_workspace_size(int32_t n, int32_t k, size_t* bytes);
int afq_natural_orbitals(int32_t n, int32_t k, const double* rdm, double* orbs, double* occ, void* work,
                         size_t work_bytes, void* stream);

/* Device-side failure status of a workspace (no counterpart in the reference,
 * whose XLA kernels have no waits of their own; its only guards are the
 * numerical masks of propagation.py:321-331 and the driver's check of the
 * initial overlaps, driver.py:76-79).  The tensor-core kernels bound every
 * mbarrier wait; a wait that runs out sets a flag in the workspace, unwinds
 * and returns, after the launching call already returned AFQ_OK, so that
 * call's walkers or energies are invalid.  afq_check_status synchronizes
 * `stream`, reads the flag, clears it and returns AFQ_ERR_TIMEOUT if it was
 * set (call it once per block: the flag stays set until read).
 * afq_status_flag returns the flag's device address (an int32, 0 = clear) for
 * code that copies it out inside a CUDA graph instead.  afq_test_wait_timeout
 * is a test hook: one thread waits on an mbarrier that nothing arrives at,
 * with the GEMMs' bounded poll loop limited to `polls` (1..4096), and sets the
 * flag when the wait runs out; no copy or MMA is in flight, so nothing faults. */
int afq_check_status(const afq_dims* d, void* work, size_t work_bytes, void* stream);
int afq_status_flag(const afq_dims* d, void* work, size_t work_bytes, int32_t** flag);
int afq_test_wait_timeout(const afq_dims* d, void* work, size_t work_bytes, uint32_t polls,
                          void* stream);

/* Instrumentation (no counterpart in the reference, which has no native
 * code): launches of one kernel family (kernel_id >= 0) or of all library
 * kernels (kernel_id < 0) since load; and CUDA-event timing of every launch
 * of one family between afq_profile_begin and afq_profile_end (events are
 * recorded on the stream of each launch).  Families: 0 green, 1 force-bias
 * GEMM, 2 field prep, 3 VHS GEMM, 4 propagator GEMMs, 5 exchange, 6 energy
 * combine, 7 weights, 8 QR, 9 reconfiguration, 10 gather, 11 block end,
 * 12 normal fields, 13 other. */
int afq_launch_count(int kernel_id, unsigned long long* count);
int afq_profile_begin(int kernel_id);
int afq_profile_end(double* total_ms, int* launches);

#ifdef __cplusplus
}
#endif

#endif /* AFQMC_B200_H */
