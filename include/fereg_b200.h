/* fereg_b200 — C ABI of the B200 fixed-effects solver.
 *
 * The entry points replace the reference's `Absorber` trait
 * (leoliu0/fereg, crates/fereg-core/src/absorber.rs:62-97) as implemented by `FeSolver`
 * (crates/fereg-core/src/solve.rs:351-1344), constructed where the reference calls
 * `solve::build` (solve.rs:338, selected by `build_absorber`, session.rs:606). A Rust shim
 * `impl Absorber for GpuAbsorber` binds them from fereg-core.
 *
 * Conventions
 *   - Plain pointers and sizes. Row blocks are N x R row-major doubles in the absorber's row
 *     order (fereg_absorber_row_order); FE coefficients are (m + g1) x R row-major,
 *     [x (m x R); alpha1 (g1 x R)] (solve.rs:7-9).
 *   - Return codes are the reference's `RfError::rc` (error.rs:24-34): 0 ok, 1 interrupted,
 *     198 invalid input, 430 convergence, 909 out of memory, 2001 too few observations,
 *     9999 internal. The message of the last failure on the calling thread is
 *     fereg_last_error(). No exception or panic crosses this boundary.
 *   - One handle is used by one host thread at a time (the reference's `Ctx` is !Sync,
 *     api.rs:198-210). Work runs on the handle's own CUDA stream.
 */
#ifndef FEREG_B200_H
#define FEREG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fereg_absorber fereg_absorber;

/* Mirror of the reference's `Ctx` hooks (api.rs:198-229): `interrupt` is polled between kernels
 * and iterations (nonzero = stop with rc 1); `log` receives phase messages when verbose >= 2. */
typedef struct fereg_ctx {
    int (*interrupt)(void* data);
    void* interrupt_data;
    void (*log)(void* data, const char* msg);
    void* log_data;
    int verbose;
} fereg_ctx;

/* absorber.rs:27-37 SolveInfo. */
typedef struct fereg_solve_info {
    uint64_t iterations; /* PCG iterations (1 for closed forms, as reghdfe e(ic)) */
    int32_t escalated;   /* the preconditioner was strengthened during this solve */
    int32_t exact;       /* solved by a direct factor or in closed form */
} fereg_solve_info;

/* Inner precision of fereg_absorber_residualize_ex. */
enum { FEREG_PREC_F64 = 0, FEREG_PREC_F32_REFINED = 1 };

/* Message of the last failed call on this thread. */
const char* fereg_last_error(void);

/* solve::build / FeSolver::new (solve.rs:338, 396): builds the cell structure of the
 * intercept-only terms and the weight state. codes[q] holds the n kept-order codes of term q,
 * each < g[q]; w (kept order, strictly positive) or NULL. ctx may be NULL. */
int fereg_absorber_create(const uint32_t* const* codes, const uint32_t* g, int nterms, const double* w, size_t n,
                          const fereg_ctx* ctx, fereg_absorber** out);

/* solve.rs:338 build with the terms' shapes (session.rs:20-42 Term): term q has codes[q] below
 * g[q], an intercept when intercept[q] != 0 (intercept NULL: every term), and nslopes[q] slope
 * variables (nslopes NULL: none), kept order, n values each, given in `slopes` term after term.
 * A term with slopes or without an intercept makes the absorber the heterogeneous-slope solver
 * (slopes.rs:2183 SlopeSolver): coefficient blocks then hold m + G_E * b_E rows (the reduced
 * coordinates, then E's level coefficients, slopes.rs:27-29) and term_values writes
 * sum_q g_q * (intercept_q + nslopes_q) values. The kernel-level hooks fereg_absorber_apply,
 * _rhs, _rhs_noalloc, _precond and _weight_state serve the intercept-only solver only (198). */
int fereg_absorber_create_terms(const uint32_t* const* codes, const uint32_t* g, const int* intercept,
                                const int* nslopes, const double* const* slopes, int nterms, const double* w, size_t n,
                                const fereg_ctx* ctx, fereg_absorber** out);
/* 1 when the absorber is the heterogeneous-slope solver. No counterpart in the reference. */
int fereg_absorber_has_slopes(const fereg_absorber* h);
/* Values fereg_absorber_term_values writes. */
size_t fereg_absorber_term_values_len(const fereg_absorber* h);
/* Test hooks of the slope solver (no counterpart in the reference): the weight state
 * (slopes.rs:527-697: M_s^+ per level of E, G_E x b_E^2; the block-Jacobi inverses, b^2 per level
 * of every block in block order; the redundant coordinates, m), one application of S and of the
 * preconditioner to host m x r blocks, the right-hand side of a host n x r block with
 * [sum w v^2; sum w v; sum w e^2] (3 x r), and the structure: n, m, E, G_E, b_E, slots per row,
 * blocks, small blocks, small coordinates (9 values) with the session term of every block. */
int fereg_slope_weight_state(const fereg_absorber* h, double* minv, double* jinv, uint8_t* redundant);
int fereg_slope_apply(fereg_absorber* h, const double* p, size_t r, double* y);
int fereg_slope_precond(fereg_absorber* h, const double* rr, size_t r, double* z);
int fereg_slope_rhs(fereg_absorber* h, const double* rows, size_t r, double* y, double* stats);
int fereg_slope_structure(const fereg_absorber* h, uint64_t* out9, uint32_t* block_terms);

void fereg_absorber_destroy(fereg_absorber* h);

/* Absorber::n (absorber.rs:64). */
size_t fereg_absorber_n(const fereg_absorber* h);

/* p = m + g1, the rows of an FeCoefs block (absorber.rs:41-46). */
size_t fereg_absorber_coefs_len(const fereg_absorber* h);

/* Absorber::row_order (absorber.rs:67): kept-observation index of each row (n values). */
int fereg_absorber_row_order(const fereg_absorber* h, uint32_t* out);

/* Absorber::weights (absorber.rs:70): row-order weights into out (n values) and *has = 1, or
 * *has = 0 when every weight is 1. */
int fereg_absorber_weights(const fereg_absorber* h, double* out, int* has);

/* Absorber::set_weights (absorber.rs:75, solve.rs:1010-1139): row-order weights, strictly
 * positive and finite (else 198), or NULL for ones. */
int fereg_absorber_set_weights(fereg_absorber* h, const double* w);

/* Absorber::set_weights with the n row-order weights in device memory of the current device:
 * the weight state (cell weights, n1, n_r, diag(S), redundant coordinates, Jacobi factors) is
 * computed on the device, as IRLS needs every iteration (glm/irls.rs:367-560). 198 when a weight
 * is not positive and finite. */
int fereg_absorber_set_weights_device(fereg_absorber* h, const double* w_dev);

/* Absorber::residualize (absorber.rs:78-86, solve.rs:1141-1311): residualizes the n x r
 * row-major host block z in place. tol: relative W-norm accuracy of each column; maxiter: PCG
 * cap (430 when reached); warm: (m+g1) x r start or NULL; coefs_out: (m+g1) x r or NULL
 * (filled when want_coefs). */
int fereg_absorber_residualize(fereg_absorber* h, double* z, size_t r, double tol, size_t maxiter, int want_coefs,
                               const double* warm, double* coefs_out, fereg_solve_info* info);

/* As fereg_absorber_residualize with a choice of inner precision (FEREG_PREC_*) and z either
 * host memory (z_on_device = 0) or device memory on the current device (z_on_device = 1). */
int fereg_absorber_residualize_ex(fereg_absorber* h, double* z, int z_on_device, size_t r, double tol, size_t maxiter,
                                  int want_coefs, const double* warm, double* coefs_out, int precision,
                                  fereg_solve_info* info);

/* Absorber::fit_rows (absorber.rs:88): FE fit of coefficient column col per row (row order). */
int fereg_absorber_fit_rows(const fereg_absorber* h, const double* coefs, size_t r, size_t col, double* out);

/* Absorber::term_values (absorber.rs:90-96, solve.rs:1319-1343): level values of column col per
 * session term, concatenated in term order (sum_q g[q] values); every term but the one with
 * the most levels has weighted mean 0. */
int fereg_absorber_term_values(const fereg_absorber* h, const double* coefs, size_t r, size_t col, double* out);

/* The handle's CUDA stream (cudaStream_t), for callers that order their own device work or
 * record CUDA events against the solver's kernels. */
void* fereg_absorber_stream(const fereg_absorber* h);

/* Phase timing with CUDA events on the handle's stream (the reference's PhaseTimer, timing.rs;
 * reported under verbose >= 2 as in solve.rs:387-392). Enabling resets the totals. Slots
 * (FEREG_PHASE_SLOTS): 0 rhs segment pass, 1 rhs coordinate-list pass, 2 operator S*P segment
 * pass, 3 preconditioner, 4 PCG vector work, 5 residualize pass, 6 host-to-device rows,
 * 7 device-to-host rows, 8 operator S*P coordinate-list pass, 9 escalations and preconditioner
 * refreshes (host wall time of the factor / hierarchy builds). */
#define FEREG_PHASE_SLOTS 10
int fereg_absorber_set_profiling(fereg_absorber* h, int on);
int fereg_absorber_phase_times(const fereg_absorber* h, double* ms, uint64_t* counts);

/* Kernel launches issued by this handle so far. */
uint64_t fereg_absorber_launches(const fereg_absorber* h);
/* Escalations so far (cg.rs:24-37 probe: a large block whose Jacobi PCG contracts slower than
 * 0.6 per iteration at iteration 12 gets a multigrid V-cycle, and PCG restarts), and the large
 * blocks currently preconditioned that way. */
int fereg_absorber_escalations(const fereg_absorber* h, uint64_t* escalations, uint64_t* blocks);

/* Kernel-level entry points used by the parity tests (device work, host buffers). */
/* n, m, g1, ncells, nb, m_small, fe1, small_work, blocks in the small super-block (9 values) */
int fereg_absorber_info(const fereg_absorber* h, uint64_t* out9);
int fereg_absorber_apply(fereg_absorber* h, const double* p, size_t r, double* y);
int fereg_absorber_rhs(fereg_absorber* h, const double* rows, size_t r, double* y, double* b1, double* wsq, double* wsum);
int fereg_absorber_precond(fereg_absorber* h, const double* rr, size_t r, double* z);
int fereg_absorber_weight_state(const fereg_absorber* h, double* n1, double* nr, double* diag, uint8_t* redundant,
                                double* sw);

/* ---------------------------------------------------------------------------------------------
 * Estimation session: the part of the reference's `Session` (session.rs) that `Session::ols`
 * (ols.rs:199-470) uses, over the B200 absorber. Codes are the prepared kept-order codes
 * (after factorize / drop_singletons / restrict, session.rs:243-280). */
typedef struct fereg_session fereg_session;

/* ols.rs Spec: vce 0 unadjusted, 1 robust (HC1), 2 cluster (CRV1 over all the session's cluster
 * dimensions, multiway by inclusion-exclusion), 3 CRV3 (the leave-one-cluster-out jackknife,
 * crv3.rs, over the same subsets; intercept-only terms, no fweights), 4 HC2, 5 HC3 (Stata regress
 * with the exact leverage of the FE columns, leverage.rs:128 and ols.rs:450-474; the reduced
 * system must fit the dense small factor, at most 1024 coordinates); firstpair: dof from the first FE pair only
 * (dof.rs DofOptions); want_groupvar: mobility groups of the first pair into out->groupvar. */
typedef struct fereg_ols_spec {
    int vce;
    int noconstant;
    int firstpair;
    int want_groupvar;
    double tol;
    size_t maxiter;
    int precision; /* FEREG_PREC_* of the FE solve */
} fereg_ols_spec;

/* EstResult of ols.rs:263-470. Buffers (NULL to skip): b (nx + 1, the constant last),
 * V ((nx + 1)^2), status (nx: 0 ok, 2 absorbed by the FE, 3 collinear), resid / d / groupvar
 * (n, kept order; d = sum of the fixed effects), dof_table (5 per FE term: levels, redundant,
 * levels - redundant, inexact, nested; 64 terms at most). */
typedef struct fereg_ols_out {
    double* b;
    double* V;
    uint8_t* status;
    double* resid;
    double* d;
    double* groupvar;
    double* dof_table;
    int32_t nslots, k_all, y_absorbed;
    double N, rank, df_r, df_m, df_a, df_a_initial, df_a_redundant, df_a_nested;
    double N_clust, N_clustervars, N_clust1, N_clust2, num_singletons, N_full, report_constant;
    double rss, tss, tss_within, mss, rmse, r2, r2_a, r2_within, r2_a_within, ll, ll_0, F, sumweights, ic;
} fereg_ols_out;

/* Session over nterms kept-order FE terms (codes[q] < g[q]; nterms = 0: noabsorb), ncl cluster
 * dimensions (kept-order codes), weights w (kept order, NULL for none) of weight_kind 1 aweight,
 * 2 fweight, 3 pweight, n kept rows; num_singletons as dropped by the preparation. */
int fereg_session_create(const uint32_t* const* codes, const uint32_t* g, int nterms, const uint32_t* const* cl_codes,
                         const uint32_t* cl_g, int ncl, const double* w, int weight_kind, size_t n,
                         uint64_t num_singletons, const fereg_ctx* ctx, fereg_session** out);
/* fereg_session_create with the terms' shapes as fereg_absorber_create_terms: slope terms make
 * the session's absorber the slope solver, and the dof slots (dof.rs:74-88) one per intercept
 * and one per slope, with the slopes' redundant levels (dof.rs:165-176). */
int fereg_session_create_terms(const uint32_t* const* codes, const uint32_t* g, const int* intercept,
                               const int* nslopes, const double* const* slopes, int nterms,
                               const uint32_t* const* cl_codes, const uint32_t* cl_g, int ncl, const double* w,
                               int weight_kind, size_t n, uint64_t num_singletons, const fereg_ctx* ctx,
                               fereg_session** out);
void fereg_session_destroy(fereg_session* s);

/* Session::row_order: the rows of an ols block (n values, kept-observation indices). */
int fereg_session_row_order(const fereg_session* s, uint32_t* out);

/* Session::ols (ols.rs:199): OLS of column 0 on columns 1..nx of the n x (1 + nx) row-major
 * block `rows` in row order, host memory or (rows_on_device = 1) device memory of the current
 * device. A device block is residualized in place; a host block is copied to the device and left
 * unchanged. */
int fereg_session_ols(fereg_session* s, double* rows, int rows_on_device, size_t nx, const fereg_ols_spec* spec,
                      fereg_ols_out* out);

/* Wild cluster bootstrap (ols.rs:204 ols_with_wildboot, wildboot/ols.rs:243-650 run_cluster_11):
 * WCR11 test of H0: b[coef] = r0 with Rademacher weights on the clusters of the session's first
 * cluster dimension (full enumeration when G <= 20 and 2^G <= reps), restricted residuals, CRV1
 * over every cluster dimension, two-tailed p-value. Draw b uses SplitMix64 stream (seed, b)
 * (rng.rs, weights.rs:65-79). Each `tile` draws are residualized together as columns of one block
 * PCG. t_boot (reps values, or 2^G under full enumeration) may be NULL. */
typedef struct fereg_boot_spec {
    size_t coef;
    double r0;
    size_t reps;
    uint64_t seed;
    size_t tile;
    double tol;
    size_t maxiter;
    int precision; /* FEREG_PREC_* of the bootstrap solves */
} fereg_boot_spec;

typedef struct fereg_boot_out {
    double stat, se, point, pvalue;
    uint64_t reps;
    int32_t full_enum;
    double* t_boot;
} fereg_boot_out;

int fereg_session_wildboot(fereg_session* s, double* rows, int rows_on_device, size_t nx, const fereg_ols_spec* spec,
                           const fereg_boot_spec* boot, fereg_boot_out* out);

/* IV / 2SLS on the session's fixed effects with ivreghdfe conventions (replaces Session::iv,
 * iv.rs:299, for b and V): rows is the n x (1 + nx + nendog + ninst) row-order block
 * [y, exog, endog, inst] (Layout {nx, nendog, ninst}, api.rs), residualized in one absorber
 * call; ivreg2 with `small` and sdofminus = max(df_a, 1). vce 0 unadjusted (pweights imply
 * robust), 1 robust, 2 cluster over the session's cluster dimensions. b and V are in e(b) order
 * [endog..., exog...] (nendog + nx); status has nx + nendog + ninst entries in block order.
 * 481 when fewer excluded instruments than endogenous regressors survive collinearity. */
typedef struct fereg_iv_spec {
    int vce;
    double tol;
    size_t maxiter;
    int precision;
} fereg_iv_spec;

typedef struct fereg_iv_out {
    double* b;
    double* V;
    uint8_t* status;
    double N, df_r, df_m, df_a, sdofminus, rss, rmse, F, N_clust, ic;
    int32_t endog_ct, inexog_ct, exexog_ct;
} fereg_iv_out;

int fereg_session_iv(fereg_session* s, double* rows, int rows_on_device, size_t nx, size_t nendog, size_t ninst,
                     const fereg_iv_spec* spec, fereg_iv_out* out);

/* GLM by IRLS on the session's fixed effects (glm/irls.rs:367-560, glm/mod.rs; replaces the
 * engine's glm_fit, engine.rs:1038, for unweighted samples): Poisson PML (ppmlhdfe conventions,
 * y >= 0) or logit (y in {0, 1}, step halving when the deviance rises) with y in column 0 of the
 * n x (1 + nx) row-order block and the regressors after it; every iteration refreshes the
 * weight state on the device and residualizes [z, X] warm-started from the previous FE
 * coefficients. vce 0 oim (the inverse Hessian; logit only), 1 robust (N / (N - 1)), 2 cluster
 * over the session's cluster dimensions (G / (G - 1), multiway eigenvalue clip). The sample is
 * taken as prepared (singletons and separated observations already dropped); unweighted
 * sessions only. 430 when IRLS does not converge within maxiter. */
#define FEREG_FAMILY_POISSON 1 /* api.rs Family::Poisson */
#define FEREG_FAMILY_LOGIT 2   /* api.rs Family::Logit */
typedef struct fereg_glm_spec {
    int vce;
    double tol;
    size_t maxiter;
    size_t inner_maxiter;
    int precision; /* FEREG_PREC_* of the FE solves */
    int family;    /* FEREG_FAMILY_*; fereg_session_poisson ignores it */
    double itol;   /* final inner tolerance (GlmOptions::itol; 0 = the default 1e-10) */
} fereg_glm_spec;

typedef struct fereg_glm_out {
    double* b;        /* nx; absorbed or collinear regressors 0 */
    double* V;        /* nx x nx */
    uint8_t* status;  /* nx: 0 ok, 2 absorbed by the FE, 3 collinear */
    double N, deviance, ll, chi2, df_m, N_clust;
    uint64_t iterations, pcg_iterations;
    int32_t converged;
} fereg_glm_out;

/* One ReLU separation check (glm/separation.rs:61-196, ppmlhdfe 2.3.3 relu_fix_separation) on
 * the session's sample: column 0 of the n x (1 + nx) block (row order) is the Poisson outcome,
 * columns 1..nx the regressors (standardized by their standard deviations inside). separated
 * (n bytes) and certificate (n values) are row order and may be NULL; out4 receives [separated
 * rows, ReLU iterations, PCG iterations, 1 when the check certified its result]. The rows it finds
 * are dropped by the caller, who prepares the remaining sample again and repeats until a check
 * finds none (glm/mod.rs:454-505 glm_separate). Unweighted sessions. */
int fereg_session_relu(fereg_session* s, double* rows, int rows_on_device, size_t nx, double itol,
                       size_t inner_maxiter, uint8_t* separated, double* certificate, uint64_t* out4);
int fereg_session_glm(fereg_session* s, double* rows, int rows_on_device, size_t nx, const fereg_glm_spec* spec,
                      fereg_glm_out* out);
/* fereg_session_glm with the Poisson family. */
int fereg_session_poisson(fereg_session* s, double* rows, int rows_on_device, size_t nx, const fereg_glm_spec* spec,
                          fereg_glm_out* out);

/* Test hook, host only (no device): the multigrid hierarchy that an escalation would build for
 * the first block above 768 levels of the given unweighted structure. sizes / nnz receive up to
 * max_levels entries; row_sum receives each level's largest |row sum| relative to its largest
 * diagonal (0 for a Laplacian, as every level must be). Returns the level count in *levels
 * (0 when no block qualifies). */
int fereg_amg_probe(const uint32_t* const* codes, const uint32_t* g, int nterms, size_t n, int max_levels,
                    uint32_t* levels, uint32_t* sizes, uint64_t* nnz, double* row_sum);

/* Test hook, host only (no device): the cell structure (structure.rs:247-527) and coordinate lists
 * that a session would build for the given terms, as counts (out[0..5]: cells, segments, reduced
 * coordinates, small coordinates, blocks, FE1 index) and a 64-bit FNV-1a digest of the row order,
 * segment offsets, first rows, cell coordinates and coordinate lists (out[6]). The host build is
 * parallel; the digest shows it does not depend on the thread count. */
int fereg_structure_digest(const uint32_t* const* codes, const uint32_t* g, int nterms, size_t n, uint64_t* out);
/* Test hook (device): builds the cell structure and coordinate lists of the codes both on the host
 * and on the device and counts the differences: out9 = [scalars and block flags, row order,
 * seg_off, cell_row, coord, list offsets, list cells, list segments, list other-block
 * coordinates]; all 0 when the device build is the host build element for element. */
int fereg_structure_compare(const uint32_t* const* codes, const uint32_t* g, int nterms, size_t n, uint64_t* out9);

/* Sample preparation on the device (Session::prepare's FE-id compression and sample drops;
 * host arrays in and out). Bit-exact with the reference's definitions.
 * fereg_factorize: factor.rs:38, dense codes in ascending value order (-0 = +0; NaN: 198).
 * fereg_combine: factor.rs:255, codes of the interaction of np code columns in lexicographic order.
 * fereg_drop_singletons: sample.rs:44-72, cyclic passes over the terms in absorb order until
 *   nterms consecutive passes drop nothing; a level with (fweight) count 1 drops its rows
 *   (when `singletons`), and with family 1 (Poisson) / 2 (logit) and its outcome y, a level
 *   whose alive rows have no nonzero outcome (logit: or only nonzero outcomes) is `fe`-separated.
 *   alive (n bytes, 0/1) is updated in place; counts of both kinds are returned.
 * fereg_restrict: factor.rs:281, the kept rows' codes renumbered densely in order (out holds
 *   the kept rows only). */
int fereg_factorize(const double* x, size_t n, uint32_t* codes, uint32_t* nlevels);
int fereg_combine(const uint32_t* const* parts, const uint32_t* nl, int np, size_t n, uint32_t* codes,
                  uint32_t* nlevels);
int fereg_drop_singletons(const uint32_t* const* codes, const uint32_t* g, int nterms, size_t n, const double* fw,
                          const double* y, int family, int singletons, uint8_t* alive, uint64_t* dropped_singletons,
                          uint64_t* dropped_separated);
int fereg_restrict(const uint32_t* codes, uint32_t g, const uint8_t* alive, size_t n, uint32_t* out,
                   uint32_t* nlevels, uint64_t* kept);

/* Serving: a request loop over independent regressions on one GPU. Requests are admitted in
 * arrival order while their estimated device memory fits the budget (hbm_budget bytes; 0 = 80%
 * of the free memory at creation); `workers` requests run at once, each on its own session and
 * CUDA stream. A request larger than the whole budget is rejected by fereg_server_submit (909).
 * Results do not depend on the other requests in flight. dry_run: the scheduler alone, no GPU
 * (each request sleeps dry_run_us; needs an explicit budget). */
typedef struct fereg_server fereg_server;
typedef struct fereg_server_config {
    int workers;
    size_t hbm_budget;
    int dry_run;
} fereg_server_config;

#define FEREG_MODEL_OLS 0
#define FEREG_MODEL_IV 1
#define FEREG_MODEL_LOGIT 2
#define FEREG_MODEL_POISSON 3

/* One regression: the prepared sample as for fereg_session_create (kept order), the data as
 * kept-order columns [y, exog (nx), endog (nendog), inst (ninst)], the estimator's options
 * (vce as the estimator's own entry point; maxiter is the inner solve's) and caller buffers for
 * b and V (k_all and k_all^2 values: OLS nx + 1, IV nendog + nx, GLM nx). Everything the
 * request points to must stay valid until fereg_server_wait returns for it. */
typedef struct fereg_request {
    int model;
    const uint32_t* const* codes;
    const uint32_t* g;
    int nterms;
    const uint32_t* const* cl_codes;
    const uint32_t* cl_g;
    int ncl;
    const double* w;
    int weight_kind;
    size_t n;
    const double* const* cols;
    size_t nx, nendog, ninst;
    int vce;
    double tol;
    size_t maxiter;
    int precision;
    double* b;
    double* V;
    uint64_t dry_run_us;
} fereg_request;

typedef struct fereg_request_result {
    int rc;                            /* the estimator's return code */
    double submit_s, admit_s, done_s;  /* seconds since the server started */
    uint64_t bytes;                    /* the admission estimate */
    double N;
    uint64_t iterations;               /* PCG iterations (GLM: over all IRLS steps) */
    int32_t converged;
    uint64_t launches;                 /* kernels the request launched */
    double prep_s;                     /* session preparation and row gather (inside admit..done) */
} fereg_request_result;

int fereg_server_create(const fereg_server_config* cfg, fereg_server** out);
int fereg_server_submit(fereg_server* srv, const fereg_request* req, uint64_t* ticket);
/* Blocks until the request is done; msg (msg_cap bytes, may be NULL) receives its error text.
 * One waiter per ticket. */
int fereg_server_wait(fereg_server* srv, uint64_t ticket, fereg_request_result* out, char* msg, size_t msg_cap);
/* 8 values: submitted, completed, rejected, peak admitted bytes, peak running, budget, running,
 * kernel launches of the completed requests. */
int fereg_server_stats(const fereg_server* srv, uint64_t* out8);
/* Waits for the running requests; pending ones are dropped. */
void fereg_server_destroy(fereg_server* srv);

/* Phase timing of the session's calls: the FEREG_PHASE_SLOTS slots of its absorber, then
 * 9 degrees of freedom, 10 column statistics, 11 Gram, 12 residuals and variance (GLM: the
 * regression update and the deviance), 13 GLM working variables and the device weight refresh. */
#define FEREG_SESSION_PHASE_SLOTS (FEREG_PHASE_SLOTS + 5)
int fereg_session_set_profiling(fereg_session* s, int on);
int fereg_session_phase_times(const fereg_session* s, double* ms, uint64_t* counts);

/* fereg_absorber_info of the session's absorber (9 values). */
int fereg_session_info(const fereg_session* s, uint64_t* out9);

/* Counters of the device PCG loop since the handle was made (no counterpart in the reference):
 * out4 = [iteration graphs captured, graph launches, host microseconds spent capturing and
 * instantiating them, FP32-refined solves that finished in FP64]. */
int fereg_absorber_solver_stats(const fereg_absorber* h, uint64_t* out4);
/* fereg_absorber_solver_stats of the session's absorber. */
int fereg_session_solver_stats(const fereg_session* s, uint64_t* out4);

/* Kernel launches of the session so far (its passes and its absorber), and its CUDA stream. */
uint64_t fereg_session_launches(const fereg_session* s);
void* fereg_session_stream(const fereg_session* s);

/* Bytes of the static device scratch of fereg_absorber_rhs_noalloc. */
#define FEREG_RHS_NOALLOC_SCRATCH_BYTES (16u << 20)

/* The right-hand side pass of fereg_absorber_rhs on device buffers, allocating nothing. No
 * counterpart in the reference. It serves callers that must not allocate device memory once they
 * run: a serving loop that shares the GPU with other streams (cudaFree waits for the whole device,
 * cudaMalloc can stall) and hosts that hand all device memory to their own pool at start-up (an
 * allocation inside the call could fail mid-run).
 * rows: n x r row-major (row order); y: m x r; b1: g1 x r; colsum: 3 x r ([sum w v^2; sum w v;
 * sum b1^2 / n1] per column); all device memory of the current device, which is the handle's.
 * Scratch comes from one static device array of FEREG_RHS_NOALLOC_SCRATCH_BYTES (16 MiB); a call
 * that needs more (many columns, many slices of long lists) returns 198 with the size in the
 * message. The first call on a device resolves the array's address (cudaGetSymbolAddress): make
 * that first call before any stream capture. The work is queued on the handle's stream
 * (fereg_absorber_stream) and the call returns without waiting for it. Every call on a device
 * uses the same scratch: calls that can overlap in time (other handles, or streams not ordered
 * against the handle's) race. */
int fereg_absorber_rhs_noalloc(fereg_absorber* h, const double* rows, size_t r, double* y, double* b1, double* colsum);

#ifdef __cplusplus
}
#endif

#endif
