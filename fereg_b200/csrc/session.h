// GpuSession: the estimation session around the B200 absorber, the part of the reference's
// `Session` (crates/fereg-core/src/session.rs) that `Session::ols` (ols.rs:199-470) uses: the
// kept-order FE term codes, cluster codes, weights and their kind, and the absorber built on the
// terms. The OLS call runs its row passes on the device (column statistics, the solve, the Gram,
// residuals and meats) and its K x K algebra on the host.
#pragma once

#include <future>
#include <memory>
#include <vector>

#include "absorber.h"

namespace fereg {

struct OlsSpec {
    int vce = 0;  // 0 unadjusted, 1 robust (HC1), 2 cluster (CRV1, one- or multiway)
    int noconstant = 0;
    int firstpair = 0;
    int want_groupvar = 0;
    double tol = 1e-8;
    size_t maxiter = 16000;
    Precision prec = Precision::F64;
};

// Results of ols.rs:263-470 (EstResult): caller buffers may be null.
struct OlsOut {
    double* b = nullptr;         // nx + 1 ([x..., _cons])
    double* V = nullptr;         // (nx + 1)^2
    uint8_t* status = nullptr;   // nx: 0 ok, 2 absorbed by the FE, 3 collinear
    double* resid = nullptr;     // n, kept order
    double* d = nullptr;         // n, kept order: sum of the fixed effects
    double* groupvar = nullptr;  // n, kept order: mobility group of the first FE pair
    double* dof_table = nullptr; // 5 per FE term (max 64): levels, redundant, k - m, inexact, nested
    int nslots = 0, k_all = 0, y_absorbed = 0;
    double N = 0, rank = 0, df_r = 0, df_m = 0, df_a = 0, df_a_initial = 0, df_a_redundant = 0, df_a_nested = 0;
    double N_clust = 0, N_clustervars = 0, N_clust1 = 0, N_clust2 = 0, num_singletons = 0, N_full = 0;
    double report_constant = 0;
    double rss = 0, tss = 0, tss_within = 0, mss = 0, rmse = 0, r2 = 0, r2_a = 0, r2_within = 0, r2_a_within = 0;
    double ll = 0, ll_0 = 0, F = 0, sumweights = 0, ic = 0;
};

struct SessionDev;
struct DofScratch;

// The shape of one absorb term beyond its codes: intercept flag and slope variables (kept order,
// n values each).
struct TermShape {
    bool intercept = true;
    std::vector<const double*> slopes;
};

class GpuSession {
   public:
    // codes[q]: kept-order codes of FE term q (< g[q]); no terms = the constant alone (noabsorb).
    // cl_codes[c]: kept-order codes of cluster dimension c. w: raw kept-order weights or null;
    // weight_kind 0 none, 1 aweight, 2 fweight, 3 pweight. num_singletons: rows the session's
    // preparation dropped as singletons (reported in N_full).
    // shapes (null: every term intercept-only): per term its intercept flag and slope variables
    // (kept order); a term with slopes or without an intercept makes the absorber the slope
    // solver (solve.rs:338).
    GpuSession(const std::vector<const u32*>& codes, const std::vector<u32>& g,
               const std::vector<const u32*>& cl_codes, const std::vector<u32>& cl_g, const double* w, int weight_kind,
               size_t n, u64 num_singletons, const Ctx& ctx, const std::vector<TermShape>* shapes = nullptr);
    ~GpuSession();

    DeviceAbsorber& absorber() { return *ab_; }
    const DeviceAbsorber& absorber() const { return *ab_; }
    size_t n() const { return n_; }
    // Kernel launches of the session passes and its absorber so far.
    u64 launches() const;

    // Phase timing: the absorber's slots (GpuAbsorber::Slot), then the session's own.
    enum Slot { S_DOF = 0, S_COLSTATS, S_GRAM, S_VARIANCE, S_WEIGHTS, S_NSLOTS };
    void set_profiling(bool on);
    void phase_times(double* ms, u64* counts) const;  // GpuAbsorber::P_NSLOTS + S_NSLOTS slots

    // Gathers R kept-order host columns (n values each) into the session's device row-order
    // block (n x R row-major, the layout every estimator reads) and returns it; it stays valid
    // until the next gather or estimator call with host rows.
    double* gather_columns(const double* const* cols, size_t R);

    // OLS of column 0 on columns 1..nx of the n x (1 + nx) row-major block `rows` (row order;
    // host memory, or device memory when on_device). A device block is residualized in place; a
    // host block is copied to the device and left unchanged.
    void ols(double* rows, bool on_device, size_t nx, const OlsSpec& spec, OlsOut& out);

    // Wild cluster bootstrap of one coefficient (see boot.cu).
    struct BootSpec {
        size_t coef = 0;    // index among the nx regressors
        double r0 = 0.0;    // H0: beta[coef] = r0
        size_t reps = 999;  // draws (full enumeration when 2^G <= reps and G <= 20)
        u64 seed = 1;
        size_t tile = 256;  // draws residualized together as block-PCG columns
        double tol = 1e-8;
        size_t maxiter = 16000;
        Precision prec = Precision::F64;
    };
    struct BootOut {
        double stat = 0, se = 0, point = 0, pvalue = 0;
        u64 reps = 0;
        bool full_enum = false;
        double* t_boot = nullptr;  // reps values
    };
    void wildboot(double* rows, bool on_device, size_t nx, const OlsSpec& ospec, const BootSpec& bs, BootOut& out);

    // IV / 2SLS on the session's FE (see session.cu).
    struct IvSpec {
        int vce = 0;  // 0 unadjusted, 1 robust, 2 cluster (one- or multiway)
        double tol = 1e-8;
        size_t maxiter = 16000;
        Precision prec = Precision::F64;
    };
    struct IvOut {
        double* b = nullptr;        // ne + nx: [endog..., exog...]; dropped columns 0
        double* V = nullptr;        // (ne + nx)^2
        uint8_t* status = nullptr;  // nx + ne + ni in block order: 0 ok, 2 absorbed, 3 collinear
        double N = 0, df_r = 0, df_m = 0, df_a = 0, sdofminus = 0, rss = 0, rmse = 0, F = 0, N_clust = 0, ic = 0;
        int endog_ct = 0, inexog_ct = 0, exexog_ct = 0;
    };
    void iv(double* rows, bool on_device, size_t nx, size_t ne, size_t ni, const IvSpec& spec, IvOut& out);

    // GLM by IRLS on the session's FE (see session.cu): Poisson PML or logit.
    struct GlmSpec {
        int family = 0;  // 0 Poisson, 1 logit
        int vce = 1;     // 0 oim (inverse Hessian), 1 robust, 2 cluster
        double tol = 1e-8;    // deviance tolerance
        double itol = 1e-10;  // final inner (FE solve) tolerance
        size_t maxiter = 10000;
        size_t inner_maxiter = 16000;
        Precision prec = Precision::F64;
    };
    struct GlmOut {
        double* b = nullptr;        // nx (absorbed / collinear columns 0)
        double* V = nullptr;        // nx x nx
        uint8_t* status = nullptr;  // nx: 0 ok, 2 absorbed, 3 collinear
        double N = 0, deviance = 0, ll = 0, chi2 = 0, df_m = 0, N_clust = 0;
        u64 iterations = 0, pcg_iterations = 0;
        bool converged = false;
    };
    void glm(double* rows, bool on_device, size_t nx, const GlmSpec& gs, GlmOut& out);

    // One ReLU separation check (glm/separation.rs:61-196) of the Poisson outcome y (column 0)
    // with the regressors (columns 1..nx) of the n x (1 + nx) block (row order; host or device
    // memory), standardized by their standard deviations (glm/mod.rs:4-6): weighted FE solves of
    // the ReLU working variable until the prediction is non-negative on the y = 0 rows.
    struct ReluSpec {
        double itol = 1e-10;  // the GLM's inner tolerance (its collinearity rule, glm/mod.rs:7-8)
        size_t inner_maxiter = 16000;
        Precision prec = Precision::F64;
    };
    struct ReluOut {
        uint8_t* separated = nullptr;  // n, row order: 1 on the separated rows
        double* certificate = nullptr; // n, row order: the certificate (positive on them, else 0)
        u64 num_separated = 0, iterations = 0, pcg_iterations = 0;
        bool complete = false;  // the check certified its result
        int dropped_collinear = 0;
    };
    void relu_separation(double* rows, bool on_device, size_t nx, const ReluSpec& rs, ReluOut& out);

   private:
    size_t n_ = 0;
    int kind_ = 0;
    u64 nsing_ = 0;
    std::vector<u32> tg_, cg_;
    std::vector<std::vector<u32>> tcodes_, ccodes_;  // kept order (host)
    std::vector<double> wk_;                         // raw kept-order weights
    double sumw_ = 0;
    std::unique_ptr<DeviceAbsorber> ab_;
    std::unique_ptr<SessionDev> d_;
    // per term: intercept flag, slope count, and per slope the levels on which it is redundant
    // (dof.rs:165-176, reghdfe dof_update_cvars), fixed by the session's data
    std::vector<bool> t_icpt_;
    std::vector<std::vector<u64>> slope_red_;
    bool irls_weights_ = false;  // a GLM call left its IRLS weights on the absorber
    void restore_weights();
    // CRV3 (crv3.rs, ols/stata_vce.rs:516-545): the jackknife meat of [b, _cons] over the cluster
    // subsets; rows: the residualized block (device), raw_h: the raw rows (host, row order),
    // g: the weighted Gram of the residualized block.
    std::vector<double> crv3_meat(const double* rows, const std::vector<double>& raw_h, int R,
                                  const std::vector<size_t>& kept, const std::vector<double>& beta,
                                  const std::vector<double>& wmean, bool report_constant, const std::vector<double>& g);

    struct DofSlot {
        u64 k = 0, m = 0;
        bool exact = false, nested = false;
    };
    struct Dof {
        std::vector<DofSlot> slots;
        u64 df_a = 0, df_a_initial = 0, df_a_redundant = 0, df_a_nested = 0;
        bool has_groupvar = false;
    };
    // The dof pass, joined at once.
    Dof estimate_dof(bool clusters, bool firstpair, bool want_groupvar);
    // The same pass started on its own stream and host thread; dof_end joins it.
    std::future<Dof> dof_begin(bool clusters, bool firstpair, bool want_groupvar);
    Dof dof_end(std::future<Dof>& job);
    Dof dof_pass(bool clusters, bool firstpair, bool want_groupvar, DofScratch& s);
    struct ColStats {
        std::vector<double> wmean, sumsq, wss_unc, sd, wss;
    };
    ColStats column_stats(const double* rows, int R);
    void column_stats_alloc(int R);
    void column_stats_launch(const double* rows, int R, cudaStream_t cs, double* s1, double* c0, int* late);
    ColStats column_stats_finish(const double* s1, const double* c0, int late, int R) const;
    std::vector<double> outer_products(const double* src, size_t nrows, int srcR, const std::vector<int>& cols,
                                       const std::vector<double>* shift, bool cst, const double* om, const int* perm,
                                       bool ssq, std::vector<double>* ss_out);
    // What the last ols() call fitted (the bootstrap's starting point).
    struct FitState {
        bool ok = false;                // a cluster variance was computed
        std::vector<size_t> kept;       // columns (1..nx) of the kept regressors
        std::vector<double> A, beta;    // raw (X~'W X~)^-1 of the kept columns, coefficients
        double crv1_scale = 0.0;        // CRV1 small-sample factor
        double* rows = nullptr;         // the residualized block (device)
        size_t R = 0;
        bool y_absorbed = false;
    };
    FitState fit_;
    u64 mobility_groups(size_t qa, size_t qb, bool save, DofScratch& s);
    bool nested_within(size_t q, size_t c, DofScratch& s);
};

}  // namespace fereg
