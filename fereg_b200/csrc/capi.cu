// extern "C" boundary: exceptions become the reference's return codes plus a thread-local
// message; nothing throws across.

#include <mutex>
#include <new>

#include "../../include/fereg_b200.h"
#include "absorber.h"
#include "amg.h"
#include "dstruct.h"
#include "prep.h"
#include "server.h"
#include "session.h"
#include "slopes.h"

using namespace fereg;

struct fereg_absorber {
    std::unique_ptr<DeviceAbsorber> a;
    GpuAbsorber* fe = nullptr;     // the intercept-only solver, when it is the absorber
    GpuSlopeSolver* sl = nullptr;  // the heterogeneous-slope solver, when it is
    explicit fereg_absorber(std::unique_ptr<GpuAbsorber> f) : fe(f.get()) { a = std::move(f); }
    explicit fereg_absorber(std::unique_ptr<GpuSlopeSolver> f) : sl(f.get()) { a = std::move(f); }
};

namespace {
// The absorber of a handle as the intercept-only solver or as the slope solver (198 otherwise).
fereg::GpuAbsorber& fe_of(const fereg_absorber* h, const char* what) {
    if (!h) throw fereg::Error(fereg::RC_INVALID_INPUT, std::string(what) + ": NULL handle");
    if (!h->fe) throw fereg::Error(fereg::RC_INVALID_INPUT, std::string(what) + ": the absorber has slope terms");
    return *h->fe;
}
fereg::GpuSlopeSolver& sl_of(const fereg_absorber* h, const char* what) {
    if (!h) throw fereg::Error(fereg::RC_INVALID_INPUT, std::string(what) + ": NULL handle");
    if (!h->sl) throw fereg::Error(fereg::RC_INVALID_INPUT, std::string(what) + ": the absorber has no slope terms");
    return *h->sl;
}
}  // namespace

struct fereg_session {
    GpuSession s;
    template <class... A>
    explicit fereg_session(A&&... args) : s(std::forward<A>(args)...) {}
};

namespace {

template <class F>
int guard(F f) {
    try {
        f();
        return RC_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.rc;
    } catch (const std::bad_alloc&) {
        set_last_error("fereg: insufficient memory");
        return RC_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        set_last_error(std::string("fereg internal error: ") + e.what());
        return RC_INTERNAL;
    } catch (...) {
        set_last_error("fereg internal error");
        return RC_INTERNAL;
    }
}

Ctx to_ctx(const fereg_ctx* c) {
    Ctx x;
    if (c) {
        x.interrupt = c->interrupt;
        x.interrupt_data = c->interrupt_data;
        x.log = c->log;
        x.log_data = c->log_data;
        x.verbose = c->verbose;
    }
    return x;
}

// Scratch of fereg_absorber_rhs_noalloc: a file-scope device array, so the call needs no
// allocation. Its address is resolved once per device (cudaGetSymbolAddress, that device current)
// by the first call on the device. Every call on a device uses the same array.
constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(FEREG_RHS_NOALLOC_SCRATCH_BYTES);
static __device__ __align__(256) double g_rhs_scratch[NOALLOC_SCRATCH_BYTES / sizeof(double)];
constexpr int NOALLOC_MAX_DEVICES = 64;
double* g_rhs_scratch_addr[NOALLOC_MAX_DEVICES] = {};
std::mutex g_rhs_scratch_mu;

double* rhs_scratch_on_current_device() {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) throw Error(RC_INTERNAL, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) throw Error(RC_INTERNAL, "fereg: device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_rhs_scratch_mu);
    if (!g_rhs_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_rhs_scratch);
        if (e != cudaSuccess) throw Error(RC_INTERNAL, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_rhs_scratch_addr[dev] = static_cast<double*>(p);
    }
    return g_rhs_scratch_addr[dev];
}

// fereg_absorber_info: n, m, g1, ncells, nb, m_small, fe1, small_work, small blocks.
// The terms of a *_create_terms call: intercept[q] (null: 1), nslopes[q] (null: 0) and the slope
// variables of all terms, term after term (sum nslopes pointers).
std::vector<SlopeTermIn> slope_terms(const uint32_t* const* codes, const uint32_t* g, const int* intercept,
                                     const int* nslopes, const double* const* slopes, int nterms) {
    std::vector<SlopeTermIn> t(static_cast<size_t>(nterms));
    size_t k = 0;
    for (int q = 0; q < nterms; q++) {
        SlopeTermIn& x = t[size_t(q)];
        x.codes = codes[q];
        x.g = g[q];
        x.intercept = intercept ? intercept[q] != 0 : true;
        const int ns = nslopes ? nslopes[q] : 0;
        if (ns < 0 || (ns > 0 && !slopes)) throw Error(RC_INVALID_INPUT, "fereg: bad slope variables");
        for (int s = 0; s < ns; s++) x.slopes.push_back(slopes[k++]);
        if (!x.codes || x.g == 0) throw Error(RC_INVALID_INPUT, "fereg: empty term");
    }
    return t;
}

void fill_info_fe(const GpuAbsorber& a, uint64_t* o) {
    const auto& st = a.structure();
    o[0] = st.n;
    o[1] = st.m;
    o[2] = st.g1;
    o[3] = st.ncells;
    o[4] = st.nb();
    o[5] = st.m_small;
    o[6] = uint64_t(int64_t(st.fe1));
    o[7] = st.small_work;
    u64 ns = 0;
    for (const auto& b : st.blocks) ns += b.small ? 1 : 0;
    o[8] = ns;
}

// The same for either absorber; the slope solver reports n, m, G_E, n (every row its own cell),
// the blocks, the small coordinates, E, 0 and the small blocks.
void fill_info(const DeviceAbsorber& a, uint64_t* o) {
    if (const auto* fe = dynamic_cast<const GpuAbsorber*>(&a)) return fill_info_fe(*fe, o);
    const auto& st = dynamic_cast<const GpuSlopeSolver&>(a).structure();
    o[0] = st.n;
    o[1] = st.m;
    o[2] = st.ge;
    o[3] = st.n;
    o[4] = st.blocks.size();
    o[5] = st.m_small;
    o[6] = st.e;
    o[7] = 0;
    o[8] = st.nsmall;
}

void fill(fereg_solve_info* info, const SolveInfo& s) {
    if (!info) return;
    info->iterations = s.iterations;
    info->escalated = s.escalated;
    info->exact = s.exact;
}

}  // namespace

extern "C" {

const char* fereg_last_error(void) { return last_error(); }

int fereg_absorber_create(const uint32_t* const* codes, const uint32_t* g, int nterms, const double* w, size_t n,
                          const fereg_ctx* ctx, fereg_absorber** out) {
    return guard([&] {
        if (!out) throw Error(RC_INVALID_INPUT, "fereg_absorber_create: out is NULL");
        *out = nullptr;
        if (nterms < 0 || (nterms > 0 && (!codes || !g))) throw Error(RC_INVALID_INPUT, "fereg_absorber_create: bad terms");
        if (n < 2) throw Error(RC_TOO_FEW_OBS, "insufficient observations");
        if (n >= (size_t(1) << 32)) throw Error(RC_INVALID_INPUT, "more than 2^32 - 1 rows");
        std::vector<const u32*> cs(codes, codes + nterms);
        std::vector<u32> gs(g, g + nterms);
        for (int q = 0; q < nterms; q++)
            if (!cs[size_t(q)] || gs[size_t(q)] == 0) throw Error(RC_INVALID_INPUT, "fereg_absorber_create: empty term");
        *out = new fereg_absorber(std::make_unique<GpuAbsorber>(cs, gs, w, n, to_ctx(ctx)));
    });
}

int fereg_absorber_create_terms(const uint32_t* const* codes, const uint32_t* g, const int* intercept,
                                const int* nslopes, const double* const* slopes, int nterms, const double* w, size_t n,
                                const fereg_ctx* ctx, fereg_absorber** out) {
    return guard([&] {
        if (!out) throw Error(RC_INVALID_INPUT, "fereg_absorber_create_terms: out is NULL");
        *out = nullptr;
        if (nterms <= 0 || !codes || !g) throw Error(RC_INVALID_INPUT, "fereg_absorber_create_terms: bad terms");
        if (n < 2) throw Error(RC_TOO_FEW_OBS, "insufficient observations");
        if (n >= (size_t(1) << 32)) throw Error(RC_INVALID_INPUT, "more than 2^32 - 1 rows");
        const std::vector<SlopeTermIn> terms = slope_terms(codes, g, intercept, nslopes, slopes, nterms);
        bool plain = true;
        for (const auto& t : terms) plain &= t.intercept && t.slopes.empty();
        if (plain) {
            std::vector<const u32*> cs(codes, codes + nterms);
            std::vector<u32> gs(g, g + nterms);
            *out = new fereg_absorber(std::make_unique<GpuAbsorber>(cs, gs, w, n, to_ctx(ctx)));
        } else {
            *out = new fereg_absorber(std::make_unique<GpuSlopeSolver>(terms, w, n, to_ctx(ctx)));
        }
    });
}

int fereg_absorber_has_slopes(const fereg_absorber* h) { return h && h->sl ? 1 : 0; }

size_t fereg_absorber_term_values_len(const fereg_absorber* h) { return h ? h->a->term_values_len() : 0; }

int fereg_slope_weight_state(const fereg_absorber* h, double* minv, double* jinv, uint8_t* redundant) {
    return guard([&] { sl_of(h, "fereg_slope_weight_state").weight_state(minv, jinv, redundant); });
}

int fereg_slope_apply(fereg_absorber* h, const double* p, size_t r, double* y) {
    return guard([&] { sl_of(h, "fereg_slope_apply").apply_host(p, r, y); });
}

int fereg_slope_precond(fereg_absorber* h, const double* rr, size_t r, double* z) {
    return guard([&] { sl_of(h, "fereg_slope_precond").precond_host(rr, r, z); });
}

int fereg_slope_rhs(fereg_absorber* h, const double* rows, size_t r, double* y, double* stats) {
    return guard([&] { sl_of(h, "fereg_slope_rhs").rhs_host(rows, r, y, stats); });
}

int fereg_slope_structure(const fereg_absorber* h, uint64_t* o, uint32_t* block_terms) {
    return guard([&] {
        const SlopeHost& st = sl_of(h, "fereg_slope_structure").structure();
        if (o) {
            o[0] = st.n;
            o[1] = st.m;
            o[2] = st.e;
            o[3] = st.ge;
            o[4] = st.be;
            o[5] = st.k;
            o[6] = st.blocks.size();
            o[7] = st.nsmall;
            o[8] = st.m_small;
        }
        if (block_terms)
            for (size_t q = 0; q < st.blocks.size(); q++) block_terms[q] = uint32_t(st.blocks[q].term);
    });
}

void fereg_absorber_destroy(fereg_absorber* h) { delete h; }

size_t fereg_absorber_n(const fereg_absorber* h) { return h ? h->a->n() : 0; }

size_t fereg_absorber_coefs_len(const fereg_absorber* h) { return h ? h->a->coefs_len() : 0; }

int fereg_absorber_row_order(const fereg_absorber* h, uint32_t* out) {
    return guard([&] {
        if (!h || !out) throw Error(RC_INVALID_INPUT, "fereg_absorber_row_order: NULL argument");
        const auto& pi = h->a->row_order();
        std::copy(pi.begin(), pi.end(), out);
    });
}

int fereg_absorber_weights(const fereg_absorber* h, double* out, int* has) {
    return guard([&] {
        if (!h || !has) throw Error(RC_INVALID_INPUT, "fereg_absorber_weights: NULL argument");
        *has = h->a->weights(out) ? 1 : 0;
    });
}

int fereg_absorber_set_weights(fereg_absorber* h, const double* w) {
    return guard([&] {
        if (!h) throw Error(RC_INVALID_INPUT, "fereg_absorber_set_weights: NULL handle");
        h->a->set_weights(w);
    });
}

int fereg_absorber_set_weights_device(fereg_absorber* h, const double* w_dev) {
    return guard([&] {
        if (!h || !w_dev) throw Error(RC_INVALID_INPUT, "fereg_absorber_set_weights_device: NULL argument");
        h->a->set_weights_device(w_dev);
    });
}

int fereg_absorber_residualize(fereg_absorber* h, double* z, size_t r, double tol, size_t maxiter, int want_coefs,
                               const double* warm, double* coefs_out, fereg_solve_info* info) {
    return fereg_absorber_residualize_ex(h, z, 0, r, tol, maxiter, want_coefs, warm, coefs_out, FEREG_PREC_F64, info);
}

int fereg_absorber_residualize_ex(fereg_absorber* h, double* z, int z_on_device, size_t r, double tol, size_t maxiter,
                                  int want_coefs, const double* warm, double* coefs_out, int precision,
                                  fereg_solve_info* info) {
    return guard([&] {
        if (!h) throw Error(RC_INVALID_INPUT, "fereg_absorber_residualize: NULL handle");
        if (r > 0 && !z) throw Error(RC_INVALID_INPUT, "residualize: block size differs from n*R");
        if (!(tol > 0.0)) throw Error(RC_INVALID_INPUT, "residualize: tol must be positive");
        if (precision != FEREG_PREC_F64 && precision != FEREG_PREC_F32_REFINED)
            throw Error(RC_INVALID_INPUT, "residualize: unknown precision");
        const Precision p = Precision(precision);
        SolveInfo s = z_on_device ? h->a->residualize_device(z, r, tol, maxiter, want_coefs != 0, warm, coefs_out, p)
                                  : h->a->residualize(z, r, tol, maxiter, want_coefs != 0, warm, coefs_out, p);
        fill(info, s);
    });
}

int fereg_absorber_fit_rows(const fereg_absorber* h, const double* coefs, size_t r, size_t col, double* out) {
    return guard([&] {
        if (!h || !coefs || !out) throw Error(RC_INVALID_INPUT, "fereg_absorber_fit_rows: NULL argument");
        if (col >= r) throw Error(RC_INVALID_INPUT, "fit_rows: column out of range");
        h->a->fit_rows(coefs, r, col, out);
    });
}

int fereg_absorber_term_values(const fereg_absorber* h, const double* coefs, size_t r, size_t col, double* out) {
    return guard([&] {
        if (!h || !coefs || !out) throw Error(RC_INVALID_INPUT, "fereg_absorber_term_values: NULL argument");
        if (col >= r) throw Error(RC_INVALID_INPUT, "term_values: column out of range");
        h->a->term_values(coefs, r, col, out);
    });
}

void* fereg_absorber_stream(const fereg_absorber* h) { return h ? static_cast<void*>(h->a->stream()) : nullptr; }

int fereg_absorber_set_profiling(fereg_absorber* h, int on) {
    return guard([&] {
        if (!h) throw Error(RC_INVALID_INPUT, "fereg_absorber_set_profiling: NULL handle");
        h->a->set_profiling(on != 0);
    });
}

int fereg_absorber_phase_times(const fereg_absorber* h, double* ms, uint64_t* counts) {
    return guard([&] {
        if (!h) throw Error(RC_INVALID_INPUT, "fereg_absorber_phase_times: NULL handle");
        h->a->phase_times(ms, counts);
    });
}

uint64_t fereg_absorber_launches(const fereg_absorber* h) { return h ? h->a->launches() : 0; }

int fereg_absorber_escalations(const fereg_absorber* h, uint64_t* escalations, uint64_t* blocks) {
    return guard([&] {
        if (!h) throw Error(RC_INVALID_INPUT, "fereg_absorber_escalations: NULL handle");
        if (escalations) *escalations = h->a->escalations();
        if (blocks) *blocks = h->a->escalated_blocks();
    });
}

int fereg_absorber_info(const fereg_absorber* h, uint64_t* o) {
    return guard([&] {
        if (!h || !o) throw Error(RC_INVALID_INPUT, "fereg_absorber_info: NULL argument");
        fill_info(*h->a, o);
    });
}

int fereg_session_info(const fereg_session* s, uint64_t* o) {
    return guard([&] {
        if (!s || !o) throw Error(RC_INVALID_INPUT, "fereg_session_info: NULL argument");
        fill_info(s->s.absorber(), o);
    });
}

int fereg_absorber_solver_stats(const fereg_absorber* h, uint64_t* o) {
    return guard([&] {
        if (!h || !o) throw Error(RC_INVALID_INPUT, "fereg_absorber_solver_stats: NULL argument");
        h->a->solver_stats(o);
    });
}

int fereg_session_solver_stats(const fereg_session* s, uint64_t* o) {
    return guard([&] {
        if (!s || !o) throw Error(RC_INVALID_INPUT, "fereg_session_solver_stats: NULL argument");
        s->s.absorber().solver_stats(o);
    });
}

int fereg_absorber_apply(fereg_absorber* h, const double* p, size_t r, double* y) {
    return guard([&] { fe_of(h, "fereg_absorber_apply").apply_host(p, r, y); });
}

int fereg_absorber_rhs(fereg_absorber* h, const double* rows, size_t r, double* y, double* b1, double* wsq, double* wsum) {
    return guard([&] { fe_of(h, "fereg_absorber_rhs").rhs_host(rows, r, y, b1, wsq, wsum); });
}

int fereg_absorber_rhs_noalloc(fereg_absorber* h, const double* rows, size_t r, double* y, double* b1,
                               double* colsum) {
    return guard([&] {
        if (!h) throw Error(RC_INVALID_INPUT, "fereg_absorber_rhs_noalloc: NULL handle");
        double* scratch = rhs_scratch_on_current_device();
        fe_of(h, "fereg_absorber_rhs_noalloc").rhs_device_scratch(rows, r, y, b1, colsum, scratch, NOALLOC_SCRATCH_BYTES / sizeof(double));
    });
}

int fereg_absorber_precond(fereg_absorber* h, const double* rr, size_t r, double* z) {
    return guard([&] { fe_of(h, "fereg_absorber_precond").precond_host(rr, r, z); });
}

int fereg_absorber_weight_state(const fereg_absorber* h, double* n1, double* nr, double* diag, uint8_t* redundant, double* sw) {
    return guard([&] { fe_of(h, "fereg_absorber_weight_state").weight_state(n1, nr, diag, redundant, sw); });
}


int fereg_session_create(const uint32_t* const* codes, const uint32_t* g, int nterms, const uint32_t* const* cl_codes,
                         const uint32_t* cl_g, int ncl, const double* w, int weight_kind, size_t n,
                         uint64_t num_singletons, const fereg_ctx* ctx, fereg_session** out) {
    return guard([&] {
        if (!out) throw Error(RC_INVALID_INPUT, "fereg_session_create: out is NULL");
        *out = nullptr;
        if (nterms < 0 || ncl < 0 || (nterms > 0 && (!codes || !g)) || (ncl > 0 && (!cl_codes || !cl_g)))
            throw Error(RC_INVALID_INPUT, "fereg_session_create: bad terms or clusters");
        if (n < 2) throw Error(RC_TOO_FEW_OBS, "insufficient observations");
        if (n >= (size_t(1) << 31)) throw Error(RC_INVALID_INPUT, "more than 2^31 - 1 rows");
        std::vector<const u32*> cs(codes, codes + nterms), cc(cl_codes, cl_codes + ncl);
        std::vector<u32> gs(g, g + nterms), cgs(cl_g, cl_g + ncl);
        for (int q = 0; q < nterms; q++)
            if (!cs[size_t(q)] || gs[size_t(q)] == 0) throw Error(RC_INVALID_INPUT, "fereg_session_create: empty term");
        for (int c = 0; c < ncl; c++)
            if (!cc[size_t(c)] || cgs[size_t(c)] == 0) throw Error(RC_INVALID_INPUT, "fereg_session_create: empty cluster");
        *out = new fereg_session(cs, gs, cc, cgs, w, weight_kind, n, num_singletons, to_ctx(ctx));
    });
}

int fereg_session_create_terms(const uint32_t* const* codes, const uint32_t* g, const int* intercept,
                               const int* nslopes, const double* const* slopes, int nterms,
                               const uint32_t* const* cl_codes, const uint32_t* cl_g, int ncl, const double* w,
                               int weight_kind, size_t n, uint64_t num_singletons, const fereg_ctx* ctx,
                               fereg_session** out) {
    return guard([&] {
        if (!out) throw Error(RC_INVALID_INPUT, "fereg_session_create_terms: out is NULL");
        *out = nullptr;
        if (nterms <= 0 || ncl < 0 || !codes || !g || (ncl > 0 && (!cl_codes || !cl_g)))
            throw Error(RC_INVALID_INPUT, "fereg_session_create_terms: bad terms or clusters");
        if (n < 2) throw Error(RC_TOO_FEW_OBS, "insufficient observations");
        if (n >= (size_t(1) << 31)) throw Error(RC_INVALID_INPUT, "more than 2^31 - 1 rows");
        const std::vector<SlopeTermIn> terms = slope_terms(codes, g, intercept, nslopes, slopes, nterms);
        std::vector<const u32*> cs(codes, codes + nterms), cc(cl_codes, cl_codes + ncl);
        std::vector<u32> gs(g, g + nterms), cgs(cl_g, cl_g + ncl);
        for (int c = 0; c < ncl; c++)
            if (!cc[size_t(c)] || cgs[size_t(c)] == 0) throw Error(RC_INVALID_INPUT, "fereg_session_create: empty cluster");
        std::vector<TermShape> shapes(terms.size());
        for (size_t q = 0; q < terms.size(); q++) {
            shapes[q].intercept = terms[q].intercept;
            shapes[q].slopes = terms[q].slopes;
        }
        *out = new fereg_session(cs, gs, cc, cgs, w, weight_kind, n, num_singletons, to_ctx(ctx), &shapes);
    });
}

void fereg_session_destroy(fereg_session* s) { delete s; }

int fereg_session_row_order(const fereg_session* s, uint32_t* out) {
    return guard([&] {
        if (!s || !out) throw Error(RC_INVALID_INPUT, "fereg_session_row_order: NULL argument");
        const auto& pi = const_cast<fereg_session*>(s)->s.absorber().row_order();
        std::copy(pi.begin(), pi.end(), out);
    });
}

int fereg_session_ols(fereg_session* s, double* rows, int rows_on_device, size_t nx, const fereg_ols_spec* spec,
                      fereg_ols_out* out) {
    return guard([&] {
        if (!s || !rows || !spec || !out) throw Error(RC_INVALID_INPUT, "fereg_session_ols: NULL argument");
        if (spec->precision != FEREG_PREC_F64 && spec->precision != FEREG_PREC_F32_REFINED)
            throw Error(RC_INVALID_INPUT, "fereg_session_ols: unknown precision");
        OlsSpec sp;
        sp.vce = spec->vce;
        sp.noconstant = spec->noconstant;
        sp.firstpair = spec->firstpair;
        sp.want_groupvar = spec->want_groupvar;
        sp.tol = spec->tol;
        sp.maxiter = spec->maxiter;
        sp.prec = spec->precision == FEREG_PREC_F32_REFINED ? Precision::F32_REFINED : Precision::F64;
        if (sp.vce < 0 || sp.vce > 5) throw Error(RC_INVALID_INPUT, "fereg_session_ols: unknown vce");
        OlsOut o;
        o.b = out->b;
        o.V = out->V;
        o.status = out->status;
        o.resid = out->resid;
        o.d = out->d;
        o.groupvar = out->groupvar;
        o.dof_table = out->dof_table;
        s->s.ols(rows, rows_on_device != 0, nx, sp, o);
        out->nslots = o.nslots;
        out->k_all = o.k_all;
        out->y_absorbed = o.y_absorbed;
        out->N = o.N;
        out->rank = o.rank;
        out->df_r = o.df_r;
        out->df_m = o.df_m;
        out->df_a = o.df_a;
        out->df_a_initial = o.df_a_initial;
        out->df_a_redundant = o.df_a_redundant;
        out->df_a_nested = o.df_a_nested;
        out->N_clust = o.N_clust;
        out->N_clustervars = o.N_clustervars;
        out->N_clust1 = o.N_clust1;
        out->N_clust2 = o.N_clust2;
        out->num_singletons = o.num_singletons;
        out->N_full = o.N_full;
        out->report_constant = o.report_constant;
        out->rss = o.rss;
        out->tss = o.tss;
        out->tss_within = o.tss_within;
        out->mss = o.mss;
        out->rmse = o.rmse;
        out->r2 = o.r2;
        out->r2_a = o.r2_a;
        out->r2_within = o.r2_within;
        out->r2_a_within = o.r2_a_within;
        out->ll = o.ll;
        out->ll_0 = o.ll_0;
        out->F = o.F;
        out->sumweights = o.sumweights;
        out->ic = o.ic;
    });
}

int fereg_session_wildboot(fereg_session* s, double* rows, int rows_on_device, size_t nx, const fereg_ols_spec* spec,
                           const fereg_boot_spec* boot, fereg_boot_out* out) {
    return guard([&] {
        if (!s || !rows || !spec || !boot || !out) throw Error(RC_INVALID_INPUT, "fereg_session_wildboot: NULL argument");
        if (spec->precision != FEREG_PREC_F64 && spec->precision != FEREG_PREC_F32_REFINED)
            throw Error(RC_INVALID_INPUT, "fereg_session_wildboot: unknown precision");
        if (boot->precision != FEREG_PREC_F64 && boot->precision != FEREG_PREC_F32_REFINED)
            throw Error(RC_INVALID_INPUT, "fereg_session_wildboot: unknown bootstrap precision");
        OlsSpec sp;
        sp.vce = 2;
        sp.noconstant = spec->noconstant;
        sp.firstpair = spec->firstpair;
        sp.tol = spec->tol;
        sp.maxiter = spec->maxiter;
        sp.prec = spec->precision == FEREG_PREC_F32_REFINED ? Precision::F32_REFINED : Precision::F64;
        GpuSession::BootSpec bs;
        bs.coef = boot->coef;
        bs.r0 = boot->r0;
        bs.reps = boot->reps;
        bs.seed = boot->seed;
        bs.tile = boot->tile;
        bs.tol = boot->tol;
        bs.maxiter = boot->maxiter;
        bs.prec = boot->precision == FEREG_PREC_F32_REFINED ? Precision::F32_REFINED : Precision::F64;
        GpuSession::BootOut bo;
        bo.t_boot = out->t_boot;
        s->s.wildboot(rows, rows_on_device != 0, nx, sp, bs, bo);
        out->stat = bo.stat;
        out->se = bo.se;
        out->point = bo.point;
        out->pvalue = bo.pvalue;
        out->reps = bo.reps;
        out->full_enum = bo.full_enum ? 1 : 0;
    });
}

int fereg_session_iv(fereg_session* s, double* rows, int rows_on_device, size_t nx, size_t nendog, size_t ninst,
                     const fereg_iv_spec* spec, fereg_iv_out* out) {
    return guard([&] {
        if (!s || !rows || !spec || !out) throw Error(RC_INVALID_INPUT, "fereg_session_iv: NULL argument");
        if (spec->vce < 0 || spec->vce > 2) throw Error(RC_INVALID_INPUT, "fereg_session_iv: vce is 0, 1 or 2");
        if (spec->precision != FEREG_PREC_F64 && spec->precision != FEREG_PREC_F32_REFINED)
            throw Error(RC_INVALID_INPUT, "fereg_session_iv: unknown precision");
        GpuSession::IvSpec is;
        is.vce = spec->vce;
        is.tol = spec->tol;
        is.maxiter = spec->maxiter;
        is.prec = spec->precision == FEREG_PREC_F32_REFINED ? Precision::F32_REFINED : Precision::F64;
        GpuSession::IvOut io;
        io.b = out->b;
        io.V = out->V;
        io.status = out->status;
        s->s.iv(rows, rows_on_device != 0, nx, nendog, ninst, is, io);
        out->N = io.N;
        out->df_r = io.df_r;
        out->df_m = io.df_m;
        out->df_a = io.df_a;
        out->sdofminus = io.sdofminus;
        out->rss = io.rss;
        out->rmse = io.rmse;
        out->F = io.F;
        out->N_clust = io.N_clust;
        out->ic = io.ic;
        out->endog_ct = io.endog_ct;
        out->inexog_ct = io.inexog_ct;
        out->exexog_ct = io.exexog_ct;
    });
}

static int session_glm(fereg_session* s, double* rows, int rows_on_device, size_t nx, const fereg_glm_spec* spec,
                       fereg_glm_out* out, int family) {
    return guard([&] {
        if (!s || !rows || !spec || !out) throw Error(RC_INVALID_INPUT, "fereg_session_glm: NULL argument");
        if (family != FEREG_FAMILY_POISSON && family != FEREG_FAMILY_LOGIT)
            throw Error(RC_INVALID_INPUT, "fereg_session_glm: family is Poisson or logit");
        if (spec->vce != 1 && spec->vce != 2 && !(spec->vce == 0 && family == FEREG_FAMILY_LOGIT))
            throw Error(RC_INVALID_INPUT, "fereg_session_glm: vce is 1 or 2 (0 for logit)");
        if (spec->precision != FEREG_PREC_F64 && spec->precision != FEREG_PREC_F32_REFINED)
            throw Error(RC_INVALID_INPUT, "fereg_session_glm: unknown precision");
        GpuSession::GlmSpec gs;
        gs.family = family == FEREG_FAMILY_LOGIT ? 1 : 0;
        gs.vce = spec->vce;
        gs.tol = spec->tol;
        gs.itol = spec->itol > 0.0 ? spec->itol : 1e-10;
        gs.maxiter = spec->maxiter;
        gs.inner_maxiter = spec->inner_maxiter;
        gs.prec = spec->precision == FEREG_PREC_F32_REFINED ? Precision::F32_REFINED : Precision::F64;
        GpuSession::GlmOut go;
        go.b = out->b;
        go.V = out->V;
        go.status = out->status;
        s->s.glm(rows, rows_on_device != 0, nx, gs, go);
        out->N = go.N;
        out->deviance = go.deviance;
        out->ll = go.ll;
        out->chi2 = go.chi2;
        out->df_m = go.df_m;
        out->N_clust = go.N_clust;
        out->iterations = go.iterations;
        out->pcg_iterations = go.pcg_iterations;
        out->converged = go.converged ? 1 : 0;
    });
}

int fereg_session_relu(fereg_session* s, double* rows, int rows_on_device, size_t nx, double itol,
                       size_t inner_maxiter, uint8_t* separated, double* certificate, uint64_t* out4) {
    return guard([&] {
        if (!s || !rows) throw Error(RC_INVALID_INPUT, "fereg_session_relu: NULL argument");
        GpuSession::ReluSpec rs;
        rs.itol = itol;
        rs.inner_maxiter = inner_maxiter;
        GpuSession::ReluOut o;
        o.separated = separated;
        o.certificate = certificate;
        s->s.relu_separation(rows, rows_on_device != 0, nx, rs, o);
        if (out4) {
            out4[0] = o.num_separated;
            out4[1] = o.iterations;
            out4[2] = o.pcg_iterations;
            out4[3] = o.complete ? 1 : 0;
        }
    });
}

int fereg_session_glm(fereg_session* s, double* rows, int rows_on_device, size_t nx, const fereg_glm_spec* spec,
                      fereg_glm_out* out) {
    return session_glm(s, rows, rows_on_device, nx, spec, out, spec ? spec->family : 0);
}

int fereg_session_poisson(fereg_session* s, double* rows, int rows_on_device, size_t nx, const fereg_glm_spec* spec,
                          fereg_glm_out* out) {
    return session_glm(s, rows, rows_on_device, nx, spec, out, FEREG_FAMILY_POISSON);
}

int fereg_session_set_profiling(fereg_session* s, int on) {
    return guard([&] {
        if (!s) throw Error(RC_INVALID_INPUT, "fereg_session_set_profiling: NULL handle");
        s->s.set_profiling(on != 0);
    });
}

int fereg_session_phase_times(const fereg_session* s, double* ms, uint64_t* counts) {
    return guard([&] {
        if (!s) throw Error(RC_INVALID_INPUT, "fereg_session_phase_times: NULL handle");
        s->s.phase_times(ms, counts);
    });
}

uint64_t fereg_session_launches(const fereg_session* s) { return s ? s->s.launches() : 0; }

void* fereg_session_stream(const fereg_session* s) {
    return s ? static_cast<void*>(const_cast<fereg_session*>(s)->s.absorber().stream()) : nullptr;
}

}  // extern "C"

struct fereg_server {
    fereg::Server s;
    fereg_server(int w, uint64_t b, bool dry) : s(w, b, dry) {}
};

int fereg_server_create(const fereg_server_config* cfg, fereg_server** out) {
    return guard([&] {
        if (!cfg || !out) throw Error(RC_INVALID_INPUT, "fereg_server_create: NULL argument");
        *out = new fereg_server(cfg->workers, cfg->hbm_budget, cfg->dry_run != 0);
    });
}

int fereg_server_submit(fereg_server* srv, const fereg_request* q, uint64_t* ticket) {
    return guard([&] {
        if (!srv || !q || !ticket) throw Error(RC_INVALID_INPUT, "fereg_server_submit: NULL argument");
        if (q->nterms < 0 || q->ncl < 0) throw Error(RC_INVALID_INPUT, "fereg_server_submit: negative count");
        if (q->nterms && (!q->codes || !q->g)) throw Error(RC_INVALID_INPUT, "fereg_server_submit: NULL codes");
        if (q->ncl && (!q->cl_codes || !q->cl_g)) throw Error(RC_INVALID_INPUT, "fereg_server_submit: NULL clusters");
        if (!q->cols) throw Error(RC_INVALID_INPUT, "fereg_server_submit: NULL columns");
        ServeRequest r;
        r.model = q->model;
        r.codes.assign(q->codes, q->codes + q->nterms);
        r.g.assign(q->g, q->g + q->nterms);
        r.cl_codes.assign(q->cl_codes, q->cl_codes + q->ncl);
        r.cl_g.assign(q->cl_g, q->cl_g + q->ncl);
        r.w = q->w;
        r.weight_kind = q->weight_kind;
        r.n = q->n;
        r.nx = q->nx;
        r.ne = q->nendog;
        r.ni = q->ninst;
        r.cols.assign(q->cols, q->cols + 1 + q->nx + q->nendog + q->ninst);
        r.vce = q->vce;
        r.tol = q->tol;
        r.maxiter = q->maxiter;
        r.precision = q->precision;
        r.b = q->b;
        r.V = q->V;
        r.dry_run_us = q->dry_run_us;
        *ticket = srv->s.submit(r);
    });
}

int fereg_server_wait(fereg_server* srv, uint64_t ticket, fereg_request_result* out, char* msg, size_t msg_cap) {
    return guard([&] {
        if (!srv || !out) throw Error(RC_INVALID_INPUT, "fereg_server_wait: NULL argument");
        const ServeResult r = srv->s.wait(ticket);
        out->rc = r.rc;
        out->submit_s = r.submit_s;
        out->admit_s = r.admit_s;
        out->done_s = r.done_s;
        out->bytes = r.bytes;
        out->N = r.N;
        out->iterations = r.iterations;
        out->converged = r.converged ? 1 : 0;
        out->launches = r.launches;
        out->prep_s = r.prep_s;
        if (msg && msg_cap) {
            const size_t k = std::min(msg_cap - 1, r.msg.size());
            std::copy(r.msg.begin(), r.msg.begin() + k, msg);
            msg[k] = 0;
        }
    });
}

int fereg_server_stats(const fereg_server* srv, uint64_t* out8) {
    return guard([&] {
        if (!srv || !out8) throw Error(RC_INVALID_INPUT, "fereg_server_stats: NULL argument");
        srv->s.stats(out8);
    });
}

void fereg_server_destroy(fereg_server* srv) { delete srv; }

int fereg_factorize(const double* x, size_t n, uint32_t* codes, uint32_t* nlevels) {
    return guard([&] {
        if ((n && (!x || !codes)) || !nlevels) throw Error(RC_INVALID_INPUT, "fereg_factorize: NULL argument");
        if (n > size_t(0xffffffffu)) throw Error(RC_INVALID_INPUT, "fereg_factorize: more than 2^32 - 1 rows");
        *nlevels = prep_factorize(x, n, codes);
    });
}

int fereg_combine(const uint32_t* const* parts, const uint32_t* nl, int np, size_t n, uint32_t* codes,
                  uint32_t* nlevels) {
    return guard([&] {
        if (!parts || !nl || np < 1 || (n && !codes) || !nlevels)
            throw Error(RC_INVALID_INPUT, "fereg_combine: NULL argument or no part");
        std::vector<const u32*> p(parts, parts + np);
        std::vector<u32> g(nl, nl + np);
        *nlevels = prep_combine(p, g, n, codes);
    });
}

int fereg_drop_singletons(const uint32_t* const* codes, const uint32_t* g, int nterms, size_t n, const double* fw,
                          const double* y, int family, int singletons, uint8_t* alive, uint64_t* dropped_singletons,
                          uint64_t* dropped_separated) {
    return guard([&] {
        if (nterms < 0 || (nterms && (!codes || !g)) || (n && !alive))
            throw Error(RC_INVALID_INPUT, "fereg_drop_singletons: NULL argument");
        if (family < 0 || family > 2 || (family && !y))
            throw Error(RC_INVALID_INPUT, "fereg_drop_singletons: family 1 / 2 needs the outcome");
        std::vector<const u32*> c(codes, codes + nterms);
        std::vector<u32> gg(g, g + nterms);
        const DropCounts d = prep_drop(c, gg, n, fw, y, family, singletons != 0, alive);
        if (dropped_singletons) *dropped_singletons = d.singletons;
        if (dropped_separated) *dropped_separated = d.separated;
    });
}

int fereg_restrict(const uint32_t* codes, uint32_t g, const uint8_t* alive, size_t n, uint32_t* out,
                   uint32_t* nlevels, uint64_t* kept) {
    return guard([&] {
        if ((n && (!codes || !alive || !out)) || !nlevels) throw Error(RC_INVALID_INPUT, "fereg_restrict: NULL argument");
        size_t k = 0;
        *nlevels = prep_restrict(codes, g, alive, n, out, &k);
        if (kept) *kept = k;
    });
}

int fereg_structure_digest(const uint32_t* const* codes, const uint32_t* g, int nterms, size_t n, uint64_t* out) {
    return guard([&] {
        if (!codes || !g || nterms < 1 || !out) throw Error(RC_INVALID_INPUT, "fereg_structure_digest: NULL argument");
        std::vector<const u32*> c(codes, codes + nterms);
        std::vector<u32> gg(g, g + nterms);
        const HostStructure hs = build_structure(c, gg, n, SMALL_LIMIT);
        const PullTable pt = build_pull_table(hs);
        u64 h = 1469598103934665603ull;  // FNV-1a over the 32-bit words, array by array
        auto mix = [&](const std::vector<u32>& v) {
            for (u32 x : v) {
                h ^= x;
                h *= 1099511628211ull;
            }
            h ^= v.size();
            h *= 1099511628211ull;
        };
        for (const auto* v : {&hs.pi, &hs.seg_off, &hs.cell_row, &hs.coord, &pt.off, &pt.cell, &pt.seg, &pt.other})
            mix(*v);
        out[0] = hs.ncells;
        out[1] = hs.g1;
        out[2] = hs.m;
        out[3] = hs.m_small;
        out[4] = hs.nb();
        out[5] = u64(int64_t(hs.fe1));
        out[6] = h;
    });
}

int fereg_structure_compare(const uint32_t* const* codes, const uint32_t* g, int nterms, size_t n, uint64_t* out) {
    return guard([&] {
        if (!codes || !g || nterms < 1 || !out) throw Error(RC_INVALID_INPUT, "fereg_structure_compare: NULL argument");
        std::vector<const u32*> c(codes, codes + nterms);
        std::vector<u32> gg(g, g + nterms);
        const HostStructure hs = build_structure(c, gg, n, SMALL_LIMIT);
        const PullTable pt = build_pull_table(hs);
        cudaStream_t st = nullptr;
        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        struct StreamGuard {
            cudaStream_t s;
            ~StreamGuard() { cudaStreamDestroy(s); }
        } sg{st};
        AllocScope alloc_scope(st);
        std::vector<DBuf<u32>> dc(static_cast<size_t>(nterms));
        std::vector<const u32*> dptr;
        for (int q = 0; q < nterms; q++) {
            dc[size_t(q)].upload(c[size_t(q)], n, st);
            dptr.push_back(dc[size_t(q)].p);
        }
        HostStructure dh = plan_structure(c, gg, n, SMALL_LIMIT);
        DeviceStructure ds;
        std::vector<u32> poff, pseg;
        build_structure_device(dptr, gg, dh, ds, poff, pseg, st);
        auto fetch = [&](const DBuf<u32>& b, size_t count) {
            std::vector<u32> h(count);
            if (count) CK(cudaMemcpyAsync(h.data(), b.p, count * 4, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            return h;
        };
        auto diff = [](const std::vector<u32>& a, const std::vector<u32>& b) {
            if (a.size() != b.size()) return u64(1) << 40;
            u64 k = 0;
            for (size_t i = 0; i < a.size(); i++) k += a[i] != b[i];
            return k;
        };
        const size_t M = dh.ncells, E = M * dh.nb();
        out[0] = (dh.ncells != hs.ncells) + (dh.fe1 != hs.fe1) + (dh.m != hs.m) + (dh.m_small != hs.m_small) +
                 (dh.small_work != hs.small_work) + (dh.g1 != hs.g1) + (dh.nb() != hs.nb());
        for (size_t b = 0; b < std::min(dh.nb(), hs.nb()); b++)
            out[0] += dh.blocks[b].small != hs.blocks[b].small || dh.blocks[b].off != hs.blocks[b].off;
        out[1] = diff(dh.pi, hs.pi);
        out[2] = diff(dh.seg_off, hs.seg_off);
        out[3] = diff(dh.cell_row, hs.cell_row);
        out[4] = diff(fetch(ds.coord, dh.nb() * M), hs.coord);
        out[5] = diff(poff, pt.off);
        out[6] = diff(fetch(ds.pl_cell, E), pt.cell);
        out[7] = diff(pseg, pt.seg);
        out[8] = diff(fetch(ds.pl_other, E * (dh.nb() > 0 ? dh.nb() - 1 : 0)), pt.other);
    });
}

int fereg_amg_probe(const uint32_t* const* codes, const uint32_t* g, int nterms, size_t n, int max_levels,
                    uint32_t* levels, uint32_t* sizes, uint64_t* nnz, double* row_sum) {
    return guard([&] {
        if (!codes || !g || nterms < 1 || !levels) throw Error(RC_INVALID_INPUT, "fereg_amg_probe: NULL argument");
        std::vector<const u32*> c(codes, codes + nterms);
        std::vector<u32> gg(g, g + nterms);
        const HostStructure hs = build_structure(c, gg, n, SMALL_LIMIT);
        // unweighted weight state (operator.rs:211-338): n1, nr, diag, redundant
        const size_t M = hs.ncells, m = hs.m, nb = hs.nb();
        std::vector<double> cw(M), n1(hs.g1, 0.0), nr(m, 0.0), dq(m, 0.0), cs(m, 0.0), diag(m);
        std::vector<uint8_t> red(m);
        for (size_t k = 0; k < M; k++) cw[k] = hs.trivial() ? 1.0 : double(hs.cell_row[k + 1] - hs.cell_row[k]);
        for (u32 s = 0; s < hs.g1; s++) {
            for (u32 k = hs.seg_off[s]; k < hs.seg_off[s + 1]; k++) n1[s] += cw[k];
            for (u32 k = hs.seg_off[s]; k < hs.seg_off[s + 1]; k++)
                for (size_t b = 0; b < nb; b++) cs[hs.coord[b * M + k]] += cw[k];
            for (u32 k = hs.seg_off[s]; k < hs.seg_off[s + 1]; k++)
                for (size_t b = 0; b < nb; b++) {
                    const u32 q = hs.coord[b * M + k];
                    nr[q] += cw[k];
                    dq[q] += cw[k] * cs[q] / n1[s];
                }
            for (u32 k = hs.seg_off[s]; k < hs.seg_off[s + 1]; k++)
                for (size_t b = 0; b < nb; b++) cs[hs.coord[b * M + k]] = 0.0;
        }
        for (size_t q = 0; q < m; q++) {
            diag[q] = nr[q] - dq[q];
            red[q] = diag[q] <= 1e-12 * nr[q];
        }
        *levels = 0;
        for (size_t b = 0; b < nb; b++) {
            if (hs.blocks[b].g <= 2 * AMG_COARSE) continue;
            const AmgHierarchy H = amg_build(hs, b, cw.data(), n1.data(), diag.data(), red.data());
            *levels = u32(H.levels.size());
            for (size_t l = 0; l < H.levels.size() && int(l) < max_levels; l++) {
                const Csr& A = H.levels[l].A;
                if (sizes) sizes[l] = H.levels[l].n;
                if (nnz) nnz[l] = A.col.size();
                double worst = 0.0, dmax = 0.0;
                for (u32 i = 0; i < A.nr; i++) {
                    double rs = 0.0;
                    for (u32 e = A.ptr[i]; e < A.ptr[i + 1]; e++) {
                        rs += A.val[e];
                        if (A.col[e] == i) dmax = std::max(dmax, A.val[e]);
                    }
                    worst = std::max(worst, std::fabs(rs));
                }
                if (row_sum) row_sum[l] = dmax > 0.0 ? worst / dmax : 0.0;
            }
            break;
        }
    });
}
