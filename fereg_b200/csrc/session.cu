// GpuSession: Session::ols (ols.rs:199-470) on the B200 absorber.
//
// Per call: column statistics of the raw rows (two device passes, stats.rs:40), the FE solve in
// place (the absorber), the weighted Gram of the residualized block (one device pass,
// stats.rs:195), collinearity and the coefficients by sweeps on the standardized Gram (host,
// K x K), the residuals and their sum of squares (device), and the variance: iid from the
// residual sum of squares, HC1 from a device meat pass, CRV1 from per-cluster score sums (device,
// rows grouped by a stable cluster permutation) and S^T S, with the inclusion-exclusion of
// multiway clusters and the eigenvalue clip (vcov.rs:480-720). Degrees of freedom
// (dof.rs:64-180) use device union-find for the mobility groups of FE pairs.

#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>
#include <sstream>

#include "linalg.h"
#include "session.h"
#include "slopes.h"
#include "boot.cuh"
#include "glm.cuh"
#include "relu.cuh"
#include "crv3.cuh"
#include "session_dev.h"
#include "stats.cuh"

namespace fereg {

namespace {

constexpr double SWEEP_TOL = 1e-13;     // vcov.rs invsym tolerance
constexpr double F_SWEEP_TOL = 1e-9;    // ols.rs Wald F: greedy sweep of the slope variance
constexpr int MAX_TABLE = 64;           // dof table slots reported

double nanv() { return std::numeric_limits<double>::quiet_NaN(); }
double finite_or_nan(double x) { return std::isfinite(x) ? x : nanv(); }

int blocks_for(size_t n, int tb) { return int(std::max<size_t>(1, std::min<size_t>((n + tb - 1) / tb, 148 * 16))); }

// Interaction codes of several dimensions (factor.rs:255 combine): the tuple key in mixed radix
// (first dimension most significant), distinct keys numbered in ascending order.
void combine_codes(const std::vector<const std::vector<u32>*>& dims, const std::vector<u32>& gs, size_t n,
                   std::vector<u32>& out, u32& g) {
    if (dims.size() == 1) {
        out = *dims[0];
        g = gs[0];
        return;
    }
    std::vector<u64> key(n, 0);
    for (size_t d = 0; d < dims.size(); d++)
        for (size_t i = 0; i < n; i++) key[i] = key[i] * u64(gs[d]) + (*dims[d])[i];
    std::vector<u64> uniq(key);
    std::sort(uniq.begin(), uniq.end());
    uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
    out.resize(n);
    for (size_t i = 0; i < n; i++) out[i] = u32(std::lower_bound(uniq.begin(), uniq.end(), key[i]) - uniq.begin());
    g = u32(uniq.size());
}

}  // namespace

namespace {

// dof.rs:255-272 redundant_slope_levels: the variable scaled by its standard deviation
// (stats.rs:187 stdev, at least 1e-3); a level is redundant when max - min <= 1e-6 (term with
// intercept) or |min| + |max| <= 1e-6 (term without).
u64 redundant_slope_levels(const u32* codes, u32 g, const double* x, size_t n, bool intercept) {
    double mean = 0.0;
    for (size_t i = 0; i < n; i++) mean += x[i];
    mean /= double(n);
    double m2 = 0.0;
    for (size_t i = 0; i < n; i++) m2 += (x[i] - mean) * (x[i] - mean);
    const double sd = std::max(std::sqrt(m2 / (double(n) - 1.0)), 1e-3);
    std::vector<double> lo(g, INFINITY), hi(g, -INFINITY);
    for (size_t i = 0; i < n; i++) {
        const double v = x[i] / sd;
        lo[codes[i]] = std::min(lo[codes[i]], v);
        hi[codes[i]] = std::max(hi[codes[i]], v);
    }
    u64 cnt = 0;
    for (u32 l = 0; l < g; l++)
        cnt += intercept ? (hi[l] - lo[l] <= 1e-6) : (std::fabs(lo[l]) + std::fabs(hi[l]) <= 1e-6);
    return cnt;
}

}  // namespace

GpuSession::GpuSession(const std::vector<const u32*>& codes, const std::vector<u32>& g,
                       const std::vector<const u32*>& cl_codes, const std::vector<u32>& cl_g, const double* w,
                       int weight_kind, size_t n, u64 num_singletons, const Ctx& ctx,
                       const std::vector<TermShape>* shapes)
    : n_(n), kind_(w ? weight_kind : 0), nsing_(num_singletons) {
    if (shapes && shapes->size() != codes.size()) throw Error(RC_INVALID_INPUT, "fereg_session_create: term shapes");
    if (weight_kind < 0 || weight_kind > 3) throw Error(RC_INVALID_INPUT, "fereg_session_create: bad weight kind");
    if (w && weight_kind == 0) throw Error(RC_INVALID_INPUT, "fereg_session_create: weights need a weight kind");
    std::vector<const u32*> tptr = codes;
    std::vector<u32> tg = g;
    std::vector<u32> constant;
    if (tptr.empty()) {  // noabsorb: the constant is the only absorbed term (ols.rs:263, dof.rs:64)
        constant.assign(n, 0u);
        tptr.push_back(constant.data());
        tg.push_back(1u);
    }
    tg_ = tg;
    cg_ = cl_g;
    for (size_t q = 0; q < tptr.size(); q++) tcodes_.emplace_back(tptr[q], tptr[q] + n);
    for (size_t c = 0; c < cl_codes.size(); c++) ccodes_.emplace_back(cl_codes[c], cl_codes[c] + n);
    if (w) {
        wk_.assign(w, w + n);
        sumw_ = 0.0;
        for (double x : wk_) sumw_ += x;
    } else {
        sumw_ = double(n);
    }
    // the term codes on the device: the session's copies, from which the absorber also builds its
    // cell structure
    d_ = std::make_unique<SessionDev>();
    SessionDev& d = *d_;
    std::vector<const u32*> dcodes;
    for (auto& c : tcodes_) {
        d.tcodes.emplace_back();
        d.tcodes.back().upload(c, nullptr);
        dcodes.push_back(d.tcodes.back().p);
    }
    CK(cudaStreamSynchronize(nullptr));
    bool slopes = false;
    for (size_t q = 0; q < tptr.size(); q++) {
        const bool icpt = shapes ? (*shapes)[q].intercept : true;
        t_icpt_.push_back(icpt);
        slope_red_.emplace_back();
        if (shapes)
            for (const double* x : (*shapes)[q].slopes) {
                if (!x) throw Error(RC_INVALID_INPUT, "fereg_session_create: missing slope variable");
                slope_red_.back().push_back(redundant_slope_levels(tptr[q], tg[q], x, n, icpt));
            }
        slopes |= !icpt || !slope_red_.back().empty();
    }
    if (slopes) {
        std::vector<SlopeTermIn> st(tptr.size());
        for (size_t q = 0; q < tptr.size(); q++) {
            st[q].codes = tptr[q];
            st[q].g = tg[q];
            st[q].intercept = t_icpt_[q];
            st[q].slopes = (*shapes)[q].slopes;
        }
        ab_ = std::make_unique<GpuSlopeSolver>(st, w, n, ctx);
    } else {
        ab_ = std::make_unique<GpuAbsorber>(tptr, tg, w, n, ctx, &dcodes);
    }
    d.st = ab_->stream();
    AllocScope alloc_scope(d.st);
    for (auto& c : ccodes_) {
        d.ccodes.emplace_back();
        d.ccodes.back().upload(c, d.st);
    }
    const std::vector<u32>& pi = ab_->row_order();
    if (w) {
        std::vector<double> raw(n), wv(n);
        for (size_t i = 0; i < n; i++) raw[i] = wk_[pi[i]];
        // ols.rs:77-108 Weights: aweights and pweights normalized to sum n, fweights as given
        const double f = (kind_ == 1 || kind_ == 3) ? double(n) / sumw_ : 1.0;
        for (size_t i = 0; i < n; i++) wv[i] = raw[i] * f;
        d.w_raw.upload(raw, d.st);
        d.wv.upload(wv, d.st);
    }
    // cluster subsets (inclusion-exclusion of vcov.rs:480-560): every non-empty subset of the
    // dimensions, its rows grouped by the combined code
    const size_t q = ccodes_.size();
    for (u32 mask = 1; mask < (1u << q); mask++) {
        std::vector<const std::vector<u32>*> dims;
        std::vector<u32> gs;
        for (size_t c = 0; c < q; c++)
            if (mask & (1u << c)) {
                dims.push_back(&ccodes_[c]);
                gs.push_back(cg_[c]);
            }
        std::vector<u32> kc;
        u32 G = 0;
        combine_codes(dims, gs, n, kc, G);
        std::vector<u32> coff(size_t(G) + 1, 0);
        for (size_t i = 0; i < n; i++) coff[kc[pi[i]] + 1]++;
        for (u32 k = 0; k < G; k++) coff[k + 1] += coff[k];
        std::vector<int> perm(n);
        std::vector<u32> pos(coff.begin(), coff.end() - 1);
        for (size_t i = 0; i < n; i++) perm[pos[kc[pi[i]]]++] = int(i);
        d.subsets.emplace_back();
        auto& s = d.subsets.back();
        s.perm.upload(perm, d.st);
        s.coff.upload(coff, d.st);
        s.G = G;
        s.sign = dims.size() % 2 == 1 ? 1.0 : -1.0;
        s.kc = std::move(kc);
    }
    CK(cudaStreamSynchronize(d.st));
}

GpuSession::~GpuSession() {
    d_.reset();
    ab_.reset();
}

u64 GpuSession::launches() const { return d_->launches + ab_->launches(); }

void GpuSession::set_profiling(bool on) {
    AllocScope alloc_scope(ab_->stream());
    d_->prof = on;
    if (on) {
        std::fill(d_->ms, d_->ms + S_NSLOTS, 0.0);
        std::fill(d_->cnt, d_->cnt + S_NSLOTS, u64(0));
    }
    ab_->set_profiling(on);
}

void GpuSession::phase_times(double* ms, u64* counts) const {
    ab_->phase_times(ms, counts);
    for (int i = 0; i < S_NSLOTS; i++) {
        if (ms) ms[GpuAbsorber::P_NSLOTS + i] = d_->ms[i];
        if (counts) counts[GpuAbsorber::P_NSLOTS + i] = d_->cnt[i];
    }
}

// dof.rs:222-256 mobility_groups of terms qa, qb on the device; save: keep the row labels.
// Runs on the dof pass's stream with its buffers.
u64 GpuSession::mobility_groups(size_t qa, size_t qb, bool save, DofScratch& s) {
    SessionDev& d = *d_;
    const cudaStream_t st = s.st.s;
    const u32 ga = tg_[qa], gb = tg_[qb], nv = ga + gb;
    s.uf.alloc(nv);
    s.flags.alloc(ga);
    s.scan.alloc(ga);
    s.bsum.alloc((ga + SCAN_TILE - 1) / SCAN_TILE + 1);
    s.total.alloc(1);
    s.err.alloc(1);
    CK(cudaMemsetAsync(s.err.p, 0, sizeof(int), st));
    k_uf_init<<<blocks_for(nv, 256), 256, 0, st>>>(s.uf.p, nv);
    k_uf_union<<<blocks_for(n_, 256), 256, 0, st>>>(d.tcodes[qa].p, d.tcodes[qb].p, ga, n_, s.uf.p, s.err.p);
    k_uf_flatten<<<blocks_for(nv, 256), 256, 0, st>>>(s.uf.p, nv);
    k_uf_roots<<<blocks_for(ga, 256), 256, 0, st>>>(s.uf.p, ga, s.flags.p);
    const u32 nblk = (ga + SCAN_TILE - 1) / SCAN_TILE;
    k_scan_sums<<<nblk, SCAN_TB, 0, st>>>(s.flags.p, ga, s.bsum.p);
    k_scan_top<<<1, SCAN_TB, 0, st>>>(s.bsum.p, nblk, s.total.p);
    k_scan_apply<<<nblk, SCAN_TB, 0, st>>>(s.flags.p, ga, s.bsum.p, s.scan.p);
    s.launches += 7;
    if (save) {
        s.gv.alloc(n_);
        k_uf_label<<<blocks_for(n_, 256), 256, 0, st>>>(d.tcodes[qa].p, n_, s.uf.p, s.scan.p, s.gv.p);
        s.launches++;
    }
    u32 total = 0;
    int err = 0;
    CK(cudaMemcpyAsync(&total, s.total.p, sizeof(u32), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&err, s.err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (err) throw Error(RC_INTERNAL, "fereg: union-find did not settle");
    return total;
}

// dof.rs:184 nested_within: every level of term q lies in one level of cluster dimension c.
bool GpuSession::nested_within(size_t q, size_t c, DofScratch& s) {
    SessionDev& d = *d_;
    const cudaStream_t st = s.st.s;
    s.map.alloc(tg_[q]);
    s.err.alloc(1);
    CK(cudaMemsetAsync(s.map.p, 0xff, size_t(tg_[q]) * sizeof(u32), st));
    CK(cudaMemsetAsync(s.err.p, 0, sizeof(int), st));
    k_nested<<<blocks_for(n_, 256), 256, 0, st>>>(d.tcodes[q].p, d.ccodes[c].p, n_, s.map.p, s.err.p);
    s.launches++;
    int flag = 0;
    CK(cudaMemcpyAsync(&flag, s.err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return flag == 0;
}

// Starts the dof pass (dof.rs:64-180 does not depend on the data columns) on a host thread of
// its own and its own stream, one priority step below the session's, so that its union-finds
// overlap the column statistics and the FE solve the caller issues on the session's stream;
// dof_end joins it. The pass waits for the work already on the session's stream (the uploaded
// codes).
std::future<GpuSession::Dof> GpuSession::dof_begin(bool clusters, bool firstpair, bool want_groupvar) {
    SessionDev& d = *d_;
    DofScratch& s = d.dof;
    if (!s.st.s) {  // one priority step below the session's stream
        int least = 0, greatest = 0, own = 0;
        CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        CK(cudaStreamGetPriority(d.st, &own));
        CK(cudaStreamCreateWithPriority(&s.st.s, cudaStreamNonBlocking, std::min(least, own + 1)));
        CK(cudaEventCreateWithFlags(&s.ready, cudaEventDisableTiming));
    }
    CK(cudaEventRecord(s.ready, d.st));
    CK(cudaStreamWaitEvent(s.st.s, s.ready, 0));
    int dev = 0;
    CK(cudaGetDevice(&dev));
    for (cudaEvent_t* e : {&s.ta, &s.tb})  // left by a call that threw before joining its pass
        if (*e) {
            d.pool.push_back(*e);
            *e = nullptr;
        }
    cudaEvent_t ta = nullptr, tb = nullptr;
    if (d.prof) {
        ta = d.event();
        tb = d.event();
    }
    s.ta = ta;
    s.tb = tb;
    return std::async(std::launch::async, [this, &s, dev, ta, tb, clusters, firstpair, want_groupvar]() {
        CK(cudaSetDevice(dev));
        AllocScope scope(s.st.s);
        if (ta) CK(cudaEventRecord(ta, s.st.s));
        Dof dof = dof_pass(clusters, firstpair, want_groupvar, s);
        if (tb) CK(cudaEventRecord(tb, s.st.s));
        return dof;
    });
}

GpuSession::Dof GpuSession::dof_end(std::future<Dof>& job) {
    SessionDev& d = *d_;
    DofScratch& s = d.dof;
    const cudaEvent_t ta = s.ta, tb = s.tb;
    s.ta = s.tb = nullptr;
    Dof dof;
    try {
        dof = job.get();
    } catch (...) {
        if (ta) d.pool.push_back(ta);
        if (tb) d.pool.push_back(tb);
        throw;
    }
    if (ta) d.open.push_back(SessionDev::Open{S_DOF, ta, tb});
    d.launches += s.launches;
    s.launches = 0;
    return dof;
}

GpuSession::Dof GpuSession::estimate_dof(bool clusters, bool firstpair, bool want_groupvar) {
    std::future<Dof> job = dof_begin(clusters, firstpair, want_groupvar);
    return dof_end(job);
}

// dof.rs:64-180 estimate_dof (the default options: clusters, pairwise and continuous; firstpair
// instead of clusters and pairwise). Slots: per term its intercept (when it has one), then one
// per slope; slot i: k levels, m redundant, exact, nested in a cluster.
GpuSession::Dof GpuSession::dof_pass(bool clusters, bool firstpair, bool want_groupvar, DofScratch& s) {
    Dof dof;
    const size_t nt = tg_.size();
    std::vector<int> icpt_term;  // per slot: the term of an intercept slot, -1 for a slope slot
    std::vector<size_t> first_slope(nt, SIZE_MAX);
    for (size_t q = 0; q < nt; q++) {
        if (t_icpt_[q]) {
            dof.slots.push_back(DofSlot{tg_[q], 0, false, false});
            icpt_term.push_back(int(q));
        }
        if (!slope_red_[q].empty()) first_slope[q] = dof.slots.size();
        for (size_t k = 0; k < slope_red_[q].size(); k++) {
            dof.slots.push_back(DofSlot{tg_[q], 0, false, false});
            icpt_term.push_back(-1);
        }
    }
    const size_t ns = dof.slots.size();
    std::vector<bool> live(ns);
    for (size_t i = 0; i < ns; i++) live[i] = icpt_term[i] >= 0;
    if (clusters && !firstpair)
        for (size_t c = 0; c < ccodes_.size(); c++) {
            if (std::none_of(live.begin(), live.end(), [](bool x) { return x; })) break;
            for (size_t i = 0; i < ns; i++) {
                if (!live[i] || dof.slots[i].exact) continue;
                if (nested_within(size_t(icpt_term[i]), c, s)) {
                    dof.slots[i].m = dof.slots[i].k;
                    dof.slots[i].exact = dof.slots[i].nested = true;
                    dof.df_a_nested += dof.slots[i].k;
                    live[i] = false;
                }
            }
        }
    const size_t remaining = size_t(std::count(live.begin(), live.end(), true));
    if (remaining > 1 || (remaining > 0 && dof.df_a_nested > 0)) {
        // each live intercept but the first keeps one redundant level (the constant), unless a
        // term nested in a cluster already carries it
        bool skip = dof.df_a_nested == 0;
        for (size_t i = 0; i < ns; i++) {
            if (!live[i]) continue;
            if (skip) {
                skip = false;
                continue;
            }
            dof.slots[i].m = 1;
        }
    }
    for (size_t i = 0; i < ns; i++)
        if (live[i]) {
            dof.slots[i].exact = true;
            break;
        }
    std::vector<size_t> idx;
    for (size_t i = 0; i < ns; i++)
        if (live[i]) idx.push_back(i);
    int pairs = 0;
    for (size_t a = 0; a < idx.size(); a++) {
        bool stop = false;
        for (size_t b = a + 1; b < idx.size(); b++) {
            pairs++;
            const bool save = pairs == 1 && want_groupvar;
            const u64 m = mobility_groups(size_t(icpt_term[idx[a]]), size_t(icpt_term[idx[b]]), save, s);
            if (save) dof.has_groupvar = true;
            dof.slots[idx[b]].m = std::max(dof.slots[idx[b]].m, m);
            if (pairs == 1) dof.slots[idx[b]].exact = true;
            if (firstpair) {
                stop = true;
                break;
            }
        }
        if (stop) break;
    }
    // slopes constant (term with intercept) or zero (term without) within a level
    for (size_t q = 0; q < nt; q++)
        for (size_t k = 0; k < slope_red_[q].size(); k++)
            if (slope_red_[q][k] > 0) dof.slots[first_slope[q] + k].m = slope_red_[q][k];
    for (auto& sl : dof.slots) {
        dof.df_a_initial += sl.k;
        dof.df_a_redundant += sl.m;
    }
    dof.df_a = dof.df_a_initial - dof.df_a_redundant;
    return dof;
}

// Outer products sum om_i a_i a_i^T over `nrows` rows of the srcR-column block src:
// a_i = [x_i[cols] + shift, 1 (cst)]; optionally the plain sums of squares of the columns.
// Returns the full msz x msz matrix (device passes, host copy of the result).
std::vector<double> GpuSession::outer_products(const double* src, size_t nrows, int srcR, const std::vector<int>& cols,
                                               const std::vector<double>* shift, bool cst, const double* om,
                                               const int* perm, bool ssq, std::vector<double>* ss_out) {
    SessionDev& d = *d_;
    cudaStream_t st = d.st;
    const int k = int(cols.size()), msz = k + (cst ? 1 : 0);
    const int P = msz * (msz + 1) / 2;
    std::vector<double> m(size_t(msz) * msz, 0.0);
    if (msz == 0) return m;
    d.col.alloc(size_t(k) + 1);
    CK(cudaMemcpyAsync(d.col.p, cols.data(), size_t(k) * sizeof(int), cudaMemcpyHostToDevice, st));
    if (shift) {
        d.shift.alloc(size_t(k) + 1);
        CK(cudaMemcpyAsync(d.shift.p, shift->data(), size_t(k) * 8, cudaMemcpyHostToDevice, st));
    }
    std::vector<double> pairs(P), sq(k);
    if (msz <= 32) {
        const int len = msz * msz + (ssq ? k : 0);
        d.part.alloc(size_t(ST_GRID) * len);
        d.sums.alloc(size_t(len));
        OpSpec sp{src, nrows, srcR, d.col.p, shift ? d.shift.p : nullptr, k, cst ? 1 : 0, msz, om, perm, 0, 0,
                  ssq ? 1 : 0};
        // a contiguous block on a 16-byte boundary streams through shared memory by bulk copies
        const bool bulk = !perm && srcR <= 32 && reinterpret_cast<uintptr_t>(src) % 16 == 0 &&
                          nrows >= size_t(CS_ROWS) * ST_GRID;
        d.err.alloc(1);
        int parts = ST_GRID;
        if (bulk) {
            CK(cudaMemsetAsync(d.err.p, 0, sizeof(int), st));
            const size_t shm = size_t(CS_STAGES) * CS_ROWS * size_t(srcR) * sizeof(double);
            auto run = [&](auto kernel) {
                if (shm > size_t(smem_limit(kernel)))  // static + dynamic can pass 48 KB: always raise it
                    throw Error(RC_INTERNAL, "fereg: the outer-product ring does not fit shared memory");
                // one wave: the CTAs resident at once (registers or the ring bound them), so that no
                // second, partial wave runs the last chunks at a fraction of the occupancy
                parts = std::max(1, std::min(ST_GRID, 148 * resident_ctas(kernel, ST_TB, shm)));
                kernel<<<parts, ST_TB, shm, st>>>(sp, d.part.p, d.err.p);
            };
            switch ((msz + 7) / 8) {
                case 1: run(k_outer_mma_bulk<1>); break;
                case 2: run(k_outer_mma_bulk<2>); break;
                case 3: run(k_outer_mma_bulk<3>); break;
                default: run(k_outer_mma_bulk<4>); break;
            }
        } else {
            switch ((msz + 7) / 8) {
                case 1: k_outer_mma<1><<<ST_GRID, ST_TB, 0, st>>>(sp, d.part.p); break;
                case 2: k_outer_mma<2><<<ST_GRID, ST_TB, 0, st>>>(sp, d.part.p); break;
                case 3: k_outer_mma<3><<<ST_GRID, ST_TB, 0, st>>>(sp, d.part.p); break;
                default: k_outer_mma<4><<<ST_GRID, ST_TB, 0, st>>>(sp, d.part.p); break;
            }
        }
        k_sum_parts<<<sum_parts_blocks(len), 256, 0, st>>>(d.part.p, parts, len, d.sums.p);
        d.launches += 2;
        std::vector<double> h(len);
        int late = 0;
        CK(cudaMemcpyAsync(h.data(), d.sums.p, size_t(len) * 8, cudaMemcpyDeviceToHost, st));
        if (bulk) CK(cudaMemcpyAsync(&late, d.err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (late) throw Error(RC_INTERNAL, "fereg: a bulk copy of the outer products did not complete");
        for (int a = 0; a < msz; a++)
            for (int b = a; b < msz; b++) m[size_t(a) * msz + b] = m[size_t(b) * msz + a] = h[size_t(a) * msz + b];
        if (ss_out) *ss_out = std::vector<double>(h.begin() + msz * msz, h.end());
        return m;
    }
    for (int p0 = 0; p0 < P; p0 += OP_MAXP) {
        const int np = std::min(OP_MAXP, P - p0);
        const bool with_sq = ssq && p0 == 0;
        const int len = np + (with_sq ? k : 0);
        d.part.alloc(size_t(ST_GRID) * len);
        d.sums.alloc(size_t(len));
        OpSpec s{src, nrows, srcR, d.col.p, shift ? d.shift.p : nullptr, k, cst ? 1 : 0, msz, om, perm, p0, np,
                 with_sq ? 1 : 0};
        k_outer<<<ST_GRID, ST_TB, 0, st>>>(s, d.part.p);
        k_sum_parts<<<sum_parts_blocks(len), 256, 0, st>>>(d.part.p, ST_GRID, len, d.sums.p);
        d.launches += 2;
        std::vector<double> h(len);
        CK(cudaMemcpyAsync(h.data(), d.sums.p, size_t(len) * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        std::copy(h.begin(), h.begin() + np, pairs.begin() + p0);
        if (with_sq) std::copy(h.begin() + np, h.end(), sq.begin());
    }
    int p = 0;
    for (int a = 0; a < msz; a++)
        for (int b = a; b < msz; b++, p++) m[size_t(a) * msz + b] = m[size_t(b) * msz + a] = pairs[p];
    if (ss_out) *ss_out = sq;
    return m;
    }

double* GpuSession::gather_columns(const double* const* cols, size_t R) {
    AllocScope alloc_scope(ab_->stream());
    SessionDev& d = *d_;
    cudaStream_t st = d.st;
    const size_t n = n_;
    if (R == 0 || R + 1 > size_t(OP_MAXM)) throw Error(RC_INVALID_INPUT, "fereg gather: 1 to 62 columns");
    for (size_t j = 0; j < R; j++)
        if (!cols[j]) throw Error(RC_INVALID_INPUT, "fereg gather: NULL column");
    if (!d.pi.p) d.pi.upload(ab_->row_order(), st);
    d.colbuf.alloc(n * R);
    for (size_t j = 0; j < R; j++)
        CK(cudaMemcpyAsync(d.colbuf.p + j * n, cols[j], n * 8, cudaMemcpyHostToDevice, st));
    d.rows.alloc(n * R);
    k_gather_cols<<<blocks_for(n, 256), 256, 0, st>>>(d.colbuf.p, d.pi.p, n, int(R), d.rows.p);
    d.launches++;
    CK(cudaGetLastError());
    return d.rows.p;
}

// Column statistics of the raw rows (stats.rs:40) in one device pass about each column's first
// value: sd (unweighted, floored at 1e-3), weighted mean, sum of squares, weighted centered and
// uncentered sums of squares. column_stats_alloc allocates the pass's buffers (on the session's
// stream); column_stats_launch issues it on stream cs, the 6 R sums, the first row and the bulk
// copies' error flag landing in host memory at s1, c0 and late once cs gets there.
void GpuSession::column_stats_alloc(int R) {
    SessionDev& d = *d_;
    d.part.alloc(size_t(ST_GRID) * size_t(R) * 6);
    d.sums.alloc(size_t(R) * 6);
    d.err.alloc(1);
}

void GpuSession::column_stats_launch(const double* rows, int R, cudaStream_t cs, double* s1, double* c0, int* late) {
    SessionDev& d = *d_;
    const size_t n = n_, r = size_t(R);
    const double* wr = wk_.empty() ? nullptr : d.w_raw.p;
    CK(cudaMemsetAsync(d.err.p, 0, sizeof(int), cs));
    // whole rows through shared memory by bulk copies when the block starts on a 16-byte boundary
    const bool bulk = R <= 32 && reinterpret_cast<uintptr_t>(rows) % 16 == 0 && n >= size_t(CS_ROWS) * ST_GRID;
    int parts = ST_GRID;
    if (bulk) {
        const size_t shm = size_t(CS_STAGES) * CS_ROWS * r * sizeof(double);
        auto run = [&](auto kernel) {
            if (shm > size_t(smem_limit(kernel)))  // static + dynamic can pass 48 KB: always raise it
                throw Error(RC_INTERNAL, "fereg: the column statistics ring does not fit shared memory");
            // one wave of resident CTAs (the ring and the reduction bound them)
            parts = std::max(1, std::min(ST_GRID, 148 * resident_ctas(kernel, ST_TB, shm)));
            kernel<<<parts, ST_TB, shm, cs>>>(rows, n, R, wr, d.part.p, d.err.p);
        };
        switch (rcp_of(R)) {
            case 1: run(k_colstats_bulk<1>); break;
            case 2: run(k_colstats_bulk<2>); break;
            case 4: run(k_colstats_bulk<4>); break;
            case 8: run(k_colstats_bulk<8>); break;
            case 16: run(k_colstats_bulk<16>); break;
            default: run(k_colstats_bulk<32>); break;
        }
        d.launches++;
    }
    for (int j0 = 0; j0 < R && !bulk; j0 += 32) {
        const int Rc = std::min(32, R - j0);
        switch (rcp_of(Rc)) {
            case 1: k_colstats1<1><<<ST_GRID, ST_TB, 0, cs>>>(rows, n, R, j0, Rc, wr, d.part.p); break;
            case 2: k_colstats1<2><<<ST_GRID, ST_TB, 0, cs>>>(rows, n, R, j0, Rc, wr, d.part.p); break;
            case 4: k_colstats1<4><<<ST_GRID, ST_TB, 0, cs>>>(rows, n, R, j0, Rc, wr, d.part.p); break;
            case 8: k_colstats1<8><<<ST_GRID, ST_TB, 0, cs>>>(rows, n, R, j0, Rc, wr, d.part.p); break;
            case 16: k_colstats1<16><<<ST_GRID, ST_TB, 0, cs>>>(rows, n, R, j0, Rc, wr, d.part.p); break;
            default: k_colstats1<32><<<ST_GRID, ST_TB, 0, cs>>>(rows, n, R, j0, Rc, wr, d.part.p); break;
        }
        d.launches++;
    }
    k_sum_parts<<<sum_parts_blocks(R * 6), 256, 0, cs>>>(d.part.p, parts, R * 6, d.sums.p);
    d.launches++;
    CK(cudaMemcpyAsync(s1, d.sums.p, r * 6 * 8, cudaMemcpyDeviceToHost, cs));
    CK(cudaMemcpyAsync(c0, rows, r * 8, cudaMemcpyDeviceToHost, cs));
    CK(cudaMemcpyAsync(late, d.err.p, sizeof(int), cudaMemcpyDeviceToHost, cs));
}

GpuSession::ColStats GpuSession::column_stats_finish(const double* s1, const double* c0, int late, int R) const {
    if (late) throw Error(RC_INTERNAL, "fereg: a bulk copy of the column statistics did not complete");
    const size_t n = n_, r = size_t(R);
    const double sumw = sumw_;
    ColStats cs;
    cs.wmean.resize(r);
    cs.sumsq.resize(r);
    cs.wss_unc.resize(r);
    cs.sd.resize(r);
    cs.wss.resize(r);
    for (size_t j = 0; j < r; j++) {
        const double* a = s1 + j * 6;
        const double m2 = std::max(0.0, a[1] - a[0] * a[0] / double(n));
        cs.sd[j] = std::max(std::sqrt(m2 / (double(n) - 1.0)), 1e-3);
        cs.wmean[j] = c0[j] + a[2] / sumw;
        cs.wss[j] = std::max(0.0, a[3] - a[2] * a[2] / sumw);
        cs.sumsq[j] = a[4];
        cs.wss_unc[j] = a[5];
    }
    return cs;
}

GpuSession::ColStats GpuSession::column_stats(const double* rows, int R) {
    SessionDev& d = *d_;
    const size_t r = size_t(R);
    column_stats_alloc(R);
    std::vector<double> s1(r * 6), c0(r);
    int late = 0;
    column_stats_launch(rows, R, d.st, s1.data(), c0.data(), &late);
    CK(cudaStreamSynchronize(d.st));
    return column_stats_finish(s1.data(), c0.data(), late, R);
}

void GpuSession::ols(double* rows_in, bool on_device, size_t nx, const OlsSpec& spec, OlsOut& out) {
    AllocScope alloc_scope(ab_->stream());
    restore_weights();
    SessionDev& d = *d_;
    cudaStream_t st = d.st;
    const size_t n = n_, r = 1 + nx;
    const int R = int(r);
    if (r + 1 > size_t(OP_MAXM)) throw Error(RC_INVALID_INPUT, "fereg ols: at most 62 regressors on the device path");
    double* rows = rows_in;
    if (!on_device) {
        d.rows.alloc(n * r);
        CK(cudaMemcpyAsync(d.rows.p, rows_in, n * r * 8, cudaMemcpyHostToDevice, st));
        rows = d.rows.p;
    }
    const std::vector<u32>& pi = ab_->row_order();
    const int kind = kind_;
    const bool weighted = !wk_.empty();
    const double sumw = sumw_;
    const double bigN = kind == 2 ? sumw : double(n);
    int vce = spec.vce;
    if (vce == 0 && kind == 3) vce = 1;  // ols.rs:150 pweights imply robust
    if (vce < 0 || vce > 5) throw Error(RC_INVALID_INPUT, "fereg ols: unknown variance");
    if (vce == 5 && kind == 3) throw Error(RC_INVALID_INPUT, "pweights not allowed with option vce(hc3)");  // ols.rs:251
    const bool clustered = vce == 2 || vce == 3;
    if (clustered && ccodes_.empty()) throw Error(RC_INVALID_INPUT, "fereg ols: cluster variance without clusters");
    if (vce == 3 && (kind == 2 || !dynamic_cast<GpuAbsorber*>(ab_.get())))
        throw Error(RC_INVALID_INPUT, "fereg ols: CRV3 needs intercept-only terms and no fweights");
    const bool has_intercept = true;  // intercept-only terms (or noabsorb) contain the constant
    const bool report_constant = has_intercept && !spec.noconstant;
    // CRV3 refits start from the raw rows (row order)
    std::vector<double> raw_h;
    if (vce == 3) {
        raw_h.resize(n * r);
        CK(cudaMemcpyAsync(raw_h.data(), rows, n * r * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }

    // the dof pass runs on its own stream beside the column statistics and the solve
    std::future<Dof> dof_job = dof_begin(clustered, spec.firstpair != 0, spec.want_groupvar != 0 && out.groupvar);

    // Pass A: column statistics of the raw rows (stats.rs:40), raw weights, in one device pass. On
    // the timed path it runs on the side stream beside the FE solve, which waits for it before it
    // writes the rows; the phase-timed calls run it in place on the session's stream.
    ColStatsSide& side = d.colstats_side();
    ColStats cs;
    bool side_pending = false;
    if (d.prof) {
        const int ph = d.begin(S_COLSTATS);
        cs = column_stats(rows, R);
        d.end(ph);
    } else {
        column_stats_alloc(R);
        CK(cudaEventRecord(side.ready, st));
        CK(cudaStreamWaitEvent(side.st.s, side.ready, 0));
        column_stats_launch(rows, R, side.st.s, side.sums, side.c0, side.late);
        CK(cudaEventRecord(side.done, side.st.s));
        ab_->set_write_fence(side.done);
        side_pending = true;
    }
    // a failed solve still waits for the side stream before the session's buffers are reused
    struct SideJoin {
        ColStatsSide& s;
        bool& pending;
        DeviceAbsorber* ab;
        ~SideJoin() {
            if (pending) {
                cudaEventSynchronize(s.done);
                ab->set_write_fence(nullptr);
            }
        }
    } side_join{side, side_pending, ab_.get()};

    // The FE solve, in place
    const bool want_coefs = out.d != nullptr;
    const size_t p_len = ab_->coefs_len();
    std::vector<double> coefs(want_coefs ? p_len * r : 0);
    const SolveInfo info =
    ab_->residualize_device(rows, r, spec.tol, spec.maxiter, want_coefs, nullptr, want_coefs ? coefs.data() : nullptr,
                            spec.prec);
    if (side_pending) {
        CK(cudaEventSynchronize(side.done));
        side_pending = false;
        cs = column_stats_finish(side.sums, side.c0, *side.late, R);
    }
    const std::vector<double>&wmean = cs.wmean, &sumsq = cs.sumsq, &wss_unc = cs.wss_unc, &sd = cs.sd, &wss = cs.wss;
    const double tscale = (kind == 1 || kind == 3) ? double(n) / sumw : 1.0;
    const double tss_y = (has_intercept ? wss[0] : wss_unc[0]) * tscale;

    // Outer products over the block: sum om a a^T of columns `cols` shifted by `shift` (+ the
    // constant), optionally the plain sums of squares; returns the full msz x msz matrix.
    auto outer = [&](const double* src, size_t nrows, int srcR, const std::vector<int>& cols,
                 const std::vector<double>* shift, bool cst, const double* om, const int* perm, bool ssq,
                 std::vector<double>* ss_out) {
        return outer_products(src, nrows, srcR, cols, shift, cst, om, perm, ssq, ss_out);
    };

    // Pass B: weighted Gram of the residualized block (stats.rs:195)
    int ph = d.begin(S_GRAM);
    const double* wv = weighted ? d.wv.p : nullptr;
    std::vector<int> all_cols(r);
    std::iota(all_cols.begin(), all_cols.end(), 0);
    std::vector<double> ss_res;
    std::vector<double> g = outer(rows, n, R, all_cols, nullptr, false, wv, nullptr, true, &ss_res);
    d.end(ph);

    // Collinearity, stage 1 (ols.rs:38 stage1_absorbed): a column absorbed by the FE
    const double ctol = std::min(1e-6, spec.tol / 10.0);
    std::vector<uint8_t> status(nx, 0);
    std::vector<bool> absorbed(r);
    for (size_t j = 0; j < r; j++) absorbed[j] = ss_res[j] / sumsq[j] <= ctol;
    const bool y_abs = nx >= 1 && absorbed[0];
    if (y_abs) {  // reghdfe zeroes the partialled-out depvar
        k_zero_col<<<blocks_for(n, 256), 256, 0, st>>>(rows, n, R, 0);
        d.launches++;
        for (size_t j = 0; j < r; j++) g[j] = g[j * r] = 0.0;
    }
    for (size_t j = 1; j < r; j++)
    if (absorbed[j]) status[j - 1] = 2;
    // stage 2: sweeps on the standardized Gram of the candidates (ols.rs:46, vcov.rs:22)
    std::vector<size_t> cand;
    for (size_t j = 1; j < r; j++)
    if (status[j - 1] == 0) cand.push_back(j);
    const size_t kc = cand.size();
    la::Mat gs(kc * kc);
    for (size_t a = 0; a < kc; a++)
    for (size_t b = 0; b < kc; b++) gs[a * kc + b] = g[cand[a] * r + cand[b]] / (sd[cand[a]] * sd[cand[b]]);
    std::vector<bool> dropped;
    const la::Mat inv_c = la::sweep_inverse(gs, kc, SWEEP_TOL, false, dropped);
    std::vector<size_t> keep_pos, kept;
    for (size_t c = 0; c < kc; c++) {
        if (dropped[c]) status[cand[c] - 1] = 3;
        else {
            keep_pos.push_back(c);
            kept.push_back(cand[c]);
        }
    }
    const size_t k = kept.size();
    la::Mat inv_s(k * k);
    for (size_t a = 0; a < k; a++)
    for (size_t b = 0; b < k; b++) inv_s[a * k + b] = inv_c[keep_pos[a] * kc + keep_pos[b]];
    const double sd_y = sd[0];
    std::vector<double> b_s(k, 0.0), beta(k);
    for (size_t a = 0; a < k; a++)
    for (size_t b = 0; b < k; b++) b_s[a] += inv_s[a * k + b] * (g[kept[b] * r] / (sd[kept[b]] * sd_y));
    for (size_t a = 0; a < k; a++) beta[a] = b_s[a] * sd_y / sd[kept[a]];
    // the fitted state the wild bootstrap starts from: kept columns, raw (X~'W X~)^-1, beta
    fit_ = FitState{};
    fit_.kept = kept;
    fit_.beta = beta;
    fit_.A.assign(k * k, 0.0);
    for (size_t a = 0; a < k; a++)
    for (size_t b = 0; b < k; b++) fit_.A[a * k + b] = inv_s[a * k + b] / (sd[kept[a]] * sd[kept[b]]);
    fit_.rows = rows;
    fit_.R = r;
    fit_.y_absorbed = y_abs;

    // residuals and their weighted sum of squares
    ph = d.begin(S_VARIANCE);
    std::vector<int> kcols(kept.begin(), kept.end());
    d.col.alloc(k + 1);
    d.beta.alloc(k + 1);
    if (k) {
        CK(cudaMemcpyAsync(d.col.p, kcols.data(), k * sizeof(int), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(d.beta.p, beta.data(), k * 8, cudaMemcpyHostToDevice, st));
    }
    // With the iid variance and no residuals asked for, rss comes from the Gram through the normal
    // equations, rss = y'Wy - b'X'Wy, unless that difference cancels (rss below 1e-6 of y'Wy); the
    // residual pass (which the other variances and the residual output need) otherwise.
    double rss = 0.0;
    bool rss_done = false;
    if (vce == 0 && !out.resid && !y_abs && g[0] > 0.0) {
        double by = 0.0;
        for (size_t a = 0; a < k; a++) by += beta[a] * g[kept[a] * r];
        const double rg = g[0] - by;
        if (rg > 1e-6 * g[0]) {
            rss = rg;
            rss_done = true;
        }
    }
    if (!rss_done) {
        d.e.alloc(n);
        d.part.alloc(ST_GRID);
        d.sums.alloc(1);
        k_resid_e<<<ST_GRID, ST_TB, 0, st>>>(rows, n, R, d.col.p, d.beta.p, int(k), y_abs ? 1 : 0, wv, d.e.p, d.part.p);
        k_sum_parts<<<1, 32, 0, st>>>(d.part.p, ST_GRID, 1, d.sums.p);
        d.launches += 2;
        CK(cudaMemcpyAsync(&rss, d.sums.p, 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
    const double rss_s = rss / (sd_y * sd_y);

    // bread: the standardized inverse, bordered by the constant (vcov.rs:220)
    std::vector<double> means_s(k), xbar(k);
    for (size_t a = 0; a < k; a++) {
        means_s[a] = wmean[kept[a]] / sd[kept[a]];
        xbar[a] = wmean[kept[a]];
    }
    double b0_s = wmean[0] / sd_y;
    for (size_t a = 0; a < k; a++) b0_s -= means_s[a] * b_s[a];
    const size_t msz = k + (report_constant ? 1 : 0);
    const double n_const = (kind == 1 || kind == 3) ? double(n) : sumw;
    const la::Mat bread = report_constant ? la::bordered(inv_s, k, means_s, n_const) : inv_s;
    std::vector<double> b_full_s = b_s;
    if (report_constant) b_full_s.push_back(b0_s);

    const Dof dof = dof_end(dof_job);
    const double df_a = double(dof.df_a), df_m = double(k);
    double df_r = bigN - df_a - df_m;
    double g_min = 0.0;
    if (!cg_.empty()) g_min = double(*std::min_element(cg_.begin(), cg_.end()));
    std::vector<double> sc(msz);
    for (size_t a = 0; a < k; a++) sc[a] = sd[kept[a]];
    if (report_constant) sc[k] = 1.0;
    auto standardize = [&](la::Mat& mt) {
        for (size_t a = 0; a < msz; a++)
            for (size_t b = 0; b < msz; b++) mt[a * msz + b] /= sc[a] * sc[b] * sd_y * sd_y;
    };
    la::Mat v_s(msz * msz, 0.0);
    if (msz > 0) {
        if (vce == 0) {
            const double f = (rss_s / bigN) * (bigN / df_r);
            for (size_t i = 0; i < msz * msz; i++) v_s[i] = f * bread[i];
        } else if (vce == 1) {
            d.om.alloc(n);
            k_meat_weights<<<blocks_for(n, 256), 256, 0, st>>>(d.e.p, wv, n, kind, 0, d.om.p);
            d.launches++;
            const std::vector<double> shift = report_constant ? xbar : std::vector<double>(k, 0.0);
            la::Mat meat = outer(rows, n, R, kcols, &shift, report_constant, d.om.p, nullptr, false, nullptr);
            standardize(meat);
            v_s = la::sandwich(bread, meat, msz, bigN / (bigN - df_a - df_m));
        } else if (vce == 4 || vce == 5) {
            // ols.rs:450-474: the full design's leverage h = h_FE + w_v x~'(X~'WX~)^-1 x~, then the
            // regress HC2 / HC3 multipliers (ols/stata_vce.rs:156-167) in the robust meat, no factor
            d.h.alloc(n);
            ab_->fe_leverage_device(d.h.p);
            DBuf<double> ginv;
            ginv.upload(fit_.A.empty() ? std::vector<double>{0.0} : fit_.A, st);
            d.om.alloc(n);
            if (k) CK(cudaMemcpyAsync(d.col.p, kcols.data(), k * sizeof(int), cudaMemcpyHostToDevice, st));
            k_hc_weights<<<blocks_for(n, 256), 256, 0, st>>>(rows, R, d.col.p, int(k), ginv.p, d.e.p, wv, d.h.p,
                                                             kind == 2 ? 1 : 0, vce == 5 ? 1 : 0, n, d.om.p);
            d.launches++;
            const std::vector<double> shift = report_constant ? xbar : std::vector<double>(k, 0.0);
            la::Mat meat = outer(rows, n, R, kcols, &shift, report_constant, d.om.p, nullptr, false, nullptr);
            standardize(meat);
            v_s = la::sandwich(bread, meat, msz, 1.0);
        } else if (vce == 2) {
            d.om.alloc(n);
            k_meat_weights<<<blocks_for(n, 256), 256, 0, st>>>(d.e.p, wv, n, kind, 1, d.om.p);
            d.launches++;
            const std::vector<double> shift = report_constant ? xbar : std::vector<double>(k, 0.0);
            if (k) CK(cudaMemcpyAsync(d.col.p, kcols.data(), k * sizeof(int), cudaMemcpyHostToDevice, st));
            la::Mat meat(msz * msz, 0.0);
            for (auto& sub : d.subsets) {
                d.S.alloc(size_t(sub.G) * msz);
                d.shift.alloc(k + 1);
                if (k) CK(cudaMemcpyAsync(d.shift.p, shift.data(), k * 8, cudaMemcpyHostToDevice, st));
                k_cluster_scores<<<ST_GRID, ST_TB, 0, st>>>(rows, R, d.col.p, d.shift.p, int(k), report_constant ? 1 : 0,
                                                           d.om.p, sub.perm.p, sub.coff.p, sub.G, d.S.p);
                d.launches++;
                std::vector<int> scols(msz);
                std::iota(scols.begin(), scols.end(), 0);
                const la::Mat part = outer(d.S.p, sub.G, int(msz), scols, nullptr, false, nullptr, nullptr, false, nullptr);
                for (size_t i = 0; i < msz * msz; i++) meat[i] += sub.sign * part[i];
                // the next subset's scores need the kept columns again
                if (k) CK(cudaMemcpyAsync(d.col.p, kcols.data(), k * sizeof(int), cudaMemcpyHostToDevice, st));
            }
            standardize(meat);
            const double nested_adj = dof.df_a_nested > 0 ? 1.0 : 0.0;
            const double q_cluster = (bigN - 1.0) / (bigN - nested_adj - df_m - df_a) * g_min / (g_min - 1.0);
            fit_.crv1_scale = q_cluster;
            fit_.ok = true;
            v_s = la::sandwich(bread, meat, msz, q_cluster);
            if (ccodes_.size() > 1) la::fix_psd(v_s, msz, report_constant);
        } else {
            const la::Mat meat = crv3_meat(rows, raw_h, R, kept, beta, wmean, report_constant, g);
            const double nested_adj = dof.df_a_nested > 0 ? 1.0 : 0.0;
            const double q_cluster = (bigN - 1.0) / (bigN - nested_adj - df_m - df_a) * g_min / (g_min - 1.0);
            for (size_t a = 0; a < msz; a++)
                for (size_t b = 0; b < msz; b++)
                    v_s[a * msz + b] = q_cluster * meat[a * msz + b] * sc[a] * sc[b] / (sd_y * sd_y);
            if (ccodes_.size() > 1) la::fix_psd(v_s, msz, report_constant);
        }
    }
    d.end(ph);
    d.collect();
    if (clustered) df_r = std::min(df_r, g_min - 1.0);
    for (size_t i = 0; i < msz; i++)
    for (size_t j = 0; j < i; j++) v_s[j * msz + i] = v_s[i * msz + j];

    // Wald F of the slopes (greedy sweep of their variance)
    double f_stat = nanv();
    if (k > 0) {
        la::Mat vkk(k * k);
        for (size_t a = 0; a < k; a++)
            for (size_t b = 0; b < k; b++) vkk[a * k + b] = v_s[a * msz + b];
        std::vector<bool> dv;
        const la::Mat iv = la::sweep_inverse(vkk, k, F_SWEEP_TOL, true, dv);
        if (std::none_of(dv.begin(), dv.end(), [](bool x) { return x; })) {
            double qf = 0.0;
            for (size_t a = 0; a < k; a++)
                for (size_t b = 0; b < k; b++) qf += b_s[a] * iv[a * k + b] * b_s[b];
            f_stat = finite_or_nan(qf / df_m);
        }
    }
    if (std::any_of(v_s.begin(), v_s.end(), [](double x) { return std::isnan(x); })) std::fill(v_s.begin(), v_s.end(), 0.0);

    // back to the raw scale, in the caller's column positions
    std::vector<double> sx(msz), b_raw(msz), v_raw(msz * msz);
    for (size_t a = 0; a < msz; a++) sx[a] = sc[a] / sd_y;
    for (size_t a = 0; a < msz; a++) b_raw[a] = b_full_s[a] / sx[a];
    for (size_t a = 0; a < msz; a++)
    for (size_t b = 0; b < msz; b++) v_raw[a * msz + b] = v_s[a * msz + b] / (sx[a] * sx[b]);
    const double b0 = report_constant ? b_raw[k] : 0.0;
    const size_t k_all = nx + (report_constant ? 1 : 0);
    std::vector<size_t> pos;
    for (size_t c : kept) pos.push_back(c - 1);
    if (report_constant) pos.push_back(nx);
    if (out.b) std::fill(out.b, out.b + k_all, 0.0);
    if (out.V) std::fill(out.V, out.V + k_all * k_all, 0.0);
    for (size_t a = 0; a < pos.size(); a++) {
        if (out.b) out.b[pos[a]] = b_raw[a];
        if (out.V)
            for (size_t b = 0; b < pos.size(); b++) out.V[pos[a] * k_all + pos[b]] = v_raw[a * msz + b];
    }
    if (out.status) std::copy(status.begin(), status.end(), out.status);
    out.k_all = int(k_all);
    out.y_absorbed = y_abs ? 1 : 0;

    const double tss = tss_y, tss_within = g[0];
    const double used_df_r = bigN - df_a - df_m - double(dof.df_a_nested);
    const double hi = has_intercept ? 1.0 : 0.0;
    const double ln2pi = std::log(2.0 * M_PI);
    out.N = bigN;
    out.rank = df_m;
    out.df_r = df_r;
    out.df_m = df_m;
    out.df_a = df_a;
    out.df_a_initial = double(dof.df_a_initial);
    out.df_a_redundant = double(dof.df_a_redundant);
    out.df_a_nested = double(dof.df_a_nested);
    out.N_clust = clustered ? g_min : nanv();
    out.N_clustervars = clustered ? double(ccodes_.size()) : nanv();
    out.N_clust1 = clustered && !cg_.empty() ? double(cg_[0]) : nanv();
    out.N_clust2 = clustered && cg_.size() > 1 ? double(cg_[1]) : nanv();
    out.num_singletons = double(nsing_);
    out.N_full = bigN + double(nsing_);
    out.report_constant = report_constant ? 1.0 : 0.0;
    out.rss = finite_or_nan(rss);
    out.tss = finite_or_nan(tss);
    out.tss_within = finite_or_nan(tss_within);
    out.mss = finite_or_nan(tss - rss);
    out.rmse = finite_or_nan(used_df_r != 0.0 ? std::sqrt(rss / used_df_r) : std::sqrt(rss));
    out.r2 = finite_or_nan(1.0 - rss / tss);
    out.r2_a = finite_or_nan(1.0 - (rss / used_df_r) / (tss / (bigN - hi)));
    out.r2_within = finite_or_nan(1.0 - rss / tss_within);
    out.r2_a_within = finite_or_nan(1.0 - (rss / used_df_r) / (tss_within / (used_df_r + df_m)));
    out.ll = finite_or_nan(-0.5 * bigN * (1.0 + ln2pi + std::log(rss / bigN)));
    out.ll_0 = finite_or_nan(-0.5 * bigN * (1.0 + ln2pi + std::log(tss_within / bigN)));
    out.F = f_stat;
    out.sumweights = sumw;
    out.ic = double(info.iterations);
    out.nslots = int(dof.slots.size());
    if (out.dof_table)
    for (size_t i = 0; i < dof.slots.size() && i < size_t(MAX_TABLE); i++) {
        const auto& s = dof.slots[i];
        double* t = out.dof_table + 5 * i;
        t[0] = double(s.k);
        t[1] = double(s.m);
        t[2] = double(s.k - s.m);
        t[3] = s.exact ? 0.0 : 1.0;
        t[4] = s.nested ? 1.0 : 0.0;
    }
    if (out.resid) {
        std::vector<double> e(n);
        CK(cudaMemcpyAsync(e.data(), d.e.p, n * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        for (size_t i = 0; i < n; i++) out.resid[pi[i]] = e[i];
    }
    if (out.d) {
        // sum of the fixed effects: the FE fit of y minus the slopes' FE fits, less the constant
        std::vector<double> comb(p_len, 0.0), fit(n);
        for (size_t i = 0; i < p_len; i++) {
            double v = coefs[i * r];
            for (size_t a = 0; a < k; a++) v -= beta[a] * coefs[i * r + kept[a]];
            comb[i] = v;
        }
        ab_->fit_rows(comb.data(), 1, 0, fit.data());
        for (size_t i = 0; i < n; i++) out.d[pi[i]] = fit[i] - b0;
    }
    if (out.groupvar) {
        if (dof.has_groupvar) {
            std::vector<u32> gv(n);
            CK(cudaMemcpyAsync(gv.data(), d.dof.gv.p, n * sizeof(u32), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            for (size_t i = 0; i < n; i++) out.groupvar[i] = double(gv[i]);
        } else {
            std::fill(out.groupvar, out.groupvar + n, nanv());
        }
    }
    CK(cudaGetLastError());
}


// ---------------------------------------------------------------------------------------------
// IV / 2SLS with ivreghdfe conventions (iv.rs:299-700: ivreg2 on the residualized block with
// `small` and `noconstant`, sdofminus = max(df_a, 1)). The block is [y, exog (nx), endog (ne),
// inst (ni)] in row order, residualized in ONE absorber call (iv.rs:409); the weighted Gram of
// the residualized block is the only other pass over all columns. Collinearity: stage 1 (absorbed
// by the FE) on every column, stage 2 on Z = [exog, inst] and then on X = [exog, endog]. With
// X = [endog, exog], Z = [inst, exog] (the coefficient order of e(b)):
//   b = (X'P_Z X)^-1 X'Z (Z'Z)^-1 Z'y,  B = (X'P_Z X)^-1 X'Z (Z'Z)^-1,
//   unadjusted V = rss / (N - K - sdof) (X'P_Z X)^-1,
//   robust V = B [sum m_i z_i z_i'] B' N / (N - K - sdof) (m_i the reghdfe robust multiplier),
//   cluster V = B [sum_g s_g s_g'] B' (N - 1) / (N - K - sdof) G / (G - 1), s_g = sum e w_v z,
// multiway by inclusion-exclusion without an eigenvalue clip (iv.rs:612-640).
void GpuSession::iv(double* rows_in, bool on_device, size_t nx, size_t ne, size_t ni, const IvSpec& spec,
                    IvOut& out) {
    AllocScope alloc_scope(ab_->stream());
    restore_weights();
    SessionDev& d = *d_;
    cudaStream_t st = d.st;
    const size_t n = n_, r = 1 + nx + ne + ni;
    const int R = int(r);
    if (tg_.empty()) throw Error(RC_INVALID_INPUT, "fereg iv: the session absorbs no fixed effects");
    if (ne == 0) throw Error(RC_INVALID_INPUT, "fereg iv: no endogenous regressor");
    if (r + 1 > size_t(OP_MAXM)) throw Error(RC_INVALID_INPUT, "fereg iv: at most 62 columns on the device path");
    double* rows = rows_in;
    if (!on_device) {
        d.rows.alloc(n * r);
        CK(cudaMemcpyAsync(d.rows.p, rows_in, n * r * 8, cudaMemcpyHostToDevice, st));
        rows = d.rows.p;
    }
    const int kind = kind_;
    const bool weighted = !wk_.empty();
    const double bigN = kind == 2 ? sumw_ : double(n);
    int vce = spec.vce;
    if (vce == 0 && kind == 3) vce = 1;  // pweights imply robust
    if (vce == 2 && ccodes_.empty()) throw Error(RC_INVALID_INPUT, "fereg iv: cluster variance without clusters");

    std::future<Dof> dof_job = dof_begin(vce == 2, false, false);
    int ph = d.begin(S_COLSTATS);
    const ColStats cs = column_stats(rows, R);
    d.end(ph);
    const SolveInfo info = ab_->residualize_device(rows, r, spec.tol, spec.maxiter, false, nullptr, nullptr, spec.prec);
    ph = d.begin(S_GRAM);
    const double* wv = weighted ? d.wv.p : nullptr;
    std::vector<int> all(r);
    std::iota(all.begin(), all.end(), 0);
    std::vector<double> ss_res;
    const std::vector<double> g = outer_products(rows, n, R, all, nullptr, false, wv, nullptr, true, &ss_res);
    d.end(ph);

    // collinearity (iv.rs:443-490)
    const double ctol = std::min(1e-6, spec.tol / 10.0);
    std::vector<uint8_t> status(r - 1, 0);
    for (size_t j = 1; j < r; j++)
        if (ss_res[j] / cs.sumsq[j] <= ctol) status[j - 1] = 2;
    auto alive = [&](size_t c) { return status[c - 1] == 0; };
    auto stage2 = [&](const std::vector<size_t>& cand) {
        const size_t kc = cand.size();
        la::Mat gs(kc * kc);
        for (size_t a = 0; a < kc; a++)
            for (size_t b = 0; b < kc; b++)
                gs[a * kc + b] = g[cand[a] * r + cand[b]] / (cs.sd[cand[a]] * cs.sd[cand[b]]);
        std::vector<bool> dropped;
        la::sweep_inverse(gs, kc, SWEEP_TOL, false, dropped);
        for (size_t c = 0; c < kc; c++)
            if (dropped[c]) status[cand[c] - 1] = 3;
    };
    auto exog = [&](size_t j) { return 1 + j; };
    auto endog = [&](size_t j) { return 1 + nx + j; };
    auto inst = [&](size_t j) { return 1 + nx + ne + j; };
    std::vector<size_t> zc, xc;
    for (size_t j = 0; j < nx; j++)
        if (alive(exog(j))) zc.push_back(exog(j));
    for (size_t j = 0; j < ni; j++)
        if (alive(inst(j))) zc.push_back(inst(j));
    stage2(zc);
    for (size_t j = 0; j < nx; j++)
        if (alive(exog(j))) xc.push_back(exog(j));
    for (size_t j = 0; j < ne; j++)
        if (alive(endog(j))) xc.push_back(endog(j));
    stage2(xc);
    std::vector<size_t> en, ex, iz;
    for (size_t j = 0; j < ne; j++)
        if (alive(endog(j))) en.push_back(endog(j));
    for (size_t j = 0; j < nx; j++)
        if (alive(exog(j))) ex.push_back(exog(j));
    for (size_t j = 0; j < ni; j++)
        if (alive(inst(j))) iz.push_back(inst(j));
    if (iz.size() < en.size())
        throw Error(RC_NOT_IDENTIFIED,
                    "equation not identified; must have at least as many instruments not in the regression as there "
                    "are instrumented variables");
    std::vector<size_t> xcols(en), zcols(iz);
    xcols.insert(xcols.end(), ex.begin(), ex.end());
    zcols.insert(zcols.end(), ex.begin(), ex.end());
    const size_t k = xcols.size(), l = zcols.size();
    if (k == 0) throw Error(RC_INVALID_INPUT, "fereg iv: every regressor was dropped");

    // cross products and 2SLS (s_crossprods, s_gmm1s)
    la::Mat xz(k * l), zz(l * l), zy(l);
    for (size_t a = 0; a < k; a++)
        for (size_t b = 0; b < l; b++) xz[a * l + b] = g[xcols[a] * r + zcols[b]];
    for (size_t a = 0; a < l; a++) {
        zy[a] = g[zcols[a] * r];
        for (size_t b = 0; b < l; b++) zz[a * l + b] = g[zcols[a] * r + zcols[b]];
    }
    la::Mat zzinv, xpzx_inv;
    if (!la::spd_inv(zz, l, zzinv)) throw Error(RC_INVALID_INPUT, "fereg iv: Z'Z is not positive definite");
    const la::Mat xz_zzinv = la::mul_rect(xz, zzinv, k, l, l);
    la::Mat xzt(l * k);
    for (size_t a = 0; a < k; a++)
        for (size_t b = 0; b < l; b++) xzt[b * k + a] = xz[a * l + b];
    la::Mat xpzx = la::mul_rect(xz_zzinv, xzt, k, l, k);
    la::symmetrize(xpzx, k);
    if (!la::spd_inv(xpzx, k, xpzx_inv)) throw Error(RC_INVALID_INPUT, "fereg iv: X'P_Z X is not positive definite");
    const la::Mat bmat = la::mul_rect(xpzx_inv, xz_zzinv, k, k, l);
    const la::Mat beta = la::mul_rect(bmat, zy, k, l, 1);

    // residuals and their weighted sum of squares
    ph = d.begin(S_VARIANCE);
    std::vector<int> kx(xcols.begin(), xcols.end()), kz(zcols.begin(), zcols.end());
    d.col.alloc(std::max(k, l) + 1);
    d.beta.alloc(k + 1);
    CK(cudaMemcpyAsync(d.col.p, kx.data(), k * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d.beta.p, beta.data(), k * 8, cudaMemcpyHostToDevice, st));
    d.e.alloc(n);
    d.part.alloc(ST_GRID);
    d.sums.alloc(1);
    k_resid_e<<<ST_GRID, ST_TB, 0, st>>>(rows, n, R, d.col.p, d.beta.p, int(k), 0, wv, d.e.p, d.part.p);
    k_sum_parts<<<1, 32, 0, st>>>(d.part.p, ST_GRID, 1, d.sums.p);
    d.launches += 2;
    double rss = 0.0;
    CK(cudaMemcpyAsync(&rss, d.sums.p, 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));

    const Dof dof = dof_end(dof_job);
    const double sdof = std::max<double>(double(dof.df_a), 1.0);
    const double nk = bigN - double(k) - sdof;
    const double g_min = cg_.empty() ? 0.0 : double(*std::min_element(cg_.begin(), cg_.end()));
    la::Mat V(k * k, 0.0);
    if (vce == 0) {
        for (size_t i = 0; i < k * k; i++) V[i] = xpzx_inv[i] * (rss / nk);
    } else {
        d.om.alloc(n);
        k_meat_weights<<<blocks_for(n, 256), 256, 0, st>>>(d.e.p, wv, n, kind, vce == 2 ? 1 : 0, d.om.p);
        d.launches++;
        la::Mat S(l * l, 0.0);
        if (vce == 1) {
            S = outer_products(rows, n, R, kz, nullptr, false, d.om.p, nullptr, false, nullptr);
        } else {
            for (auto& sub : d.subsets) {
                CK(cudaMemcpyAsync(d.col.p, kz.data(), l * sizeof(int), cudaMemcpyHostToDevice, st));
                d.S.alloc(size_t(sub.G) * l);
                k_cluster_scores<<<ST_GRID, ST_TB, 0, st>>>(rows, R, d.col.p, nullptr, int(l), 0, d.om.p, sub.perm.p,
                                                           sub.coff.p, sub.G, d.S.p);
                d.launches++;
                std::vector<int> sc(l);
                std::iota(sc.begin(), sc.end(), 0);
                const la::Mat part = outer_products(d.S.p, sub.G, int(l), sc, nullptr, false, nullptr, nullptr, false,
                                                    nullptr);
                for (size_t i = 0; i < l * l; i++) S[i] += sub.sign * part[i];
            }
        }
        la::Mat bt(l * k);
        for (size_t a = 0; a < k; a++)
            for (size_t b = 0; b < l; b++) bt[b * k + a] = bmat[a * l + b];
        V = la::mul_rect(la::mul_rect(bmat, S, k, l, l), bt, k, l, k);
        la::symmetrize(V, k);
        const double adj = vce == 2 ? (bigN - 1.0) / (bigN - double(k) - sdof) * g_min / (g_min - 1.0) : bigN / nk;
        for (double& x : V) x *= adj;
    }
    d.end(ph);
    d.collect();

    // Wald F of all coefficients (greedy sweep of V)
    double f_stat = nanv();
    {
        std::vector<bool> dv;
        const la::Mat vi = la::sweep_inverse(V, k, F_SWEEP_TOL, true, dv);
        if (std::none_of(dv.begin(), dv.end(), [](bool x) { return x; })) {
            double q = 0.0;
            for (size_t a = 0; a < k; a++)
                for (size_t b = 0; b < k; b++) q += beta[a] * vi[a * k + b] * beta[b];
            f_stat = finite_or_nan(q / double(k));
        }
    }
    // results in e(b) order [endog..., exog...]
    const size_t k_all = ne + nx;
    auto pos = [&](size_t c) { return c > nx ? c - 1 - nx : ne + (c - 1); };
    if (out.b) std::fill(out.b, out.b + k_all, 0.0);
    if (out.V) std::fill(out.V, out.V + k_all * k_all, 0.0);
    for (size_t a = 0; a < k; a++) {
        if (out.b) out.b[pos(xcols[a])] = beta[a];
        if (out.V)
            for (size_t b = 0; b < k; b++) out.V[pos(xcols[a]) * k_all + pos(xcols[b])] = V[a * k + b];
    }
    if (out.status) std::copy(status.begin(), status.end(), out.status);
    out.N = bigN;
    out.df_m = double(k);
    out.df_r = vce == 2 ? g_min - 1.0 : nk;
    out.df_a = double(dof.df_a);
    out.sdofminus = sdof;
    out.rss = rss;
    out.rmse = std::sqrt(rss / nk);
    out.F = f_stat;
    out.N_clust = vce == 2 ? g_min : nanv();
    out.ic = double(info.iterations);
    out.endog_ct = int(en.size());
    out.inexog_ct = int(ex.size());
    out.exexog_ct = int(iz.size());
    CK(cudaGetLastError());
}

// ---------------------------------------------------------------------------------------------
// Wild cluster bootstrap WCR11 of coefficient bs.coef (H0: beta = r0): Rademacher weights on
// the clusters of the session's first cluster dimension, restricted residuals (impose_null),
// CRV1 over all the session's cluster dimensions, two-tailed p-value
// (wildboot/ols.rs:243-650, weights.rs:39-160, mod.rs:529 compute_pvalue). Each tile of draws is
// one n x tile block residualized by the absorber as block-PCG columns; see boot.cuh.
void GpuSession::wildboot(double* rows, bool on_device, size_t nx, const OlsSpec& ospec, const BootSpec& bs,
                          BootOut& out) {
    AllocScope alloc_scope(ab_->stream());
    restore_weights();
    if (ccodes_.empty()) throw Error(RC_INVALID_INPUT, "fereg wildboot: the session has no cluster dimension");
    if (bs.coef >= nx) throw Error(RC_INVALID_INPUT, "fereg wildboot: coefficient index out of range");
    if (bs.reps == 0 || bs.tile == 0) throw Error(RC_INVALID_INPUT, "fereg wildboot: reps and tile must be positive");
    if (d_->subsets.size() > size_t(BOOT_MAX_SUB)) throw Error(RC_INVALID_INPUT, "fereg wildboot: at most 3 cluster dimensions");
    OlsSpec os = ospec;
    os.vce = 2;
    const size_t k_all = nx + 1;
    std::vector<double> b(k_all), V(k_all * k_all);
    OlsOut oo;
    oo.b = b.data();
    oo.V = V.data();
    ols(rows, on_device, nx, os, oo);
    if (!fit_.ok) throw Error(RC_INTERNAL, "fereg wildboot: no cluster variance");
    SessionDev& d = *d_;
    cudaStream_t st = d.st;
    const size_t n = n_, k = fit_.kept.size();
    const int R = int(fit_.R);
    size_t pj = k;
    for (size_t a = 0; a < k; a++)
        if (fit_.kept[a] == bs.coef + 1) pj = a;
    if (pj == k) throw Error(RC_INVALID_INPUT, "fereg wildboot: the tested coefficient was dropped (collinear or absorbed)");
    const std::vector<double>& A = fit_.A;
    const std::vector<double>& beta = fit_.beta;
    // restricted coefficients (q = 1): beta_r = beta - A e_j (beta_j - r0) / A_jj
    std::vector<double> beta_r(k), ca(k);
    const double lam = (beta[pj] - bs.r0) / A[pj * k + pj];
    for (size_t a = 0; a < k; a++) {
        beta_r[a] = beta[a] - A[a * k + pj] * lam;
        ca[a] = -A[pj * k + a];  // k_resid_e on a zero y gives c = a' x~
    }
    const double* wv = wk_.empty() ? nullptr : d.wv.p;
    const int blocks = int(std::min<size_t>((n + 255) / 256, 148 * 16));
    std::vector<int> kcols(fit_.kept.begin(), fit_.kept.end());
    DBuf<int> col;
    DBuf<double> bvec, er, cvec, cw, om, Phi, part;
    col.upload(kcols, st);
    bvec.upload(beta_r, st);
    er.alloc(n);
    cvec.alloc(n);
    cw.alloc(n);
    om.alloc(n);
    part.alloc(ST_GRID);
    k_resid_e<<<ST_GRID, ST_TB, 0, st>>>(fit_.rows, n, R, col.p, bvec.p, int(k), fit_.y_absorbed ? 1 : 0, nullptr, er.p,
                                         part.p);
    bvec.upload(ca, st);
    k_resid_e<<<ST_GRID, ST_TB, 0, st>>>(fit_.rows, n, R, col.p, bvec.p, int(k), 1, nullptr, cvec.p, part.p);
    k_mul<<<blocks, 256, 0, st>>>(cvec.p, wv, n, cw.p);      // w c
    k_mul<<<blocks, 256, 0, st>>>(er.p, wv, n, om.p);        // w e_r
    d.launches += 4;
    // phi_g over the bootstrap clusters (first dimension), psi_{s,g} and the original statistic's
    // cluster sums over every subset
    const auto& s0 = d.subsets[0];
    Phi.alloc(size_t(s0.G) * k + 1);
    k_cluster_scores<<<ST_GRID, ST_TB, 0, st>>>(fit_.rows, R, col.p, nullptr, int(k), 0, om.p, s0.perm.p, s0.coff.p,
                                               s0.G, Phi.p);
    DBuf<double> ucw;
    ucw.alloc(n);
    k_mul<<<blocks, 256, 0, st>>>(cw.p, d.e.p, n, ucw.p);   // w c e_u
    std::vector<DBuf<double>> Psi(d.subsets.size()), T1(d.subsets.size()), Tu(d.subsets.size());
    double v_orig = 0.0;
    for (size_t si = 0; si < d.subsets.size(); si++) {
        const auto& sub = d.subsets[si];
        Psi[si].alloc(size_t(sub.G) * k + 1);
        k_cluster_scores<<<ST_GRID, ST_TB, 0, st>>>(fit_.rows, R, col.p, nullptr, int(k), 0, cw.p, sub.perm.p,
                                                   sub.coff.p, sub.G, Psi[si].p);
        Tu[si].alloc(sub.G);
        k_cluster_scores<<<ST_GRID, ST_TB, 0, st>>>(fit_.rows, R, col.p, nullptr, 0, 1, ucw.p, sub.perm.p, sub.coff.p,
                                                   sub.G, Tu[si].p);
        d.launches += 2;
        std::vector<double> h(sub.G);
        CK(cudaMemcpyAsync(h.data(), Tu[si].p, size_t(sub.G) * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        double acc = 0.0;
        for (double x : h) acc += x * x;
        v_orig += sub.sign * acc;
    }
    d.launches += 3;
    v_orig *= fit_.crv1_scale;
    out.point = beta[pj];
    out.se = v_orig > 0.0 ? std::sqrt(v_orig) : nanv();
    out.stat = v_orig > 0.0 ? (beta[pj] - bs.r0) / out.se : nanv();

    // draws (weights.rs:39-63 resolve_reps): full enumeration of the 2^G sign patterns when
    // G <= 20 and 2^G <= reps
    const u32 G0 = s0.G;
    const bool full = G0 <= 20 && (size_t(1) << G0) <= bs.reps;
    const size_t reps = full ? (size_t(1) << G0) : bs.reps;
    out.reps = reps;
    out.full_enum = full;
    const u32 nwords = (G0 + 63) / 64;
    const std::vector<u32>& pi = ab_->row_order();
    std::vector<u32> bcode(n);
    for (size_t i = 0; i < n; i++) bcode[i] = ccodes_[0][pi[i]];
    DBuf<u32> bcode_d;
    bcode_d.upload(bcode, st);
    DBuf<double> Adev, U, D, Z, tb;
    Adev.upload(A, st);
    const size_t tile = std::min(bs.tile, reps);
    DBuf<u64> Wd;
    Wd.alloc(tile * nwords);
    U.alloc(tile * k + 1);
    D.alloc(tile * k + 1);
    Z.alloc(n * tile);
    tb.alloc(tile);
    for (size_t si = 0; si < d.subsets.size(); si++) T1[si].alloc(size_t(d.subsets[si].G) * tile);
    std::vector<double> t_host(reps);
    for (size_t b0 = 0; b0 < reps; b0 += tile) {
        ab_->ctx().check();
        const u32 bt = u32(std::min(tile, reps - b0));
        k_boot_words<<<std::max(1, int((size_t(bt) * nwords + 255) / 256)), 256, 0, st>>>(bs.seed, b0, bt, nwords,
                                                                                         full ? 1 : 0, Wd.p);
        k_boot_gen<<<int(std::min<size_t>((n * bt + 255) / 256, 148 * 32)), 256, 0, st>>>(n, bt, er.p, bcode_d.p, Wd.p,
                                                                                          nwords, Z.p);
        d.launches += 2;
        ab_->residualize_device(Z.p, bt, bs.tol, bs.maxiter, false, nullptr, nullptr, bs.prec);
        if (k) {
            k_boot_u<<<std::max(1, int((size_t(bt) * k + 127) / 128)), 128, 0, st>>>(bt, G0, int(k), Wd.p, nwords, Phi.p,
                                                                                    U.p);
            k_boot_delta<<<std::max(1, int((size_t(bt) * k + 127) / 128)), 128, 0, st>>>(bt, int(k), Adev.p, U.p, D.p);
            d.launches += 2;
        }
        BootSubsets subs{};
        subs.n = int(d.subsets.size());
        for (size_t si = 0; si < d.subsets.size(); si++) {
            const auto& sub = d.subsets[si];
            const size_t warps = size_t(sub.G) * ((bt + 31) / 32);
            k_boot_t1<<<int(std::min<size_t>((warps * 32 + 255) / 256, 148 * 32)), 256, 0, st>>>(Z.p, bt, cw.p, sub.perm.p,
                                                                                               sub.coff.p, sub.G, T1[si].p);
            d.launches++;
            subs.T1[si] = T1[si].p;
            subs.Psi[si] = Psi[si].p;
            subs.G[si] = sub.G;
            subs.sign[si] = sub.sign;
        }
        k_boot_var<<<int(std::min<u32>(bt, 148 * 8)), BOOT_TB, 0, st>>>(bt, subs, D.p, int(k), int(pj), fit_.crv1_scale,
                                                                      tb.p);
        d.launches++;
        CK(cudaMemcpyAsync(t_host.data() + b0, tb.p, size_t(bt) * 8, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    CK(cudaGetLastError());
    if (out.t_boot) std::copy(t_host.begin(), t_host.end(), out.t_boot);
    // mod.rs:529 compute_pvalue, two-tailed: share of finite draws with |t*| > |t| + 1e-12 (1 + |t|)
    out.pvalue = nanv();
    if (std::isfinite(out.stat)) {
        const double eps = 1e-12 * (1.0 + std::fabs(out.stat));
        size_t feas = 0, hi = 0;
        for (double x : t_host) {
            if (!std::isfinite(x)) continue;
            feas++;
            if (std::fabs(x) > std::fabs(out.stat) + eps) hi++;
        }
        if (feas) out.pvalue = double(hi) / double(feas);
    }
}

// ---------------------------------------------------------------------------------------------
// GLM by IRLS, Poisson PML or logit (glm/irls.rs:367-560 with ppmlhdfe conventions,
// glm/mod.rs:1053-1140 for the variance). Each iteration: the family's w and z (device), the weight state
// refreshed on the device, [z, X] residualized warm-started from the previous FE coefficients at
// an inner tolerance tightened toward max(1e-12, min(itol, 0.1 tol)) by ppmlhdfe's heuristic
// schedule (irls.rs:900-911, with its eps prediction), the weighted regression on the
// residualized block (device Gram, host sweep), eta = z - e and mu = exp(eta) with the deviance
// (device). Stops when the relative deviance change |D - D'| / max(min(D, D'), 0.1) < tol with the
// inner tolerance at its floor. Collinearity is settled in the first iteration (ppmlhdfe
// remove_collinears): columns absorbed by the FE, then columns collinear with the others. The
// variance uses the last iteration's weights: robust, (X~'WX~)^-1 [sum (e w)^2 x~ x~'] (X~'WX~)^-1
// N / (N - 1), clustered with G / (G - 1) and the multiway eigenvalue clip, or (logit `oim`)
// the inverse Hessian (X~'WX~)^-1.
namespace {

constexpr double EPS1 = 2.220446049250313e-16;  // Mata epsilon(1)

bool inrange(double x, double lb, double ub) { return !std::isnan(lb) && lb <= x && (std::isnan(ub) || x <= ub); }

// ppmlhdfe predict_eps (irls.rs:105-140): ln eps of the last three iterations; once all three
// are known, the cubic through (i, ln eps_i), i = 1..3 without a constant, evaluated at i = 4.
struct EpsHistory {
    double h[3] = {nanv(), nanv(), nanv()};
    double predict(double eps) {
        int pos = 0;
        for (double v : h) pos += !std::isnan(v);
        const bool abort = pos + 1 < 3;
        const double le = eps > 0.0 ? std::log(eps) : nanv();
        if (pos < 3) {
            h[pos] = le;
        } else {
            h[0] = h[1];
            h[1] = h[2];
            h[2] = le;
        }
        if (abort || std::isnan(h[0]) || std::isnan(h[1]) || std::isnan(h[2])) return nanv();
        double a[3][4] = {{1, 1, 1, h[0]}, {2, 4, 8, h[1]}, {3, 9, 27, h[2]}};
        for (int p = 0; p < 3; p++)
            for (int r = p + 1; r < 3; r++) {
                const double f = a[r][p] / a[p][p];
                for (int j = p; j < 4; j++) a[r][j] -= f * a[p][j];
            }
        double c[3] = {0, 0, 0};
        for (int p = 2; p >= 0; p--) {
            double s = a[p][3];
            for (int j = p + 1; j < 3; j++) s -= a[p][j] * c[j];
            c[p] = s / a[p][p];
        }
        return std::exp(4.0 * c[0] + 16.0 * c[1] + 64.0 * c[2]);
    }
};

}  // namespace

void GpuSession::glm(double* rows_in, bool on_device, size_t nx, const GlmSpec& gs, GlmOut& out) {
    AllocScope alloc_scope(ab_->stream());
    if (!wk_.empty()) throw Error(RC_INVALID_INPUT, "fereg glm: weighted sessions are not supported");
    if (gs.family != 0 && gs.family != 1) throw Error(RC_INVALID_INPUT, "fereg glm: family is 0 (Poisson) or 1 (logit)");
    const int fam = gs.family;
    if (gs.vce == 2 && ccodes_.empty()) throw Error(RC_INVALID_INPUT, "fereg glm: cluster variance without clusters");
    if (1 + nx + 1 > size_t(OP_MAXM)) throw Error(RC_INVALID_INPUT, "fereg glm: at most 62 regressors");
    SessionDev& d = *d_;
    cudaStream_t st = d.st;
    const size_t n = n_, r = 1 + nx;
    const int R = int(r);
    const int blocks = int(std::min<size_t>((n + 255) / 256, 148 * 16));
    DBuf<double> raw, B, mu, eta, eta_old, z, w, e, part, om;
    DBuf<int> flag;
    raw.alloc(n * r);
    CK(cudaMemcpyAsync(raw.p, rows_in, n * r * 8, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
    B.alloc(n * r);
    mu.alloc(n);
    eta.alloc(n);
    if (fam == 1) eta_old.alloc(n);
    z.alloc(n);
    w.alloc(n);
    e.alloc(n);
    om.alloc(n);
    part.alloc(GLM_TB * 8);
    flag.alloc(1);
    CK(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
    k_glm_ysum<<<GLM_TB, GLM_TB, 0, st>>>(raw.p, n, R, fam, part.p, flag.p);
    auto host_sum = [&](int parts) {
        std::vector<double> h(static_cast<size_t>(parts));
        CK(cudaMemcpyAsync(h.data(), part.p, size_t(parts) * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        double t = 0.0;
        for (double x : h) t += x;
        return t;
    };
    const double ysum = host_sum(GLM_TB);
    int neg = 0;
    CK(cudaMemcpyAsync(&neg, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (neg)
        throw Error(RC_INVALID_INPUT, fam == 0 ? "fereg glm: the dependent variable must be nonnegative"
                                               : "fereg glm: the logit outcome must be 0 or 1");
    if (!(ysum > 0.0)) throw Error(RC_TOO_FEW_OBS, "insufficient observations (the dependent variable is all zero)");
    if (fam == 1 && !(ysum < double(n))) throw Error(RC_TOO_FEW_OBS, "insufficient observations (the outcome never varies)");
    k_glm_start<<<blocks, 256, 0, st>>>(raw.p, n, R, fam == 0 ? ysum / double(n) : 0.5, fam, mu.p, eta.p);
    d.launches += 2;

    // unweighted sums of squares of the raw regressors (stage-1 collinearity, ols.rs:38)
    std::vector<int> all(r);
    std::iota(all.begin(), all.end(), 0);
    std::vector<double> sumsq;
    outer_products(raw.p, n, R, all, nullptr, false, nullptr, nullptr, true, &sumsq);
    const double highest = std::max(1e-12, std::min(gs.itol, 0.1 * gs.tol));  // glm/mod.rs:826
    double tol_in = std::max(1e-4, gs.tol);
    double dev_old = nanv(), dev = nanv(), eps = nanv(), alt_tol = nanv();
    EpsHistory hist;
    bool have_warm = false, converged = false;
    std::vector<uint8_t> status(nx, 0);
    std::vector<size_t> kept;
    la::Mat inv;
    std::vector<double> beta;
    u64 iters = 0, pcg = 0;
    for (size_t it = 1; it <= gs.maxiter; it++) {
        ab_->ctx().check();
        iters = it;
        const double predicted = hist.predict(eps);
        int ph = d.begin(S_WEIGHTS);
        k_glm_work<<<blocks, 256, 0, st>>>(raw.p, n, R, fam, mu.p, eta.p, B.p, z.p, w.p);
        d.launches++;
        ab_->set_weights_device(w.p);
        d.end(ph);
        // warm start: the previous iteration's reduced solution, left on the device
        const SolveInfo si = have_warm ? ab_->residualize_device_warm_last(B.p, r, tol_in, gs.inner_maxiter, gs.prec)
                                       : ab_->residualize_device(B.p, r, tol_in, gs.inner_maxiter, false, nullptr,
                                                                 nullptr, gs.prec);
        pcg += si.iterations;
        std::vector<double> ss_res;
        ph = d.begin(S_GRAM);
        const std::vector<double> G = outer_products(B.p, n, R, all, nullptr, false, w.p, nullptr, true, &ss_res);
        d.end(ph);
        ph = d.begin(S_VARIANCE);
        if (it == 1) {  // columns absorbed by the FE, then collinear ones
            const double ctol = std::min(1e-6, gs.tol / 10.0);
            std::vector<size_t> cand;
            for (size_t j = 1; j < r; j++) {
                if (ss_res[j] / sumsq[j] <= ctol) status[j - 1] = 2;
                else cand.push_back(j);
            }
            const size_t kc = cand.size();
            la::Mat gc(kc * kc);
            for (size_t a = 0; a < kc; a++)
                for (size_t b = 0; b < kc; b++) gc[a * kc + b] = G[cand[a] * r + cand[b]];
            std::vector<bool> dropped;
            la::sweep_inverse(gc, kc, SWEEP_TOL, false, dropped);
            for (size_t c = 0; c < kc; c++) {
                if (dropped[c]) status[cand[c] - 1] = 3;
                else kept.push_back(cand[c]);
            }
        }
        const size_t k = kept.size();
        la::Mat gk(k * k);
        for (size_t a = 0; a < k; a++)
            for (size_t b = 0; b < k; b++) gk[a * k + b] = G[kept[a] * r + kept[b]];
        std::vector<bool> dk;
        inv = la::sweep_inverse(gk, k, SWEEP_TOL, false, dk);
        beta.assign(k, 0.0);
        for (size_t a = 0; a < k; a++)
            for (size_t b = 0; b < k; b++) beta[a] += inv[a * k + b] * G[kept[b] * r];
        std::vector<int> kc(kept.begin(), kept.end());
        d.col.alloc(k + 1);
        d.beta.alloc(k + 1);
        if (k) {
            CK(cudaMemcpyAsync(d.col.p, kc.data(), k * sizeof(int), cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(d.beta.p, beta.data(), k * 8, cudaMemcpyHostToDevice, st));
        }
        k_resid_e<<<ST_GRID, ST_TB, 0, st>>>(B.p, n, R, d.col.p, d.beta.p, int(k), 0, nullptr, e.p, part.p);
        k_glm_update<<<GLM_TB, GLM_TB, 0, st>>>(raw.p, n, R, fam, z.p, e.p, eta.p, fam == 1 ? eta_old.p : nullptr,
                                                mu.p, part.p);
        d.launches += 2;
        dev = 2.0 * host_sum(GLM_TB);
        // logit step halving while the deviance rose (irls.rs:739-748, at most 25 halvings)
        if (fam == 1 && it > 1) {
            for (int h = 0; h < 25 && (std::isnan(dev) || dev > dev_old + 1e-9 * std::max(std::fabs(dev_old), 1.0));
                 h++) {
                k_glm_halve<<<GLM_TB, GLM_TB, 0, st>>>(raw.p, n, R, fam, eta_old.p, eta.p, mu.p, part.p);
                d.launches++;
                dev = 2.0 * host_sum(GLM_TB);
            }
        }
        d.end(ph);
        if (!std::isfinite(dev)) throw Error(RC_CONVERGENCE, "fereg glm: the deviance is not finite");
        have_warm = true;
        if (it > 1) {
            double delta = dev_old - dev;
            if (!std::isnan(delta) && dev < 0.1 * delta) delta = dev;
            eps = std::fabs(delta) / std::max(std::min(dev, dev_old), 0.1);
            if (eps < gs.tol && tol_in <= 1.1 * highest) {
                converged = true;
                dev_old = dev;
                break;
            }
            // inner tolerance schedule (irls.rs:900-911, ppmlhdfe use_heuristic_tol): a decade,
            // or down to the decade of 0.1 eps seen at the previous tightening, and one more
            // decade when the predicted eps is already below tol
            if (eps < tol_in) {
                tol_in = std::max(std::min(0.1 * tol_in, alt_tol), highest);
                alt_tol = std::pow(10.0, -std::ceil(std::log10(1.0 / std::max(0.1 * eps, EPS1))));
            }
            if (inrange(gs.tol, predicted, eps) && inrange(tol_in / highest, 1.1, 10.1)) tol_in *= 0.1;
        }
        dev_old = dev;
    }
    if (!converged) throw Error(RC_CONVERGENCE, "fereg glm: IRLS did not converge");

    // variance on the last iteration's weights (w, e and the residualized block B)
    const size_t k = kept.size();
    std::vector<int> kc(kept.begin(), kept.end());
    la::Mat V(k * k, 0.0);
    const double bigN = double(n);
    if (k) {
        if (gs.vce == 2) {
            k_glm_score<<<blocks, 256, 0, st>>>(e.p, w.p, n, 0, om.p);
            d.launches++;
            la::Mat meat(k * k, 0.0);
            for (auto& sub : d.subsets) {
                d.S.alloc(size_t(sub.G) * k);
                d.col.alloc(k + 1);
                CK(cudaMemcpyAsync(d.col.p, kc.data(), k * sizeof(int), cudaMemcpyHostToDevice, st));
                k_cluster_scores<<<ST_GRID, ST_TB, 0, st>>>(B.p, R, d.col.p, nullptr, int(k), 0, om.p, sub.perm.p,
                                                           sub.coff.p, sub.G, d.S.p);
                d.launches++;
                std::vector<int> sc(k);
                std::iota(sc.begin(), sc.end(), 0);
                const la::Mat pm = outer_products(d.S.p, sub.G, int(k), sc, nullptr, false, nullptr, nullptr, false, nullptr);
                for (size_t i = 0; i < k * k; i++) meat[i] += sub.sign * pm[i];
            }
            const double gmin = double(*std::min_element(cg_.begin(), cg_.end()));
            V = la::sandwich(inv, meat, k, gmin > 1.0 ? gmin / (gmin - 1.0) : 0.0);
            if (ccodes_.size() > 1) la::fix_psd(V, k, false);
            out.N_clust = gmin;
        } else if (gs.vce == 1) {
            k_glm_score<<<blocks, 256, 0, st>>>(e.p, w.p, n, 1, om.p);
            d.launches++;
            const la::Mat meat = outer_products(B.p, n, R, kc, nullptr, false, om.p, nullptr, false, nullptr);
            V = la::sandwich(inv, meat, k, bigN / (bigN - 1.0));
        } else {
            V = inv;  // oim: the inverse Hessian (X~'WX~)^-1
        }
    }
    // Wald chi2 of the slopes (greedy sweep of V)
    double chi2 = nanv();
    if (k) {
        std::vector<bool> dv;
        const la::Mat iv = la::sweep_inverse(V, k, F_SWEEP_TOL, true, dv);
        if (std::none_of(dv.begin(), dv.end(), [](bool x) { return x; })) {
            double q = 0.0;
            for (size_t a = 0; a < k; a++)
                for (size_t b = 0; b < k; b++) q += beta[a] * iv[a * k + b] * beta[b];
            chi2 = finite_or_nan(q);
        }
    }
    k_glm_ll<<<GLM_TB, GLM_TB, 0, st>>>(raw.p, n, R, fam, eta.p, mu.p, part.p);
    d.launches++;
    const double ll = host_sum(GLM_TB);
    if (out.b) std::fill(out.b, out.b + nx, 0.0);
    if (out.V) std::fill(out.V, out.V + nx * nx, 0.0);
    for (size_t a = 0; a < k; a++) {
        if (out.b) out.b[kept[a] - 1] = beta[a];
        if (out.V)
            for (size_t b = 0; b < k; b++) out.V[(kept[a] - 1) * nx + (kept[b] - 1)] = V[a * k + b];
    }
    if (out.status) std::copy(status.begin(), status.end(), out.status);
    out.N = bigN;
    out.deviance = dev;
    out.ll = ll;
    out.chi2 = chi2;
    out.df_m = double(k);
    out.iterations = iters;
    out.pcg_iterations = pcg;
    out.converged = converged;
    d.collect();
    CK(cudaGetLastError());
    irls_weights_ = true;  // the absorber holds the last IRLS weights
}

// The absorber back on the session's weights after a GLM call left its IRLS weights there (the
// GLM runs on unweighted sessions only).
void GpuSession::restore_weights() {
    if (!irls_weights_) return;
    ab_->set_weights(nullptr);
    irls_weights_ = false;
}

// glm/separation.rs:61-196 relu on the device: the method of weighting (M = ceil(eps^-1/2) on
// y > 0, 1 on y = 0) of the ReLU working variable u (start 1[y = 0]) regressed on X / sd and the
// fixed effects, until the prediction xbd = u - e is non-negative on the boundary (y = 0) or no
// boundary residual is negative; past 100 iterations it continues while the negative predictions
// keep shrinking (1% over 10 iterations), up to 2000. The regressors absorbed by the fixed
// effects or collinear with the others (the first solve's Gram, ols.rs:38-46 rules) are left out.
// The absorber's weights return to the session's afterwards.
void GpuSession::relu_separation(double* rows_in, bool on_device, size_t nx, const ReluSpec& rs, ReluOut& out) {
    AllocScope alloc_scope(ab_->stream());
    if (!wk_.empty()) throw Error(RC_INVALID_INPUT, "fereg relu: weighted sessions are not supported");
    if (1 + nx + 1 > size_t(OP_MAXM)) throw Error(RC_INVALID_INPUT, "fereg relu: at most 62 regressors");
    SessionDev& d = *d_;
    const cudaStream_t st = d.st;
    const size_t n = n_, r = 1 + nx, k = nx;
    const int R = int(r);
    const int blocks = int(std::min<size_t>((n + 255) / 256, 148 * 16));
    constexpr double RELU_TOL = 1e-4, RELU_ZERO_TOL = 1e-8, RELU_STALL = 0.99;
    constexpr size_t RELU_MAXITER = 100, RELU_HARD_MAXITER = 2000, RELU_STALL_SPAN = 10;
    const double regtol = std::max(RELU_TOL * RELU_TOL, 1e-13);
    const double big_m = std::ceil(std::pow(std::numeric_limits<double>::epsilon(), -0.5));
    DBuf<double> raw, xs, w, u, B, resid, xbd, part, bdev;
    DBuf<int> kdev;
    raw.alloc(n * r);
    CK(cudaMemcpyAsync(raw.p, rows_in, n * r * 8, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
    xs.alloc(std::max<size_t>(1, n * k));
    w.alloc(n);
    u.alloc(n);
    B.alloc(n * r);
    resid.alloc(n);
    xbd.alloc(n);
    part.alloc(size_t(blocks) * std::max<size_t>(RELU_PARTS, 2 * k));
    auto parts = [&](size_t len) {
        std::vector<double> h(size_t(blocks) * len);
        CK(cudaMemcpyAsync(h.data(), part.p, h.size() * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return h;
    };
    // y must be a Poisson outcome
    DBuf<int> flag;
    flag.alloc(1);
    CK(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
    k_glm_ysum<<<blocks, GLM_TB, 0, st>>>(raw.p, n, R, 0, part.p, flag.p);
    int neg = 0;
    CK(cudaMemcpyAsync(&neg, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (neg) throw Error(RC_INVALID_INPUT, "fereg relu: the dependent variable must be nonnegative");
    // standardization: unweighted sd per regressor (stats.rs:187, floored at 1e-3)
    std::vector<double> sd(std::max<size_t>(1, k), 1.0);
    if (k) {
        k_relu_colsums<<<blocks, GLM_TB, 0, st>>>(raw.p, n, R, part.p);
        const std::vector<double> h = parts(2 * k);
        for (size_t j = 0; j < k; j++) {
            double s1 = 0.0, s2 = 0.0;
            for (int b = 0; b < blocks; b++) {
                s1 += h[size_t(b) * 2 * k + j];
                s2 += h[size_t(b) * 2 * k + k + j];
            }
            const double mean = s1 / double(n);
            const double m2 = std::max(0.0, s2 - double(n) * mean * mean);
            sd[j] = std::max(std::sqrt(m2 / (double(n) - 1.0)), 1e-3);
        }
    }
    DBuf<double> sdd;
    sdd.upload(sd, st);
    k_relu_init<<<blocks, GLM_TB, 0, st>>>(raw.p, n, R, sdd.p, big_m, xs.p, w.p, u.p, part.p);
    d.launches += 4;
    double ratio = 1.0;
    if (k) {
        const std::vector<double> h = parts(2 * k);
        double nb = 0.0, bd = 0.0;
        for (size_t j = 0; j < k; j++) {
            double a = 0.0, c = 0.0;
            for (int b = 0; b < blocks; b++) {
                a += h[size_t(b) * 2 * k + j];
                c += h[size_t(b) * 2 * k + k + j];
            }
            nb = std::max(nb, a);
            bd = std::max(bd, c);
        }
        ratio = nb / bd;
        ratio = std::isfinite(ratio) ? std::max(ratio, 1.0) : 1.0;
    }
    ab_->set_weights_device(w.p);
    std::vector<int> all(r);
    std::iota(all.begin(), all.end(), 0);
    std::vector<double> sumsq;
    std::vector<size_t> kept;
    bool found = false, first = true;
    u64 num_sep = 0, pcg = 0;
    size_t iter = 0;
    std::vector<double> hist;
    for (;;) {
        iter++;
        ab_->ctx().check();
        k_relu_block<<<blocks, GLM_TB, 0, st>>>(u.p, xs.p, n, R, B.p, part.p);
        d.launches++;
        double uu = 0.0;
        for (double v : parts(1)) uu += v;
        if (first && k) {
            // the regressors' sums of squares before the solve (the collinearity reference)
            outer_products(B.p, n, R, all, nullptr, false, nullptr, nullptr, true, &sumsq);
        }
        const SolveInfo si = first ? ab_->residualize_device(B.p, r, regtol, rs.inner_maxiter, false, nullptr, nullptr, rs.prec)
                                   : ab_->residualize_device_warm_last(B.p, r, regtol, rs.inner_maxiter, rs.prec);
        pcg += si.iterations;
        std::vector<double> b;
        if (k) {
            std::vector<double> ss_res;
            const std::vector<double> G = outer_products(B.p, n, R, all, nullptr, false, w.p, nullptr, true, &ss_res);
            if (first) {
                const double ctol = std::min(1e-6, rs.itol / 10.0);  // glm/mod.rs:7-8
                std::vector<size_t> cand;
                for (size_t j = 1; j < r; j++)
                    if (!(ss_res[j] / sumsq[j] <= ctol)) cand.push_back(j);
                const size_t kc = cand.size();
                la::Mat gc(kc * kc);
                for (size_t a = 0; a < kc; a++)
                    for (size_t c = 0; c < kc; c++) gc[a * kc + c] = G[cand[a] * r + cand[c]];
                std::vector<bool> dropped;
                la::sweep_inverse(gc, kc, SWEEP_TOL, false, dropped);
                for (size_t c = 0; c < kc; c++)
                    if (!dropped[c]) kept.push_back(cand[c]);
                out.dropped_collinear = int(k - kept.size());
            }
            const size_t kk = kept.size();
            la::Mat gk(kk * kk);
            for (size_t a = 0; a < kk; a++)
                for (size_t c = 0; c < kk; c++) gk[a * kk + c] = G[kept[a] * r + kept[c]];
            std::vector<bool> dk;
            const la::Mat inv = la::sweep_inverse(gk, kk, SWEEP_TOL, false, dk);
            b.assign(kk, 0.0);
            for (size_t a = 0; a < kk; a++)
                for (size_t c = 0; c < kk; c++) b[a] += inv[a * kk + c] * G[kept[c] * r];
        }
        first = false;
        const int nk = int(b.size());
        bdev.upload(b.empty() ? std::vector<double>{0.0} : b, st);
        std::vector<int> kc(kept.begin(), kept.end());
        kdev.upload(kc.empty() ? std::vector<int>{0} : kc, st);
        // solve_lse's implied tolerance (ppmlhdfe_functions.mata, maxiter = 0)
        const double epsilon = std::max(uu / big_m * ratio * ratio, 1e-8);
        const double delta = epsilon + RELU_TOL;
        k_relu_step<<<blocks, GLM_TB, 0, st>>>(raw.p, B.p, u.p, n, R, R, bdev.p, kdev.p, nk, delta, RELU_ZERO_TOL,
                                                 resid.p, xbd.p, part.p);
        d.launches++;
        const std::vector<double> h = parts(RELU_PARTS);
        double cneg = 0.0, cpos = 0.0, mn = INFINITY, negsum = 0.0;
        for (int c = 0; c < blocks; c++) {
            cneg += h[size_t(c) * RELU_PARTS];
            cpos += h[size_t(c) * RELU_PARTS + 1];
            mn = std::min(mn, h[size_t(c) * RELU_PARTS + 2]);
            negsum += h[size_t(c) * RELU_PARTS + 3];
        }
        if (cneg == 0.0) {  // the prediction is non-negative on the boundary
            num_sep = u64(cpos);
            found = true;
            break;
        }
        if (mn >= 0.0) {  // no negative boundary residual
            k_relu_trim<<<blocks, GLM_TB, 0, st>>>(raw.p, n, R, resid.p, delta, xbd.p, part.p);
            d.launches++;
            double c2 = 0.0;
            for (double v : parts(1)) c2 += v;
            num_sep = u64(c2);
            found = true;
            break;
        }
        hist.push_back(negsum);
        const size_t hn = hist.size();
        const bool stalled = hn > RELU_STALL_SPAN && hist[hn - 1] > RELU_STALL * hist[hn - 1 - RELU_STALL_SPAN];
        if (iter >= RELU_MAXITER && (stalled || iter >= RELU_HARD_MAXITER)) break;
        k_relu_update<<<blocks, 256, 0, st>>>(raw.p, n, R, xbd.p, u.p);
        d.launches++;
    }
    ab_->set_weights(nullptr);
    out.iterations = iter;
    out.pcg_iterations = pcg;
    out.complete = found;
    out.num_separated = found ? num_sep : 0;
    DBuf<uint8_t> sep;
    DBuf<double> cert;
    sep.alloc(n);
    cert.alloc(n);
    if (found && num_sep > 0) {
        k_relu_out<<<blocks, 256, 0, st>>>(raw.p, n, R, xbd.p, sep.p, cert.p);
        d.launches++;
    } else {
        CK(cudaMemsetAsync(sep.p, 0, n, st));
        CK(cudaMemsetAsync(cert.p, 0, n * 8, st));
    }
    if (out.separated) CK(cudaMemcpyAsync(out.separated, sep.p, n, cudaMemcpyDeviceToHost, st));
    if (out.certificate) CK(cudaMemcpyAsync(out.certificate, cert.p, n * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
}

// crv3.rs:84-426 for OLS on the device: beta_(-g) for every cluster g of every subset of the
// cluster dimensions. Closed form when every FE term is nested in the subset's clusters (leaving g
// out removes whole FE levels, so the residualized block restricted to the other rows is theirs):
// the weighted Gram of all rows minus g's own (k_cluster_grams). Otherwise a refit: the rows
// outside g with their FE levels renumbered, a device absorber built on them, the raw [y, x]
// residualized and its Gram. Each solve is fixest's collinearity rule (vcov.rs:124 chol_collin,
// tol 1e-9; a coefficient it removes is an error). With a reported constant every refit gets the
// regression-through-the-means constant of its sample (ols/stata_vce.rs:572-600, raw weights).
// The meat is sum_S sign_S sum_g (theta_(-g) - theta)(theta_(-g) - theta)'.
std::vector<double> GpuSession::crv3_meat(const double* rows, const std::vector<double>& raw_h, int R,
                                          const std::vector<size_t>& kept, const std::vector<double>& beta,
                                          const std::vector<double>& wmean, bool report_constant,
                                          const std::vector<double>& g) {
    constexpr double COLLIN_TOL = 1e-9;  // fit/mod.rs:325
    SessionDev& d = *d_;
    const cudaStream_t st = d.st;
    const size_t n = n_, r = size_t(R), k = kept.size(), k1 = 1 + k;
    const std::vector<u32>& pi = ab_->row_order();
    const size_t kt = k + (report_constant ? 1 : 0);
    std::vector<double> theta(beta.begin(), beta.end());
    if (report_constant) {
        double b0 = wmean[0];
        for (size_t a = 0; a < k; a++) b0 -= wmean[kept[a]] * beta[a];
        theta.push_back(b0);
    }
    std::vector<int> cols(k1, 0);
    for (size_t a = 0; a < k; a++) cols[1 + a] = int(kept[a]);
    std::vector<double> wr(n, 1.0);  // raw weights, row order
    if (!wk_.empty())
        for (size_t i = 0; i < n; i++) wr[i] = wk_[pi[i]];
    const double* wv = wk_.empty() ? nullptr : d.wv.p;
    // beta from the Gram C of [y, x] (k1 x k1)
    auto solve = [&](const std::vector<double>& C, u32 cluster) {
        la::Mat cxx(k * k);
        for (size_t a = 0; a < k; a++)
            for (size_t b = 0; b < k; b++) cxx[a * k + b] = C[(1 + a) * k1 + 1 + b];
        std::vector<bool> excl;
        const la::Mat inv = la::chol_collin(cxx, k, COLLIN_TOL, excl);
        for (size_t a = 0; a < k; a++)
            if (excl[a]) {
                std::ostringstream os;
                os << "CRV3: regressor " << a << " is not estimable without cluster " << cluster;
                throw Error(RC_INVALID_INPUT, os.str());
            }
        std::vector<double> b(k, 0.0);
        for (size_t a = 0; a < k; a++)
            for (size_t c = 0; c < k; c++) b[a] += inv[a * k + c] * C[(1 + c) * k1];
        return b;
    };
    std::vector<double> meat(kt * kt, 0.0);
    DBuf<int> dcol;
    dcol.upload(cols, st);
    for (auto& sub : d.subsets) {
        const u32 G = sub.G;
        std::vector<u32> cl(n);  // cluster of every row (row order)
        for (size_t i = 0; i < n; i++) cl[i] = sub.kc[pi[i]];
        bool nested_all = true;
        for (size_t q = 0; q < tcodes_.size() && nested_all; q++) {
            std::vector<u32> map(tg_[q], UINT32_MAX);
            for (size_t i = 0; i < n && nested_all; i++) {
                u32& m = map[tcodes_[q][i]];
                if (m == UINT32_MAX) m = sub.kc[i];
                else nested_all = m == sub.kc[i];
            }
        }
        std::vector<double> betas(size_t(G) * k);
        if (nested_all) {
            d.cgram.alloc(std::max<size_t>(1, size_t(G) * k1 * k1));
            k_cluster_grams<<<std::min<u32>(G, 148 * 8), 128, 0, st>>>(rows, R, dcol.p, int(k1), wv, sub.perm.p,
                                                                      sub.coff.p, G, d.cgram.p);
            d.launches++;
            std::vector<double> cg(size_t(G) * k1 * k1);
            CK(cudaMemcpyAsync(cg.data(), d.cgram.p, cg.size() * 8, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            CK(cudaGetLastError());
            std::vector<double> C(k1 * k1);
            for (u32 gg = 0; gg < G; gg++) {
                for (size_t a = 0; a < k1; a++)
                    for (size_t b = 0; b < k1; b++)
                        C[a * k1 + b] = g[size_t(cols[a]) * r + size_t(cols[b])] - cg[(size_t(gg) * k1 + a) * k1 + b];
                const std::vector<double> b = solve(C, gg);
                std::copy(b.begin(), b.end(), betas.begin() + size_t(gg) * k);
            }
        } else {
            for (u32 gg = 0; gg < G; gg++) {
                ab_->ctx().check();
                std::vector<u32> idx;  // rows (row order) of the leave-out sample
                for (size_t i = 0; i < n; i++)
                    if (cl[i] != gg) idx.push_back(u32(i));
                const size_t m = idx.size();
                std::vector<std::vector<u32>> sc(tcodes_.size());
                std::vector<const u32*> sp;
                std::vector<u32> sg;
                for (size_t q = 0; q < tcodes_.size(); q++) {
                    std::vector<u32> map(tg_[q], UINT32_MAX);
                    for (u32 i : idx) map[tcodes_[q][pi[i]]] = 0;
                    u32 next = 0;
                    for (auto& v : map)
                        if (v == 0) v = next++;
                    sc[q].resize(m);
                    for (size_t j = 0; j < m; j++) sc[q][j] = map[tcodes_[q][pi[idx[j]]]];
                    sp.push_back(sc[q].data());
                    sg.push_back(next);
                }
                std::vector<double> ws;
                if (!wk_.empty()) {
                    ws.resize(m);
                    for (size_t j = 0; j < m; j++) ws[j] = wk_[pi[idx[j]]];
                }
                GpuAbsorber sab(sp, sg, ws.empty() ? nullptr : ws.data(), m, ab_->ctx());
                const std::vector<u32>& spi = sab.row_order();
                std::vector<u32> gidx(m);
                for (size_t t = 0; t < m; t++) gidx[t] = idx[spi[t]];
                DBuf<u32> didx;
                didx.upload(gidx, st);
                d.jk.alloc(m * k1);
                // the raw rows of the sample, from the host copy
                std::vector<double> blk(m * k1);
                for (size_t t = 0; t < m; t++)
                    for (size_t a = 0; a < k1; a++) blk[t * k1 + a] = raw_h[size_t(gidx[t]) * r + size_t(cols[a])];
                CK(cudaMemcpyAsync(d.jk.p, blk.data(), blk.size() * 8, cudaMemcpyHostToDevice, st));
                CK(cudaStreamSynchronize(st));
                sab.residualize_device(d.jk.p, k1, 1e-14, 100000, false, nullptr, nullptr);
                DBuf<double> wsub;
                if (!ws.empty()) {
                    std::vector<double> wsr(m);
                    for (size_t t = 0; t < m; t++) wsr[t] = ws[spi[t]];
                    wsub.upload(wsr, st);
                }
                std::vector<int> all(k1);
                std::iota(all.begin(), all.end(), 0);
                const std::vector<double> C =
                    outer_products(d.jk.p, m, int(k1), all, nullptr, false, ws.empty() ? nullptr : wsub.p, nullptr,
                                   false, nullptr);
                const std::vector<double> b = solve(C, gg);
                std::copy(b.begin(), b.end(), betas.begin() + size_t(gg) * k);
            }
        }
        // per-cluster raw sums for the refits' constants
        std::vector<double> cs(size_t(G) * (1 + k1), 0.0), tot(1 + k1, 0.0);
        for (size_t i = 0; i < n; i++) {
            double* row = &cs[size_t(cl[i]) * (1 + k1)];
            row[0] += wr[i];
            for (size_t a = 0; a < k1; a++) row[1 + a] += wr[i] * raw_h[i * r + size_t(cols[a])];
        }
        for (u32 gg = 0; gg < G; gg++)
            for (size_t a = 0; a <= k1; a++) tot[a] += cs[size_t(gg) * (1 + k1) + a];
        std::vector<double> dv(kt);
        for (u32 gg = 0; gg < G; gg++) {
            const double* b = &betas[size_t(gg) * k];
            for (size_t a = 0; a < k; a++) dv[a] = b[a] - theta[a];
            if (report_constant) {
                const double* row = &cs[size_t(gg) * (1 + k1)];
                const double sw = tot[0] - row[0];
                double b0 = (tot[1] - row[1]) / sw;
                for (size_t a = 0; a < k; a++) b0 -= b[a] * (tot[2 + a] - row[2 + a]) / sw;
                dv[k] = b0 - theta[k];
            }
            for (size_t a = 0; a < kt; a++)
                for (size_t c = 0; c < kt; c++) meat[a * kt + c] += sub.sign * dv[a] * dv[c];
        }
    }
    return meat;
}

}  // namespace fereg
