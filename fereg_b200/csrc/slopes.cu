// GpuSlopeSolver (slopes.h): host structure and weight state, the device passes (slopes.cuh)
// and the solve (slopes.rs:2338-2433 residualize) on the PcgDriver loop.
#include "slopes.h"

#include <algorithm>
#include <cmath>
#include <numeric>

#include "device.cuh"
#include "pcg_driver.h"
#include "slopes.cuh"

namespace fereg {

namespace {

constexpr double LEVEL_TOL = 1e-12;   // slopes.rs:57 per-level generalized inverses of E
constexpr double JACOBI_TOL = 1e-10;  // slopes.rs:59 block-Jacobi inverses
constexpr double REDUNDANT = 1e-12;   // operator.rs:21
constexpr size_t SMALL_LIMIT_S = 4096;  // structure.rs:23
// slopes.rs:62-78: the small-set cost model (seconds on the reference's machine)
constexpr double C_ROW = 1e-9, C_SMALL_ASM = 1e-9, C_FLOP = 1.2e-11, SMALL_FLOOR = 1e-3, SMALL_ITERS = 8.0;

int sl_grid(size_t work) {
    return int(std::max<size_t>(1, std::min<size_t>((work + SL_TB - 1) / SL_TB, 148 * 8)));
}

// slopes.rs:347-352 small_cost.
double small_cost(const std::vector<u32>& seg_off, size_t ms, size_t bs) {
    const u64 n = seg_off.back();
    u64 work = 0;
    for (size_t s = 0; s + 1 < seg_off.size(); s++) {
        const u64 v = std::min<u64>(u64(seg_off[s + 1] - seg_off[s]) * bs, ms);
        work += v * v;
    }
    work += n * u64(bs * bs);
    return C_SMALL_ASM * double(work) + C_FLOP * std::pow(double(ms), 3) / 3.0;
}

// cmc += C' M^+ C for C (be x b) and M^+ (be x be) (slopes.rs:699-714).
void add_cmc(const double* c, const double* mv, size_t be, size_t b, double* cmc) {
    for (size_t a = 0; a < b; a++)
        for (size_t bb = 0; bb < b; bb++) {
            double acc = 0.0;
            for (size_t l = 0; l < be; l++) {
                double t = 0.0;
                for (size_t l2 = 0; l2 < be; l2++) t += mv[l * be + l2] * c[l2 * b + bb];
                acc += c[l * b + a] * t;
            }
            cmc[a * b + bb] += acc;
        }
}

}  // namespace

void sweep_ginv(double* a, size_t k, const double* refd, double tol) {
    for (size_t p = 0; p < k; p++) {
        const double d = a[p * k + p];
        if (!(d > tol * refd[p] && d > 0.0 && std::isfinite(d))) {
            for (size_t j = 0; j < k; j++) a[p * k + j] = a[j * k + p] = 0.0;
            continue;
        }
        const double inv = 1.0 / d;
        for (size_t j = 0; j < k; j++) a[p * k + j] *= inv;
        for (size_t i = 0; i < k; i++) {
            if (i == p) continue;
            const double c = a[i * k + p];
            if (c == 0.0) continue;
            for (size_t j = 0; j < k; j++) a[i * k + j] -= c * a[p * k + j];
            a[i * k + p] = -c * inv;
        }
        a[p * k + p] = inv;
    }
}

SlopeHost build_slope_structure(const std::vector<SlopeTermIn>& terms, size_t n) {
    if (terms.empty()) throw Error(RC_INTERNAL, "slopes: no absorb terms");
    for (const auto& t : terms) {
        if (!t.intercept && t.slopes.empty()) throw Error(RC_INVALID_INPUT, "absorb term without intercept or slopes");
        if (!t.codes || t.g == 0) throw Error(RC_INVALID_INPUT, "slopes: empty term");
        for (const double* x : t.slopes)
            if (!x) throw Error(RC_INVALID_INPUT, "slopes: missing slope variable");
    }
    if (n > size_t(UINT32_MAX)) throw Error(RC_INVALID_INPUT, "slopes: too many rows");
    for (const auto& t : terms)
        for (size_t i = 0; i < n; i++)
            if (t.codes[i] >= t.g) throw Error(RC_INVALID_INPUT, "term code out of range of its level count");
    SlopeHost h;
    h.n = n;
    // E: the intercept-only term with the most levels (absorber.rs:100 fe1_index), else the term
    // with the most levels (first of equals)
    int e = -1;
    for (size_t q = 0; q < terms.size(); q++)
        if (terms[q].intercept && terms[q].slopes.empty() && (e < 0 || terms[q].g > terms[size_t(e)].g)) e = int(q);
    if (e < 0) {
        e = 0;
        for (size_t q = 0; q < terms.size(); q++)
            if (terms[q].g > terms[size_t(e)].g) e = int(q);
    }
    h.e = size_t(e);
    const SlopeTermIn& te = terms[h.e];
    h.ge = te.g;
    h.e_icpt = te.intercept;
    h.e_ns = u32(te.slopes.size());
    h.be = u32(te.intercept ? 1 : 0) + h.e_ns;
    if (h.be > u32(SL_BE_MAX)) throw Error(RC_INVALID_INPUT, "slopes: at most 8 design columns in the eliminated term");

    // rows sorted stably by the level of E (counting sort: ids ascend within each level)
    h.seg_off.assign(size_t(h.ge) + 1, 0);
    for (size_t i = 0; i < n; i++) h.seg_off[size_t(te.codes[i]) + 1]++;
    for (size_t s = 0; s < h.ge; s++) h.seg_off[s + 1] += h.seg_off[s];
    h.pi.resize(n);
    {
        std::vector<u32> pos(h.seg_off.begin(), h.seg_off.end() - 1);
        for (size_t i = 0; i < n; i++) h.pi[pos[te.codes[i]]++] = u32(i);
    }

    // blocks: the small set first (slopes.rs:412-438), then the large ones, each in term order
    std::vector<size_t> others;
    for (size_t q = 0; q < terms.size(); q++)
        if (q != h.e) others.push_back(q);
    auto width = [&](size_t q) { return size_t(terms[q].intercept ? 1 : 0) + terms[q].slopes.size(); };
    size_t slots = h.be;
    for (size_t q : others) slots += width(q);
    const double matvec = C_ROW * double(n) * double(slots + 2);
    std::vector<size_t> by_size = others;
    std::stable_sort(by_size.begin(), by_size.end(), [&](size_t a, size_t b) {
        const size_t ca = size_t(terms[a].g) * width(a), cb = size_t(terms[b].g) * width(b);
        return ca != cb ? ca < cb : a < b;
    });
    std::vector<bool> small(terms.size(), false);
    size_t total = 0, bs = 0;
    for (size_t q : by_size) {
        const size_t c = size_t(terms[q].g) * width(q);
        if (total + c > SMALL_LIMIT_S ||
            small_cost(h.seg_off, total + c, bs + width(q)) > std::max(SMALL_FLOOR, SMALL_ITERS * matvec))
            break;
        total += c;
        bs += width(q);
        small[q] = true;
    }
    std::vector<size_t> order;
    for (size_t q : others)
        if (small[q]) order.push_back(q);
    h.nsmall = u32(order.size());
    for (size_t q : others)
        if (!small[q]) order.push_back(q);
    size_t off = 0, s0 = 0;
    for (size_t q : order) {
        SlopeBlock b;
        b.term = q;
        b.g = terms[q].g;
        b.icpt = terms[q].intercept;
        b.ns = u32(terms[q].slopes.size());
        b.b = u32(width(q));
        if (b.b > u32(SL_B_MAX)) throw Error(RC_INVALID_INPUT, "slopes: at most 8 design columns per absorb term");
        b.s0 = u32(s0);
        b.off = u32(off);
        b.small = small[q];
        h.blocks.push_back(b);
        off += size_t(b.g) * b.b;
        s0 += b.b;
        if (off > size_t(UINT32_MAX)) throw Error(RC_INVALID_INPUT, "too many fixed-effect coefficients");
    }
    h.m = u32(off);
    h.k = u32(s0);
    for (u32 q = 0; q < h.nsmall; q++) h.m_small += h.blocks[q].g * h.blocks[q].b;

    // slot coordinates and values, E's slopes, in row order
    h.sc.resize(n * h.k);
    h.sv.resize(n * h.k);
    h.he.resize(n * h.e_ns);
#pragma omp parallel for schedule(static)
    for (long long ii = 0; ii < (long long)n; ii++) {
        const size_t i = size_t(ii), o = h.pi[i];
        for (const SlopeBlock& b : h.blocks) {
            const SlopeTermIn& t = terms[b.term];
            const u32 c0 = b.off + t.codes[o] * b.b;
            for (u32 d = 0; d < b.b; d++) h.sc[i * h.k + b.s0 + d] = c0 + d;
            const u32 first = b.s0 + (b.icpt ? 1u : 0u);
            if (b.icpt) h.sv[i * h.k + b.s0] = 1.0;
            for (u32 s = 0; s < b.ns; s++) h.sv[i * h.k + first + s] = t.slopes[s][o];
        }
        for (u32 s = 0; s < h.e_ns; s++) h.he[i * h.e_ns + s] = te.slopes[s][o];
    }

    // coordinate-sorted slot lists: entries of a coordinate in row order
    h.pl_off.assign(size_t(h.m) + 1, 0);
    for (size_t e2 = 0; e2 < n * h.k; e2++) h.pl_off[size_t(h.sc[e2]) + 1]++;
    for (size_t c = 0; c < h.m; c++) h.pl_off[c + 1] += h.pl_off[c];
    h.pl_row.resize(n * h.k);
    h.pl_val.resize(n * h.k);
    {
        std::vector<u32> pos(h.pl_off.begin(), h.pl_off.end() - 1);
        for (size_t i = 0; i < n; i++)
            for (u32 t = 0; t < h.k; t++) {
                const size_t e2 = i * h.k + t;
                const u32 at = pos[h.sc[e2]]++;
                h.pl_row[at] = u32(i);
                h.pl_val[at] = h.sv[e2];
            }
    }
    // block-Jacobi units: one per (block, level)
    u32 jo = 0;
    for (const SlopeBlock& b : h.blocks)
        for (u32 l = 0; l < b.g; l++) {
            h.un_c0.push_back(b.off + l * b.b);
            h.un_b.push_back(b.b);
            h.un_joff.push_back(jo);
            jo += b.b * b.b;
        }
    h.jlen = jo;
    return h;
}

struct SlopeDevBufs {
    DBuf<u32> seg_off, sc, pl_off, pl_row, un_c0, un_b, un_joff;
    DBuf<double> sv, he, pl_val, w, minv, jinv;
    DBuf<double> Z, rhs, x, part, stats, coefs, zbuf, pin, pout;
    PcgDriver pcg;
    u64 launches = 0;
    SlopeDev dev(const SlopeHost& h, bool weighted) const {
        return SlopeDev{u32(h.n), h.ge,     h.k,  h.m, h.be, h.e_ns, h.e_icpt ? 1 : 0,
                        seg_off.p, sc.p, sv.p, he.p, weighted ? w.p : nullptr, minv.p};
    }
};

namespace {

// The slope operator seen by PcgDriver: S p by the segment and coordinate passes, z = J r.
struct SlopeOp final : DevOperator {
    const SlopeHost& h;
    SlopeDevBufs& d;
    SlopeDev D;
    SlopeOp(const SlopeHost& h_, SlopeDevBufs& d_, const SlopeDev& D_) : h(h_), d(d_), D(D_) {}
    u32 m() const override { return h.m; }
    void apply(double* p, int R, double* q, cudaStream_t st) override {
        d.Z.alloc(std::max<size_t>(1, h.n * size_t(R)));
        k_sl_seg<SL_APPLY><<<sl_grid(size_t(h.ge) * R), SL_TB, 0, st>>>(D, p, R, R, nullptr, 0, d.Z.p, R, nullptr,
                                                                        nullptr, 0, nullptr);
        k_sl_pull<<<sl_grid(size_t(h.m) * R), SL_TB, 0, st>>>(h.m, R, d.pl_off.p, d.pl_row.p, d.pl_val.p, d.Z.p, R, q,
                                                               R);
        d.launches += 2;
    }
    void precond(double* r, double* z, int R, cudaStream_t st) override {
        const u32 nu = u32(h.un_c0.size());
        k_sl_jacobi<<<sl_grid(size_t(nu) * R), SL_TB, 0, st>>>(nu, R, d.un_c0.p, d.un_b.p, d.un_joff.p, d.jinv.p, r, z,
                                                                R);
        d.launches++;
    }
    void key(std::vector<u64>& k) const override {
        for (const void* ptr : {(const void*)d.Z.p, (const void*)d.seg_off.p, (const void*)d.sc.p, (const void*)d.sv.p,
                                (const void*)d.he.p, (const void*)D.w, (const void*)d.minv.p, (const void*)d.pl_off.p,
                                (const void*)d.pl_row.p, (const void*)d.pl_val.p, (const void*)d.jinv.p})
            k.push_back(u64(reinterpret_cast<uintptr_t>(ptr)));
    }
};

}  // namespace

GpuSlopeSolver::GpuSlopeSolver(const std::vector<SlopeTermIn>& terms, const double* w, size_t n, const Ctx& ctx)
    : ctx_(ctx) {
    if (w) check_weights_host(w, n);
    hs_ = build_slope_structure(terms, n);
    for (const auto& t : terms) {
        t_icpt_.push_back(t.intercept);
        t_ns_.push_back(u32(t.slopes.size()));
        t_g_.push_back(t.g);
    }
    for (size_t q = 0; q < terms.size(); q++)
        if (terms[q].intercept && terms[q].slopes.empty() && (fe1_ < 0 || terms[q].g > terms[size_t(fe1_)].g))
            fe1_ = int(q);
    ctx_.check();
    keep_pool_mapped();
    CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    AllocScope alloc_scope(stream_);
    d_ = std::make_unique<SlopeDevBufs>();
    SlopeDevBufs& d = *d_;
    d.seg_off.upload(hs_.seg_off, stream_);
    d.sc.upload(hs_.sc, stream_);
    d.sv.upload(hs_.sv, stream_);
    d.he.upload(hs_.he, stream_);
    d.pl_off.upload(hs_.pl_off, stream_);
    d.pl_row.upload(hs_.pl_row, stream_);
    d.pl_val.upload(hs_.pl_val, stream_);
    d.un_c0.upload(hs_.un_c0, stream_);
    d.un_b.upload(hs_.un_b, stream_);
    d.un_joff.upload(hs_.un_joff, stream_);
    if (w) {
        w_rows_.resize(n);
        for (size_t i = 0; i < n; i++) w_rows_[i] = w[hs_.pi[i]];
    }
    refresh_weights();
    CK(cudaStreamSynchronize(stream_));
}

GpuSlopeSolver::~GpuSlopeSolver() {
    if (stream_) {
        cudaStreamSynchronize(stream_);
        {
            AllocScope alloc_scope(stream_);
            d_.reset();
        }
        cudaStreamSynchronize(stream_);
        cudaStreamDestroy(stream_);
    }
}

// slopes.rs:553-697: M_s^+ per level of E, the diagonal blocks of S per level of every other
// block, their redundant coordinates and block-Jacobi inverses. Sums run in row order.
void GpuSlopeSolver::refresh_weights() {
    const SlopeHost& h = hs_;
    const size_t n = h.n, be = h.be, be2 = be * be, ns = h.e_ns;
    const bool weighted = !w_rows_.empty();
    auto w = [&](size_t i) { return weighted ? w_rows_[i] : 1.0; };
    sw_ = 0.0;
    for (size_t i = 0; i < n; i++) sw_ += w(i);
    minv_.assign(size_t(h.ge) * be2, 0.0);
#pragma omp parallel for schedule(dynamic, 256)
    for (long long ss = 0; ss < (long long)h.ge; ss++) {
        const size_t s = size_t(ss), r0 = h.seg_off[s], r1 = h.seg_off[s + 1];
        double* out = &minv_[s * be2];
        if (h.e_icpt && be == 1) {
            double sw = 0.0;
            for (size_t i = r0; i < r1; i++) sw += w(i);
            out[0] = 1.0 / sw;
            continue;
        }
        std::vector<double> g(ns * ns, 0.0), xbar(ns, 0.0), refd(ns, 0.0);
        if (h.e_icpt) {
            double sw = 0.0;
            for (size_t i = r0; i < r1; i++) {
                const double wi = w(i);
                sw += wi;
                for (size_t k = 0; k < ns; k++) {
                    const double x = h.he[i * ns + k];
                    xbar[k] += wi * x;
                    refd[k] += wi * x * x;
                }
            }
            for (auto& v : xbar) v /= sw;
            for (size_t i = r0; i < r1; i++) {
                const double wi = w(i);
                for (size_t k = 0; k < ns; k++) {
                    const double dk = wi * (h.he[i * ns + k] - xbar[k]);
                    for (size_t l = 0; l <= k; l++) g[k * ns + l] += dk * (h.he[i * ns + l] - xbar[l]);
                }
            }
            for (size_t k = 0; k < ns; k++)
                for (size_t l = 0; l < k; l++) g[l * ns + k] = g[k * ns + l];
            sweep_ginv(g.data(), ns, refd.data(), LEVEL_TOL);
            std::vector<double> gx(ns, 0.0);
            for (size_t k = 0; k < ns; k++)
                for (size_t l = 0; l < ns; l++) gx[k] += g[k * ns + l] * xbar[l];
            double q0 = 1.0 / sw;
            for (size_t k = 0; k < ns; k++) q0 += xbar[k] * gx[k];
            out[0] = q0;
            for (size_t k = 0; k < ns; k++) {
                out[1 + k] = -gx[k];
                out[(1 + k) * be] = -gx[k];
                for (size_t l = 0; l < ns; l++) out[(1 + k) * be + 1 + l] = g[k * ns + l];
            }
        } else {
            for (size_t i = r0; i < r1; i++) {
                const double wi = w(i);
                for (size_t k = 0; k < ns; k++)
                    for (size_t l = 0; l <= k; l++) g[k * ns + l] += wi * h.he[i * ns + k] * h.he[i * ns + l];
            }
            for (size_t k = 0; k < ns; k++) {
                refd[k] = g[k * ns + k];
                for (size_t l = 0; l < k; l++) g[l * ns + k] = g[k * ns + l];
            }
            sweep_ginv(g.data(), ns, refd.data(), LEVEL_TOL);
            std::copy(g.begin(), g.end(), out);
        }
    }
    // diagonal blocks: gram_l = sum w h h' over the rows of level l, cmc_l = sum_s C_sl' M_s^+ C_sl
    // with C_sl = sum over the rows of segment s at level l of w h_E h'
    jinv_.assign(h.jlen, 0.0);
    red_.assign(h.m, 0);
    for (size_t q = 0; q < h.blocks.size(); q++) {
        const SlopeBlock& blk = h.blocks[q];
        const size_t b = blk.b, b2 = b * b;
        std::vector<double> gram(size_t(blk.g) * b2, 0.0), cmc(size_t(blk.g) * b2, 0.0);
        std::vector<std::pair<u32, u32>> items;
        std::vector<double> c(be * b), hev(be);
        for (size_t s = 0; s < h.ge; s++) {
            items.clear();
            for (u32 i = h.seg_off[s]; i < h.seg_off[s + 1]; i++) items.emplace_back(h.sc[size_t(i) * h.k + blk.s0], i);
            std::sort(items.begin(), items.end());
            const double* mv = &minv_[s * be2];
            size_t kk = 0;
            while (kk < items.size()) {
                const u32 c0 = items[kk].first;
                const size_t gb2 = size_t(c0 - blk.off) * b;  // level x b^2
                std::fill(c.begin(), c.end(), 0.0);
                double* gl = &gram[gb2];
                while (kk < items.size() && items[kk].first == c0) {
                    const size_t i = items[kk].second;
                    const double wi = w(i);
                    const double* hq = &h.sv[i * h.k + blk.s0];
                    for (size_t a = 0; a < b; a++)
                        for (size_t bb = 0; bb < b; bb++) gl[a * b + bb] += wi * hq[a] * hq[bb];
                    for (size_t l = 0; l < be; l++) {
                        hev[l] = h.e_icpt ? (l == 0 ? 1.0 : h.he[i * ns + l - 1]) : h.he[i * ns + l];
                        for (size_t a = 0; a < b; a++) c[l * b + a] += wi * hev[l] * hq[a];
                    }
                    kk++;
                }
                add_cmc(c.data(), mv, be, b, &cmc[gb2]);
            }
        }
        for (u32 l = 0; l < blk.g; l++) {
            double* dl = &cmc[size_t(l) * b2];
            const double* gl = &gram[size_t(l) * b2];
            for (size_t t = 0; t < b2; t++) dl[t] = gl[t] - dl[t];
            std::vector<double> jl(dl, dl + b2), refd(b);
            std::vector<uint8_t> rl(b);
            for (size_t a = 0; a < b; a++) rl[a] = !(dl[a * b + a] > REDUNDANT * gl[a * b + a]);
            for (size_t a = 0; a < b; a++) {
                refd[a] = dl[a * b + a];
                if (rl[a])
                    for (size_t bb = 0; bb < b; bb++) jl[a * b + bb] = jl[bb * b + a] = 0.0;
            }
            sweep_ginv(jl.data(), b, refd.data(), JACOBI_TOL);
            const size_t u = size_t(std::lower_bound(h.un_c0.begin(), h.un_c0.end(), blk.off + l * blk.b) -
                                    h.un_c0.begin());
            std::copy(jl.begin(), jl.end(), jinv_.begin() + h.un_joff[u]);
            for (size_t a = 0; a < b; a++) red_[size_t(blk.off) + size_t(l) * b + a] = rl[a];
        }
    }
    AllocScope alloc_scope(stream_);
    SlopeDevBufs& d = *d_;
    d.minv.upload(minv_, stream_);
    d.jinv.upload(jinv_, stream_);
    if (!w_rows_.empty()) d.w.upload(w_rows_, stream_);
    CK(cudaStreamSynchronize(stream_));
}

bool GpuSlopeSolver::weights(double* out) const {
    if (w_rows_.empty()) return false;
    if (out) std::copy(w_rows_.begin(), w_rows_.end(), out);
    return true;
}

void GpuSlopeSolver::set_weights(const double* w) {
    if (w) {
        check_weights_host(w, hs_.n);
        w_rows_.assign(w, w + hs_.n);
    } else {
        w_rows_.clear();
    }
    refresh_weights();
}

void GpuSlopeSolver::set_weights_device(const double* w_dev) {
    if (!w_dev) {
        set_weights(nullptr);
        return;
    }
    std::vector<double> h(hs_.n);
    CK(cudaMemcpyAsync(h.data(), w_dev, hs_.n * 8, cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    set_weights(h.data());
}

size_t GpuSlopeSolver::term_values_len() const {
    size_t t = 0;
    for (size_t q = 0; q < t_g_.size(); q++) t += size_t(t_g_[q]) * ((t_icpt_[q] ? 1 : 0) + t_ns_[q]);
    return t;
}

SolveInfo GpuSlopeSolver::residualize(double* z, size_t r, double tol, size_t maxiter, bool want_coefs,
                                      const double* warm, double* coefs, Precision) {
    AllocScope alloc_scope(stream_);
    SlopeDevBufs& d = *d_;
    d.zbuf.alloc(std::max<size_t>(1, hs_.n * r));
    if (hs_.n * r) CK(cudaMemcpyAsync(d.zbuf.p, z, hs_.n * r * 8, cudaMemcpyHostToDevice, stream_));
    const SolveInfo info = solve(d.zbuf.p, r, tol, maxiter, want_coefs, warm, coefs, false);
    if (hs_.n * r) CK(cudaMemcpyAsync(z, d.zbuf.p, hs_.n * r * 8, cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    return info;
}

SolveInfo GpuSlopeSolver::residualize_device(double* z_dev, size_t r, double tol, size_t maxiter, bool want_coefs,
                                             const double* warm, double* coefs, Precision) {
    AllocScope alloc_scope(stream_);
    return solve(z_dev, r, tol, maxiter, want_coefs, warm, coefs, false);
}

SolveInfo GpuSlopeSolver::residualize_device_warm_last(double* z_dev, size_t r, double tol, size_t maxiter,
                                                       Precision) {
    AllocScope alloc_scope(stream_);
    return solve(z_dev, r, tol, maxiter, false, nullptr, nullptr, true);
}

// slopes.rs:2338-2433: rhs with [sum w v^2, sum w v, sum w e^2], ss0 = sum w v^2 - (sum w v)^2 /
// sum w (0 below 1e-15 sum w v^2), ss1 = sum w e^2; PCG from the warm start (columns with ss0 = 0
// start at 0); then the rows lose the FE fit and E's projection, alpha_E from the last.
SolveInfo GpuSlopeSolver::solve(double* z, size_t r, double tol, size_t maxiter, bool want_coefs, const double* warm,
                                double* coefs, bool warm_last) {
    SolveInfo info;
    info.iterations = 1;
    if (r == 0) {
        wait_write_fence(stream_);
        return info;
    }
    ctx_.check();
    SlopeDevBufs& d = *d_;
    const SlopeHost& h = hs_;
    const cudaStream_t st = stream_;
    const size_t m = h.m, n = h.n, rv = (r + 3) / 4 * 4;
    const int R = int(r), RV = int(rv);
    const SlopeDev D = d.dev(h, !w_rows_.empty());
    std::vector<double> x_host;
    d.x.alloc(std::max<size_t>(1, m * rv));
    d.coefs.alloc(std::max<size_t>(1, coefs_len() * r));
    if (m > 0) {
        // right-hand side and its statistics
        d.Z.alloc(std::max<size_t>(1, n * rv));
        d.rhs.alloc(m * rv);
        d.part.alloc(std::max<size_t>(1, size_t(h.ge) * 3 * r));
        d.stats.alloc(3 * r);
        CK(cudaMemsetAsync(d.rhs.p, 0, m * rv * 8, st));
        k_sl_seg<SL_RHS><<<sl_grid(size_t(h.ge) * r), SL_TB, 0, st>>>(D, z, R, R, nullptr, 0, d.Z.p, RV, nullptr,
                                                                      nullptr, 0, d.part.p);
        k_sl_pull<<<sl_grid(m * r), SL_TB, 0, st>>>(h.m, R, d.pl_off.p, d.pl_row.p, d.pl_val.p, d.Z.p, RV, d.rhs.p, RV);
        d.launches += 2;
        d.pcg.col_sums(d.part.p, int(h.ge), 3 * R, d.stats.p, st);
        std::vector<double> ex(3 * r);
        CK(cudaMemcpyAsync(ex.data(), d.stats.p, 3 * r * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        ctx_.check();
        std::vector<double> ss0(rv, 0.0), ss1(rv, 0.0);
        for (size_t j = 0; j < r; j++) {
            const double wsq = ex[j], wsum = ex[r + j];
            const double s = wsq - wsum * wsum / sw_;
            ss0[j] = s > 1e-15 * wsq ? s : 0.0;
            ss1[j] = ex[2 * r + j];
        }
        // the start: the previous solution, the caller's, or 0; columns with ss0 = 0 at 0
        const bool have_last = warm_last && last_r_ == r;
        bool start = false;
        if (have_last) {
            start = true;  // d.x holds it
        } else if (warm) {
            std::vector<double> w0(m * rv, 0.0);
            for (size_t i = 0; i < m; i++)
                for (size_t j = 0; j < r; j++) w0[i * rv + j] = warm[i * r + j];
            CK(cudaMemcpyAsync(d.x.p, w0.data(), m * rv * 8, cudaMemcpyHostToDevice, st));
            CK(cudaStreamSynchronize(st));
            start = true;
        } else {
            CK(cudaMemsetAsync(d.x.p, 0, m * rv * 8, st));
        }
        if (start) {
            std::vector<double> xv(m * rv);
            CK(cudaMemcpyAsync(xv.data(), d.x.p, m * rv * 8, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            for (size_t j = 0; j < rv; j++)
                if (ss0[j] == 0.0)
                    for (size_t i = 0; i < m; i++) xv[i * rv + j] = 0.0;
            CK(cudaMemcpyAsync(d.x.p, xv.data(), m * rv * 8, cudaMemcpyHostToDevice, st));
            CK(cudaStreamSynchronize(st));
        }
        SlopeOp op(h, d, D);
        info.iterations = std::max<u64>(1, d.pcg.run(op, d.x.p, d.rhs.p, RV, ss0, ss1, tol, maxiter, start, ctx_, st));
        ctx_.check();
        // the unpadded solution
        CK(cudaMemcpy2DAsync(d.coefs.p, r * 8, d.x.p, rv * 8, r * 8, m, cudaMemcpyDeviceToDevice, st));
    }
    // residualization: v <- d - h_E't with d = v - u(x), alpha_E = t
    double* alpha = want_coefs ? d.coefs.p + m * r : nullptr;
    wait_write_fence(st);
    k_sl_seg<SL_RESID><<<sl_grid(size_t(h.ge) * r), SL_TB, 0, st>>>(D, z, R, R, m > 0 ? d.coefs.p : nullptr, R,
                                                                    nullptr, 0, z, alpha, R, nullptr);
    d.launches++;
    CK(cudaGetLastError());
    if (want_coefs && coefs) CK(cudaMemcpyAsync(coefs, d.coefs.p, coefs_len() * r * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    last_r_ = m > 0 ? r : 0;
    info.exact = false;
    return info;
}

// slopes.rs:1559-1580 fit_rows: per row the FE fit of coefficient column `col` (row order).
void GpuSlopeSolver::fit_rows(const double* coefs, size_t r, size_t col, double* out) const {
    const SlopeHost& h = hs_;
    const size_t be = h.be, m = h.m;
    for (size_t s = 0; s < h.ge; s++)
        for (u32 i = h.seg_off[s]; i < h.seg_off[s + 1]; i++) {
            double f = 0.0;
            for (size_t l = 0; l < be; l++) {
                const double hv = h.e_icpt ? (l == 0 ? 1.0 : h.he[size_t(i) * h.e_ns + l - 1]) : h.he[size_t(i) * h.e_ns + l];
                f += hv * coefs[(m + s * be + l) * r + col];
            }
            if (m > 0) {
                double u = 0.0;
                for (u32 t = 0; t < h.k; t++) {
                    const size_t e = size_t(i) * h.k + t;
                    u += h.sv[e] * coefs[size_t(h.sc[e]) * r + col];
                }
                f += u;
            }
            out[i] = f;
        }
}

// slopes.rs:2441-2474 term_values: per term its slot vectors (intercept, then slopes; levels in
// order); the intercepts of the intercept-only terms other than FE1 are centred at their
// weighted mean, which moves to FE1.
void GpuSlopeSolver::term_values(const double* coefs, size_t r, size_t col, double* out) const {
    const SlopeHost& h = hs_;
    const size_t nt = t_g_.size();
    std::vector<std::vector<std::vector<double>>> vals(nt);
    vals[h.e].assign(h.be, std::vector<double>(h.ge));
    for (size_t k = 0; k < h.be; k++)
        for (size_t g = 0; g < h.ge; g++) vals[h.e][k][g] = coefs[(h.m + g * h.be + k) * r + col];
    std::vector<size_t> by_term(nt, SIZE_MAX);
    for (size_t q = 0; q < h.blocks.size(); q++) {
        const SlopeBlock& b = h.blocks[q];
        by_term[b.term] = q;
        vals[b.term].assign(b.b, std::vector<double>(b.g));
        for (size_t k = 0; k < b.b; k++)
            for (size_t g = 0; g < b.g; g++) vals[b.term][k][g] = coefs[(b.off + g * b.b + k) * r + col];
    }
    if (fe1_ >= 0) {
        for (size_t tq = 0; tq < nt; tq++) {
            if (int(tq) == fe1_ || !t_icpt_[tq] || t_ns_[tq] > 0) continue;
            const SlopeBlock& b = h.blocks[by_term[tq]];
            std::vector<double> nr(t_g_[tq], 0.0);
            for (size_t i = 0; i < h.n; i++)
                nr[(h.sc[i * h.k + b.s0] - b.off) / b.b] += w_rows_.empty() ? 1.0 : w_rows_[i];
            double mean = 0.0;
            for (size_t g = 0; g < nr.size(); g++) mean += vals[tq][0][g] * nr[g];
            mean /= sw_;
            for (auto& a : vals[tq][0]) a -= mean;
            for (auto& a : vals[size_t(fe1_)][0]) a += mean;
        }
    }
    size_t o = 0;
    for (auto& t : vals)
        for (auto& v : t) {
            std::copy(v.begin(), v.end(), out + o);
            o += v.size();
        }
}

void GpuSlopeSolver::phase_times(double* ms, u64* counts) const {
    for (int i = 0; i < GpuAbsorber::P_NSLOTS; i++) {
        if (ms) ms[i] = 0.0;
        if (counts) counts[i] = 0;
    }
}

u64 GpuSlopeSolver::launches() const { return d_->launches + d_->pcg.launches(); }

void GpuSlopeSolver::solver_stats(u64* o) const { d_->pcg.stats(o); }

void GpuSlopeSolver::weight_state(double* minv, double* jinv, uint8_t* red) const {
    if (minv) std::copy(minv_.begin(), minv_.end(), minv);
    if (jinv) std::copy(jinv_.begin(), jinv_.end(), jinv);
    if (red) std::copy(red_.begin(), red_.end(), red);
}

void GpuSlopeSolver::apply_host(const double* p, size_t r, double* y) {
    AllocScope alloc_scope(stream_);
    SlopeDevBufs& d = *d_;
    const size_t m = hs_.m;
    if (m == 0 || r == 0) return;
    d.pin.alloc(m * r);
    d.pout.alloc(m * r);
    CK(cudaMemcpyAsync(d.pin.p, p, m * r * 8, cudaMemcpyHostToDevice, stream_));
    SlopeOp op(hs_, d, d.dev(hs_, !w_rows_.empty()));
    op.apply(d.pin.p, int(r), d.pout.p, stream_);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(y, d.pout.p, m * r * 8, cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
}

void GpuSlopeSolver::precond_host(const double* rr, size_t r, double* z) {
    AllocScope alloc_scope(stream_);
    SlopeDevBufs& d = *d_;
    const size_t m = hs_.m;
    if (m == 0 || r == 0) return;
    d.pin.alloc(m * r);
    d.pout.alloc(m * r);
    CK(cudaMemcpyAsync(d.pin.p, rr, m * r * 8, cudaMemcpyHostToDevice, stream_));
    SlopeOp op(hs_, d, d.dev(hs_, !w_rows_.empty()));
    op.precond(d.pin.p, d.pout.p, int(r), stream_);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(z, d.pout.p, m * r * 8, cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
}

void GpuSlopeSolver::rhs_host(const double* rows, size_t r, double* y, double* stats) {
    AllocScope alloc_scope(stream_);
    SlopeDevBufs& d = *d_;
    const SlopeHost& h = hs_;
    const size_t m = h.m, n = h.n;
    if (r == 0) return;
    const SlopeDev D = d.dev(h, !w_rows_.empty());
    d.zbuf.alloc(std::max<size_t>(1, n * r));
    d.Z.alloc(std::max<size_t>(1, n * r));
    d.rhs.alloc(std::max<size_t>(1, m * r));
    d.part.alloc(std::max<size_t>(1, size_t(h.ge) * 3 * r));
    d.stats.alloc(3 * r);
    const int R = int(r);
    CK(cudaMemcpyAsync(d.zbuf.p, rows, n * r * 8, cudaMemcpyHostToDevice, stream_));
    k_sl_seg<SL_RHS><<<sl_grid(size_t(h.ge) * r), SL_TB, 0, stream_>>>(D, d.zbuf.p, R, R, nullptr, 0, d.Z.p, R,
                                                                       nullptr, nullptr, 0, d.part.p);
    if (m) k_sl_pull<<<sl_grid(m * r), SL_TB, 0, stream_>>>(h.m, R, d.pl_off.p, d.pl_row.p, d.pl_val.p, d.Z.p, R,
                                                            d.rhs.p, R);
    d.pcg.col_sums(d.part.p, int(h.ge), 3 * R, d.stats.p, stream_);
    CK(cudaGetLastError());
    if (m) CK(cudaMemcpyAsync(y, d.rhs.p, m * r * 8, cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(stats, d.stats.p, 3 * r * 8, cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
}

}  // namespace fereg
