// TEST INFRASTRUCTURE — the CPU oracle of the fixed-effects solve.
//
// A plain FP64 C++ restatement of the reference solver (leoliu0/fereg, crate fereg-core),
// used only as the checker by tests/, __graft_entry__.smoke() and the cpu_baseline leg of
// bench.py. Nothing in the product (fereg_b200/) links or calls it.
//
// Each function cites the reference file:line it follows (paths inside the reference project).
// The floating-point summation order is not the reference's (its parallel chunking is a property
// of its thread pool); the algorithm, stopping rule, grounding and integer results are. Parity
// of this file with the reference is pinned by the reference's own reghdfe fixtures
// (crates/fereg-core/tests/data/ols_s*.json, extracted to tests/golden/ by
// tests/golden/make_golden.py) — see tests/test_oracle_fixtures.py.
//
// Parallel loops use a fixed task partition (independent of the thread count) with partial
// sums combined in task order, so results are the same at any OMP_NUM_THREADS.

#include <algorithm>
#include <array>
#include <functional>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>
#include <omp.h>

namespace orc {

using u32 = uint32_t;
using u64 = uint64_t;
using Vec = std::vector<double>;

static thread_local std::string g_err;

// ---------------------------------------------------------------------------------------------
// rng.rs:4-31 — SplitMix64 with independent streams.
struct SplitMix64 {
    u64 state;
    explicit SplitMix64(u64 seed) : state(seed) {}
    static SplitMix64 stream(u64 seed, u64 index) {
        SplitMix64 s(seed ^ (index * 0xD1B54A32D192ED03ull));
        s.next_u64();
        return s;
    }
    u64 next_u64() {
        state += 0x9E3779B97F4A7C15ull;
        u64 z = state;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double next_f64() { return double(next_u64() >> 11) * (1.0 / double(1ull << 53)); }
};

// ---------------------------------------------------------------------------------------------
// factor.rs:26-31 f64_key, :38 factorize (dense codes in ascending value order; every path of
// the reference gives this unique result), :255 combine (lexicographic order of the tuple over
// the combinations that occur), :281 restrict (renumber after drops, order preserving).
static u64 f64_key(double x) {
    if (x == 0.0) x = 0.0;
    u64 bits;
    std::memcpy(&bits, &x, 8);
    return (bits >> 63) ? ~bits : (bits | (1ull << 63));
}

static int factorize_keys(const std::vector<u64>& keys, std::vector<u32>& codes, u32& nlev) {
    std::vector<u64> uniq(keys);
    std::sort(uniq.begin(), uniq.end());
    uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
    codes.resize(keys.size());
    for (size_t i = 0; i < keys.size(); i++)
        codes[i] = u32(std::lower_bound(uniq.begin(), uniq.end(), keys[i]) - uniq.begin());
    nlev = u32(uniq.size());
    return 0;
}

static int factorize_f64(const double* x, size_t n, std::vector<u32>& codes, u32& nlev) {
    std::vector<u64> keys(n);
    for (size_t i = 0; i < n; i++) {
        if (std::isnan(x[i])) { g_err = "missing values in factor"; return 198; }
        keys[i] = f64_key(x[i]);
    }
    return factorize_keys(keys, codes, nlev);
}

static int combine(const std::vector<const std::vector<u32>*>& parts, const std::vector<u32>& nl,
                   std::vector<u32>& out, u32& nlev) {
    if (parts.size() == 1) { out = *parts[0]; nlev = nl[0]; return 0; }
    size_t n = parts[0]->size();
    std::vector<u64> keys(n, 0);
    for (size_t i = 0; i < n; i++) {
        u64 k = 0;
        for (size_t p = 0; p < parts.size(); p++) k = k * u64(nl[p]) + (*parts[p])[i];
        keys[i] = k;
    }
    return factorize_keys(keys, out, nlev);
}

static void restrict_codes(const std::vector<u32>& codes, u32 g, const std::vector<u32>& kept,
                           std::vector<u32>& out, u32& nlev) {
    std::vector<u32> present(g, 0);
    out.resize(kept.size());
    for (size_t k = 0; k < kept.size(); k++) { out[k] = codes[kept[k]]; present[out[k]] = 1; }
    std::vector<u32> id(g);
    u32 next = 0;
    for (u32 l = 0; l < g; l++) { id[l] = next; next += present[l]; }
    for (auto& c : out) c = id[c];
    nlev = next;
}

// ---------------------------------------------------------------------------------------------
// sample.rs:44-72 drop_singletons + pass_serial :198: cycle over the terms in absorb order until
// `nterms` consecutive passes drop nothing; a level with (weighted) count 1 drops its rows.
static u64 drop_singletons(const std::vector<std::vector<u32>>& codes, const std::vector<u32>& g,
                           const double* fw, std::vector<uint8_t>& alive) {
    size_t nterms = codes.size();
    if (nterms == 0) return 0;
    u64 dropped = 0;
    size_t remaining = nterms, i = 0;
    while (remaining > 0) {
        size_t t = i % nterms;
        i++;
        const auto& c = codes[t];
        std::vector<double> count(g[t], 0.0);
        for (size_t o = 0; o < c.size(); o++)
            if (alive[o]) count[c[o]] += fw ? fw[o] : 1.0;
        u64 s = 0;
        for (size_t o = 0; o < c.size(); o++)
            if (alive[o] && count[c[o]] == 1.0) { alive[o] = 0; s++; }
        dropped += s;
        remaining = s > 0 ? nterms - 1 : remaining - 1;
    }
    return dropped;
}

// ---------------------------------------------------------------------------------------------
// dof.rs:222-256 mobility_groups: connected components of the bipartite graph between the levels
// of two terms, numbered 1.. by the smallest first-term level of each component.
struct DSU {
    std::vector<u32> p;
    explicit DSU(size_t n) : p(n) { std::iota(p.begin(), p.end(), 0u); }
    u32 find(u32 x) { while (p[x] != x) { p[x] = p[p[x]]; x = p[x]; } return x; }
    void unite(u32 a, u32 b) {  // the root is always the smaller vertex
        a = find(a); b = find(b);
        if (a == b) return;
        if (a < b) p[b] = a; else p[a] = b;
    }
};

static u64 mobility_groups(const std::vector<u32>& a, u32 ga, const std::vector<u32>& b, u32 gb,
                           std::vector<u32>* gv) {
    DSU d(size_t(ga) + gb);
    for (size_t i = 0; i < a.size(); i++) d.unite(a[i], ga + b[i]);
    std::vector<u32> id(ga, 0);
    u32 next = 0;
    for (u32 l = 0; l < ga; l++) if (d.find(l) == l) id[l] = ++next;
    if (gv) {
        gv->resize(a.size());
        for (size_t i = 0; i < a.size(); i++) (*gv)[i] = id[d.find(a[i])];
    }
    return next;
}

// dof.rs:184 nested_within: every level maps to a single cluster value.
static bool nested_within(const std::vector<u32>& codes, u32 g, const std::vector<u32>& cl) {
    std::vector<u32> map(g, UINT32_MAX);
    for (size_t i = 0; i < codes.size(); i++) {
        u32& s = map[codes[i]];
        if (s == UINT32_MAX) s = cl[i];
        else if (s != cl[i]) return false;
    }
    return true;
}

struct DofSlot { u64 k, m; bool exact, nested; };
struct Dof {
    std::vector<DofSlot> slots;
    u64 df_a = 0, df_a_initial = 0, df_a_redundant = 0, df_a_nested = 0;
    std::vector<u32> groupvar;
    bool has_groupvar = false;
};

// dof.rs:64-180 estimate_dof (intercept-only terms; options pairwise + clusters, as the
// reference's default `DofOptions`; `firstpair` replaces them).
static Dof estimate_dof(const std::vector<std::vector<u32>>& tcodes, const std::vector<u32>& tg,
                        const std::vector<std::vector<u32>>& ccodes, size_t n, bool firstpair,
                        bool want_groupvar) {
    std::vector<std::vector<u32>> codes = tcodes;
    std::vector<u32> g = tg;
    if (codes.empty()) { codes.push_back(std::vector<u32>(n, 0)); g.push_back(1); }
    Dof d;
    std::vector<int> iidx;
    for (size_t q = 0; q < codes.size(); q++) {
        d.slots.push_back({g[q], 0, false, false});
        iidx.push_back(int(q));
    }
    bool clusters_rule = !firstpair, pairwise = !firstpair;
    if (!ccodes.empty() && clusters_rule) {
        for (const auto& c : ccodes) {
            bool any = false;
            for (int v : iidx) any |= v >= 0;
            if (!any) break;
            for (size_t i = 0; i < d.slots.size(); i++) {
                if (iidx[i] < 0 || d.slots[i].exact) continue;
                if (nested_within(codes[iidx[i]], g[iidx[i]], c)) {
                    d.slots[i].m = d.slots[i].k;
                    d.slots[i].exact = d.slots[i].nested = true;
                    d.df_a_nested += d.slots[i].k;
                    iidx[i] = -1;
                }
            }
        }
    }
    size_t remaining = 0;
    for (int v : iidx) remaining += v >= 0;
    if (remaining > 1 || (remaining > 0 && d.df_a_nested > 0)) {
        bool skip_next = d.df_a_nested == 0;
        for (size_t i = 0; i < d.slots.size(); i++) {
            if (iidx[i] < 0) continue;
            if (skip_next) { skip_next = false; continue; }
            d.slots[i].m = 1;
        }
    }
    for (size_t i = 0; i < iidx.size(); i++) if (iidx[i] >= 0) { d.slots[i].exact = true; break; }
    if (pairwise || firstpair) {
        std::vector<std::pair<size_t, int>> idx;
        for (size_t i = 0; i < iidx.size(); i++) if (iidx[i] >= 0) idx.push_back({i, iidx[i]});
        int pair_count = 0;
        for (size_t a = 0; a < idx.size(); a++) {
            bool stop = false;
            for (size_t b = a + 1; b < idx.size(); b++) {
                int qa = idx[a].second, qb = idx[b].second;
                size_t j = idx[b].first;
                pair_count++;
                bool save = pair_count == 1 && want_groupvar;
                u64 m = mobility_groups(codes[qa], g[qa], codes[qb], g[qb], save ? &d.groupvar : nullptr);
                if (save) d.has_groupvar = true;
                d.slots[j].m = std::max(d.slots[j].m, m);
                if (pair_count == 1) d.slots[j].exact = true;
                if (firstpair) { stop = true; break; }
            }
            if (stop) break;
        }
    }
    for (auto& s : d.slots) { d.df_a_initial += s.k; d.df_a_redundant += s.m; }
    d.df_a = d.df_a_initial - d.df_a_redundant;
    return d;
}

// ---------------------------------------------------------------------------------------------
// structure.rs — the cell structure.
constexpr size_t SMALL_LIMIT = 4096;           // structure.rs:23
constexpr size_t ELIM_CANDIDATE_SHARE = 4;     // structure.rs:234
constexpr u64 ELIM_CHEAP_PER_OBS = 64;         // structure.rs:236

struct Block { size_t term; u32 g; size_t off; bool small; };

struct Structure {
    size_t n = 0;
    int fe1 = -1;              // eliminated term, -1 under noabsorb
    u32 g1 = 1;
    std::vector<u32> pi;       // kept observation of each row
    std::vector<u32> seg_off;  // g1 + 1
    std::vector<u32> cell_obs_off;  // M + 1 (empty when every cell holds one row)
    size_t ncells = 0;
    size_t nb = 0;
    std::vector<u32> cell_codes;  // M x nb
    std::vector<Block> blocks;
    size_t m = 0, m_small = 0;
    u64 small_work = 0;
    bool trivial() const { return cell_obs_off.empty(); }
    size_t row0(size_t c) const { return trivial() ? c : cell_obs_off[c]; }
    size_t row1(size_t c) const { return trivial() ? c + 1 : cell_obs_off[c + 1]; }
};

// absorber.rs:100 fe1_index: the term with the most levels, first on ties.
static int fe1_index(const std::vector<u32>& g) {
    int best = -1;
    for (size_t q = 0; q < g.size(); q++)
        if (best < 0 || g[q] > g[best]) best = int(q);
    return best;
}

// structure.rs:256-352 choose_elimination and distinct_work.
static int choose_elimination(const std::vector<std::vector<u32>>& codes, const std::vector<u32>& g) {
    int f0 = fe1_index(g);
    if (f0 < 0 || codes.size() < 3) return f0;
    std::vector<size_t> cands;
    for (size_t q = 0; q < g.size(); q++)
        if (size_t(g[q]) * ELIM_CANDIDATE_SHARE >= g[f0]) cands.push_back(q);
    if (cands.size() < 2) return f0;
    size_t n = codes[f0].size();
    std::vector<u64> size(g[f0], 0);
    for (u32 c : codes[f0]) size[c]++;
    u64 bound = 0;
    for (u64 s : size) bound += s * s;
    bound *= u64(codes.size() - 1);
    if (bound <= ELIM_CHEAP_PER_OBS * n) return f0;
    // minimise (E, -g, index)
    bool have = false;
    u64 bestE = 0; u32 bestG = 0; size_t bestF = 0;
    for (size_t f : cands) {
        // observations sorted by f (stable)
        std::vector<u32> off(g[f] + 1, 0), ids(n);
        for (u32 c : codes[f]) off[c + 1]++;
        for (u32 k = 0; k < g[f]; k++) off[k + 1] += off[k];
        std::vector<u32> cur(off.begin(), off.end() - 1);
        for (size_t i = 0; i < n; i++) ids[cur[codes[f][i]]++] = u32(i);
        u64 E = 0;
        std::vector<std::vector<u32>> stamps;
        std::vector<size_t> others;
        for (size_t q = 0; q < codes.size(); q++) if (q != f) { others.push_back(q); stamps.emplace_back(g[q], 0); }
        for (u32 s = 0; s < g[f]; s++) {
            u32 tag = s + 1;
            for (size_t k = 0; k < others.size(); k++) {
                u64 dk = 0;
                for (u32 p = off[s]; p < off[s + 1]; p++) {
                    u32 c = codes[others[k]][ids[p]];
                    if (stamps[k][c] != tag) { stamps[k][c] = tag; dk++; }
                }
                E += dk * dk;
            }
        }
        bool better = !have || E < bestE || (E == bestE && (g[f] > bestG || (g[f] == bestG && f < bestF)));
        if (better) { have = true; bestE = E; bestG = g[f]; bestF = f; }
    }
    return int(bestF);
}

// structure.rs:356-527 build.
static Structure build_structure(const std::vector<std::vector<u32>>& codes, const std::vector<u32>& g,
                                 size_t n, size_t small_limit) {
    Structure st;
    st.n = n;
    st.fe1 = choose_elimination(codes, g);
    st.g1 = st.fe1 >= 0 ? g[st.fe1] : 1;
    std::vector<size_t> others;
    for (size_t q = 0; q < g.size(); q++) if (int(q) != st.fe1) others.push_back(q);
    std::vector<size_t> by_g = others;
    std::stable_sort(by_g.begin(), by_g.end(), [&](size_t a, size_t b) { return g[a] != g[b] ? g[a] < g[b] : a < b; });
    std::vector<bool> small_set(g.size(), false);
    size_t total = 0;
    for (size_t q : by_g) {
        if (total + g[q] > small_limit) break;
        total += g[q];
        small_set[q] = true;
    }
    std::vector<size_t> order;
    for (size_t q : others) if (small_set[q]) order.push_back(q);
    for (size_t q : others) if (!small_set[q]) order.push_back(q);
    size_t off = 0;
    for (size_t q : order) { st.blocks.push_back({q, g[q], off, bool(small_set[q])}); off += g[q]; }
    st.m = off;
    st.m_small = 0;
    for (auto& b : st.blocks) if (b.small) st.m_small += b.g;
    st.nb = st.blocks.size();
    size_t nb = st.nb;

    // Rows sorted by (g1, block codes in block order, obs).
    std::vector<u32> rows(n);
    std::iota(rows.begin(), rows.end(), 0u);
    auto key_less = [&](u32 a, u32 b) {
        if (st.fe1 >= 0) {
            u32 ca = codes[st.fe1][a], cb = codes[st.fe1][b];
            if (ca != cb) return ca < cb;
        }
        for (size_t k = 0; k < nb; k++) {
            u32 ca = codes[st.blocks[k].term][a], cb = codes[st.blocks[k].term][b];
            if (ca != cb) return ca < cb;
        }
        return a < b;
    };
    std::sort(rows.begin(), rows.end(), key_less);
    st.pi = rows;
    st.seg_off.assign(st.g1 + 1, 0);
    std::vector<u32> starts;
    auto same_cell = [&](u32 a, u32 b) {
        if (st.fe1 >= 0 && codes[st.fe1][a] != codes[st.fe1][b]) return false;
        for (size_t k = 0; k < nb; k++)
            if (codes[st.blocks[k].term][a] != codes[st.blocks[k].term][b]) return false;
        return true;
    };
    for (size_t r = 0; r < n; r++) {
        if (r == 0 || !same_cell(rows[r - 1], rows[r])) {
            starts.push_back(u32(r));
            u32 s = st.fe1 >= 0 ? codes[st.fe1][rows[r]] : 0;
            st.seg_off[s + 1]++;
            for (size_t k = 0; k < nb; k++) st.cell_codes.push_back(codes[st.blocks[k].term][rows[r]]);
        }
    }
    for (u32 s = 0; s < st.g1; s++) st.seg_off[s + 1] += st.seg_off[s];
    st.ncells = starts.size();
    if (st.ncells != n) {
        st.cell_obs_off = starts;
        st.cell_obs_off.push_back(u32(n));
    }
    // sum over segments of (distinct small coordinates)^2
    std::vector<u32> mark(st.m_small, 0);
    u64 work = 0;
    for (u32 s = 0; s < st.g1; s++) {
        u64 d = 0;
        for (u32 c = st.seg_off[s]; c < st.seg_off[s + 1]; c++)
            for (size_t k = 0; k < nb; k++) {
                if (!st.blocks[k].small) continue;
                u32 x = u32(st.blocks[k].off) + st.cell_codes[c * nb + k];
                if (mark[x] != s + 1) { mark[x] = s + 1; d++; }
            }
        work += d * d;
    }
    st.small_work = work;
    if (st.m_small > 0 && work > 64 * u64(st.ncells)) {
        for (auto& b : st.blocks) b.small = false;
        st.m_small = 0;
    }
    return st;
}

// ---------------------------------------------------------------------------------------------
// Fixed task partition of the segments (thread-count independent).
constexpr int NTASK = 32;
static std::vector<u32> seg_tasks(const Structure& st) {
    std::vector<u32> t{0};
    for (int j = 1; j < NTASK; j++) {
        size_t target = st.ncells * j / NTASK;
        u32 s = u32(std::lower_bound(st.seg_off.begin(), st.seg_off.end() - 1, u32(target)) - st.seg_off.begin());
        if (s > t.back() && s < st.g1) t.push_back(s);
    }
    t.push_back(st.g1);
    return t;
}

// operator.rs:44-63 WeightState; :211-338 refresh_weights; :344-570 level_weights.
constexpr double REDUNDANT = 1e-12;  // operator.rs:21
struct WeightState {
    bool weighted = false;
    Vec w_rows;     // row order
    Vec cell_w;     // W_c (empty: every W_c is 1)
    Vec n1, nr, diag;
    std::vector<uint8_t> redundant;
    double sw = 0;
    double cw(size_t c) const { return cell_w.empty() ? 1.0 : cell_w[c]; }
};

static void refresh_weights(const Structure& st, WeightState& ws, const double* w_kept) {
    ws.weighted = w_kept != nullptr;
    ws.w_rows.clear();
    ws.cell_w.clear();
    if (w_kept) {
        ws.w_rows.resize(st.n);
        for (size_t r = 0; r < st.n; r++) ws.w_rows[r] = w_kept[st.pi[r]];
    }
    if (!st.trivial()) {
        ws.cell_w.resize(st.ncells);
        for (size_t c = 0; c < st.ncells; c++) {
            double s = 0;
            for (size_t r = st.row0(c); r < st.row1(c); r++) s += w_kept ? ws.w_rows[r] : 1.0;
            ws.cell_w[c] = s;
        }
    } else if (w_kept) {
        ws.cell_w = ws.w_rows;
    }
    ws.n1.assign(st.g1, 0.0);
    for (u32 s = 0; s < st.g1; s++) {
        double a = 0;
        for (u32 c = st.seg_off[s]; c < st.seg_off[s + 1]; c++) a += ws.cw(c);
        ws.n1[s] = a;
    }
    ws.sw = 0;
    for (double v : ws.n1) ws.sw += v;
    // n_r and sum_s c_{s,k}^2 / n1_s
    size_t m = st.m, nb = st.nb;
    ws.nr.assign(m, 0.0);
    Vec dq(m, 0.0), cs(m, 0.0);
    for (u32 s = 0; s < st.g1; s++) {
        for (u32 c = st.seg_off[s]; c < st.seg_off[s + 1]; c++)
            for (size_t b = 0; b < nb; b++) cs[st.blocks[b].off + st.cell_codes[c * nb + b]] += ws.cw(c);
        for (u32 c = st.seg_off[s]; c < st.seg_off[s + 1]; c++)
            for (size_t b = 0; b < nb; b++) {
                size_t k = st.blocks[b].off + st.cell_codes[c * nb + b];
                ws.nr[k] += ws.cw(c);
                dq[k] += ws.cw(c) * cs[k] / ws.n1[s];
            }
        for (u32 c = st.seg_off[s]; c < st.seg_off[s + 1]; c++)
            for (size_t b = 0; b < nb; b++) cs[st.blocks[b].off + st.cell_codes[c * nb + b]] = 0.0;
    }
    ws.diag.resize(m);
    ws.redundant.resize(m);
    for (size_t k = 0; k < m; k++) {
        ws.diag[k] = ws.nr[k] - dq[k];
        ws.redundant[k] = ws.diag[k] <= REDUNDANT * ws.nr[k];
    }
}

// ---------------------------------------------------------------------------------------------
// operator.rs kernels. Reduced vectors are m x r row-major, row blocks n x r row-major.
struct Ops {
    const Structure& st;
    const WeightState& ws;

    // Per-task accumulators combined in task order.
    template <class F>
    void scatter_tasks(size_t r, double* y, F body) const {
        auto tb = seg_tasks(st);
        int nt = int(tb.size()) - 1;
        std::vector<Vec> acc(nt, Vec(st.m * r, 0.0));
#pragma omp parallel for schedule(dynamic, 1)
        for (int t = 0; t < nt; t++) body(tb[t], tb[t + 1], acc[t].data());
        std::fill(y, y + st.m * r, 0.0);
        for (int t = 0; t < nt; t++)
            for (size_t i = 0; i < st.m * r; i++) y[i] += acc[t][i];
    }

    // operator.rs:1375 apply / :894-948 apply_task_inner: Y = S P.
    void apply(const double* p, size_t r, double* y) const {
        size_t nb = st.nb;
        scatter_tasks(r, y, [&](u32 s0, u32 s1, double* acc) {
            Vec u, t(r);
            for (u32 s = s0; s < s1; s++) {
                u32 c0 = st.seg_off[s], c1 = st.seg_off[s + 1];
                u.assign(size_t(c1 - c0) * r, 0.0);
                for (u32 c = c0; c < c1; c++)
                    for (size_t b = 0; b < nb; b++) {
                        const double* pv = p + (st.blocks[b].off + st.cell_codes[c * nb + b]) * r;
                        for (size_t j = 0; j < r; j++) u[(c - c0) * r + j] += pv[j];
                    }
                std::fill(t.begin(), t.end(), 0.0);
                for (u32 c = c0; c < c1; c++)
                    for (size_t j = 0; j < r; j++) t[j] += ws.cw(c) * u[(c - c0) * r + j];
                double inv = 1.0 / ws.n1[s];
                for (size_t j = 0; j < r; j++) t[j] *= inv;
                for (u32 c = c0; c < c1; c++) {
                    double w = ws.cw(c);
                    for (size_t j = 0; j < r; j++) u[(c - c0) * r + j] = w * (u[(c - c0) * r + j] - t[j]);
                    for (size_t b = 0; b < nb; b++) {
                        double* a = acc + (st.blocks[b].off + st.cell_codes[c * nb + b]) * r;
                        for (size_t j = 0; j < r; j++) a[j] += u[(c - c0) * r + j];
                    }
                }
            }
        });
    }

    // operator.rs:1382 rhs / :969-1066 rhs_task_inner.
    void rhs(const double* rows, size_t r, double* y, double* b1, double* wsq, double* wsum) const {
        size_t nb = st.nb;
        auto tb = seg_tasks(st);
        int nt = int(tb.size()) - 1;
        std::vector<Vec> acc(nt, Vec(st.m * r, 0.0)), ex(nt, Vec(2 * r, 0.0));
#pragma omp parallel for schedule(dynamic, 1)
        for (int t = 0; t < nt; t++) {
            Vec u;
            double* a = acc[t].data();
            for (u32 s = tb[t]; s < tb[t + 1]; s++) {
                u32 c0 = st.seg_off[s], c1 = st.seg_off[s + 1];
                u.assign(size_t(c1 - c0) * r, 0.0);
                double* bs = b1 + size_t(s) * r;
                std::fill(bs, bs + r, 0.0);
                for (u32 c = c0; c < c1; c++) {
                    for (size_t row = st.row0(c); row < st.row1(c); row++) {
                        double w = ws.weighted ? ws.w_rows[row] : 1.0;
                        for (size_t j = 0; j < r; j++) {
                            double v = rows[row * r + j], wv = w * v;
                            u[(c - c0) * r + j] += wv;
                            ex[t][j] += wv * v;
                            ex[t][r + j] += wv;
                        }
                    }
                    for (size_t j = 0; j < r; j++) bs[j] += u[(c - c0) * r + j];
                }
                double inv = 1.0 / ws.n1[s];
                for (u32 c = c0; c < c1; c++) {
                    double w = ws.cw(c) * inv;
                    for (size_t j = 0; j < r; j++) u[(c - c0) * r + j] -= w * bs[j];
                    for (size_t b = 0; b < nb; b++) {
                        double* ap = a + (st.blocks[b].off + st.cell_codes[c * nb + b]) * r;
                        for (size_t j = 0; j < r; j++) ap[j] += u[(c - c0) * r + j];
                    }
                }
            }
        }
        std::fill(y, y + st.m * r, 0.0);
        std::fill(wsq, wsq + r, 0.0);
        std::fill(wsum, wsum + r, 0.0);
        for (int t = 0; t < nt; t++) {
            for (size_t i = 0; i < st.m * r; i++) y[i] += acc[t][i];
            for (size_t j = 0; j < r; j++) { wsq[j] += ex[t][j]; wsum[j] += ex[t][r + j]; }
        }
    }

    // operator.rs:1395 residualize_rows / :1107-1179: alpha1 = (b1 - sum_c W_c u_c)/n1 and
    // v_i -= alpha1 + u_c for every row of every cell.
    void residualize_rows(double* rows, size_t r, const double* x, const double* b1, double* alpha) const {
        size_t nb = st.nb;
        auto tb = seg_tasks(st);
        int nt = int(tb.size()) - 1;
#pragma omp parallel for schedule(dynamic, 1)
        for (int t = 0; t < nt; t++) {
            Vec u, a(r);
            for (u32 s = tb[t]; s < tb[t + 1]; s++) {
                u32 c0 = st.seg_off[s], c1 = st.seg_off[s + 1];
                u.assign(size_t(c1 - c0) * r, 0.0);
                for (u32 c = c0; c < c1; c++)
                    for (size_t b = 0; b < nb; b++) {
                        const double* xv = x + (st.blocks[b].off + st.cell_codes[c * nb + b]) * r;
                        for (size_t j = 0; j < r; j++) u[(c - c0) * r + j] += xv[j];
                    }
                for (size_t j = 0; j < r; j++) a[j] = b1[size_t(s) * r + j];
                for (u32 c = c0; c < c1; c++)
                    for (size_t j = 0; j < r; j++) a[j] -= ws.cw(c) * u[(c - c0) * r + j];
                double inv = 1.0 / ws.n1[s];
                for (size_t j = 0; j < r; j++) a[j] *= inv;
                if (alpha) for (size_t j = 0; j < r; j++) alpha[size_t(s) * r + j] = a[j];
                for (u32 c = c0; c < c1; c++) {
                    for (size_t j = 0; j < r; j++) u[(c - c0) * r + j] += a[j];
                    for (size_t row = st.row0(c); row < st.row1(c); row++)
                        for (size_t j = 0; j < r; j++) rows[row * r + j] -= u[(c - c0) * r + j];
                }
            }
        }
    }

    // operator.rs:1424-1452 fit_rows: alpha1[g1] + sum_b x_b[g_b] per row.
    void fit_rows(const double* x, const double* alpha, double* out) const {
        size_t nb = st.nb;
        for (u32 s = 0; s < st.g1; s++)
            for (u32 c = st.seg_off[s]; c < st.seg_off[s + 1]; c++) {
                double f = alpha[s];
                for (size_t b = 0; b < nb; b++) f += x[st.blocks[b].off + st.cell_codes[c * nb + b]];
                for (size_t row = st.row0(c); row < st.row1(c); row++) out[row] = f;
            }
    }

    // The explicit small super-block S_SS (operator.rs:1457-1523 assemble_small / the fused
    // weight pass :357-568): n_r on the diagonal, cross-block cell-weight counts off it, minus
    // sum_s c_s c_s^T / n1_s.
    Vec assemble_small() const {
        size_t ms = st.m_small, nb = st.nb;
        Vec a(ms * ms, 0.0), cs(ms, 0.0);
        std::vector<size_t> touched;
        size_t ns = 0;
        for (auto& b : st.blocks) ns += b.small;
        for (u32 s = 0; s < st.g1; s++) {
            touched.clear();
            for (u32 c = st.seg_off[s]; c < st.seg_off[s + 1]; c++) {
                double w = ws.cw(c);
                for (size_t b = 0; b < ns; b++) {
                    size_t k = st.blocks[b].off + st.cell_codes[c * nb + b];
                    if (cs[k] == 0.0) touched.push_back(k);
                    cs[k] += w;
                    a[k * ms + k] += w;
                    for (size_t b2 = 0; b2 < ns; b2++) {
                        if (b2 == b) continue;
                        size_t l = st.blocks[b2].off + st.cell_codes[c * nb + b2];
                        a[k * ms + l] += w;
                    }
                }
            }
            std::sort(touched.begin(), touched.end());
            touched.erase(std::unique(touched.begin(), touched.end()), touched.end());
            double inv = 1.0 / ws.n1[s];
            for (size_t k : touched)
                for (size_t l : touched) a[k * ms + l] -= cs[k] * cs[l] * inv;
            for (size_t k : touched) cs[k] = 0.0;
        }
        return a;
    }
};

// ---------------------------------------------------------------------------------------------
// precond/dense.rs:26-28, :79-160 — grounded LDL^T of the unit-diagonal-scaled S_SS over the kept
// coordinates (non-redundant, positive diagonal). A pivot <= PIVOT_TOL is replaced by GROUND,
// which makes the factor a reflexive generalized inverse on singular (per-component) blocks.
constexpr double PIVOT_TOL = 1e-10;
constexpr double GROUND = 1e30;

struct DenseFactor {
    std::vector<u32> keep;
    Vec scale, l, d;  // unit-lower L (k x k row-major), D
    void factor(const Vec& a, size_t ms, const std::vector<uint8_t>& red) {
        keep.clear();
        for (size_t i = 0; i < ms; i++) if (!red[i] && a[i * ms + i] > 0.0) keep.push_back(u32(i));
        size_t k = keep.size();
        scale.resize(k);
        for (size_t i = 0; i < k; i++) scale[i] = 1.0 / std::sqrt(a[keep[i] * (ms + 1)]);
        l.assign(k * k, 0.0);
        d.assign(k, 0.0);
        for (size_t i = 0; i < k; i++)
            for (size_t j = 0; j <= i; j++) l[i * k + j] = a[keep[i] * ms + keep[j]] * scale[i] * scale[j];
        // left-looking LDL^T
        Vec tmp(k);
        for (size_t j = 0; j < k; j++) {
            for (size_t p = 0; p < j; p++) tmp[p] = l[j * k + p] * d[p];
            double dj = l[j * k + j];
            for (size_t p = 0; p < j; p++) dj -= l[j * k + p] * tmp[p];
            if (dj <= PIVOT_TOL) dj = GROUND;
            d[j] = dj;
            l[j * k + j] = 1.0;
            for (size_t i = j + 1; i < k; i++) {
                double v = l[i * k + j];
                for (size_t p = 0; p < j; p++) v -= l[i * k + p] * tmp[p];
                l[i * k + j] = v / dj;
            }
        }
    }
    // z[0..ms] = S_SS^+ r[0..ms] (w columns; redundant rows get 0).
    void apply(const double* r, double* z, size_t ms, size_t w) const {
        std::fill(z, z + ms * w, 0.0);
        size_t k = keep.size();
        Vec y(k);
        for (size_t j = 0; j < w; j++) {
            for (size_t i = 0; i < k; i++) y[i] = r[keep[i] * w + j] * scale[i];
            for (size_t i = 0; i < k; i++) {
                double v = y[i];
                for (size_t p = 0; p < i; p++) v -= l[i * k + p] * y[p];
                y[i] = v;
            }
            for (size_t i = 0; i < k; i++) y[i] /= d[i];
            for (size_t i = k; i-- > 0;) {
                double v = y[i];
                for (size_t p = i + 1; p < k; p++) v -= l[p * k + i] * y[p];
                y[i] = v;
            }
            for (size_t i = 0; i < k; i++) z[keep[i] * w + j] = y[i] * scale[i];
        }
    }
};

// precond/mod.rs:74-157 (small factor + Jacobi blocks) and precond/jacobi.rs:7-12.
struct Precond {
    bool has_small = false;
    DenseFactor small;
    Vec inv_diag;
    void apply(const Structure& st, const double* r, double* z, size_t w) const {
        size_t ms = st.m_small, m = st.m;
        bool has_large = ms < m;
        if (has_small) {
            if (has_large)
                for (size_t i = ms; i < m; i++)
                    for (size_t j = 0; j < w; j++) z[i * w + j] = inv_diag[i] * r[i * w + j];
            small.apply(r, z, ms, w);
        } else {
            for (size_t i = 0; i < m; i++)
                for (size_t j = 0; j < w; j++) z[i * w + j] = inv_diag[i] * r[i * w + j];
        }
    }
};

// ---------------------------------------------------------------------------------------------
// cg.rs:24-37 constants and :132-292 pcg (lockstep, per-column scalars, Hestenes-Stiefel window
// stopping rule, round-off stop). The probes act only through escalation, which this oracle
// does not have; an exact preconditioner solves in one step (:171-198).
constexpr size_t WINDOW = 5;

static void dots(const double* a, const double* b, size_t m, size_t w, double* out) {
    std::fill(out, out + w, 0.0);
    for (size_t i = 0; i < m; i++)
        for (size_t j = 0; j < w; j++) out[j] += a[i * w + j] * b[i * w + j];
}

struct PcgOut { size_t iterations = 0; bool exact = false; int rc = 0; };

static PcgOut pcg(const Ops& ops, const Precond& pre, bool exact_pre, const double* rhs, double* x, size_t w,
                  const Vec& ss1, const Vec& ss0, double tol, size_t maxiter) {
    size_t m = ops.st.m, n = m * w;
    Vec r(n, 0.0), z(n, 0.0), p(n, 0.0), q(n, 0.0);
    std::vector<bool> active(w);
    for (size_t j = 0; j < w; j++) active[j] = ss0[j] > 0.0;
    Vec floor_(w), thr(w, 0.0);
    for (size_t j = 0; j < w; j++) floor_[j] = 1e-26 * ss0[j];
    PcgOut out;
    bool xnz = false;
    for (size_t i = 0; i < n; i++) xnz |= x[i] != 0.0;
    if (xnz) {
        ops.apply(x, w, q.data());
        for (size_t i = 0; i < n; i++) r[i] = rhs[i] - q[i];
    } else {
        std::copy(rhs, rhs + n, r.begin());
    }
    pre.apply(ops.st, r.data(), z.data(), w);
    if (exact_pre) {
        for (size_t i = 0; i < m; i++)
            for (size_t j = 0; j < w; j++) if (active[j]) x[i * w + j] += z[i * w + j];
        out.iterations = 1;
        out.exact = true;
        return out;
    }
    p = z;
    Vec rho(w), rho_new(w), pq(w), gamma(w), xb(w), xr(w);
    dots(r.data(), z.data(), m, w, rho.data());
    for (size_t j = 0; j < w; j++) if (!(rho[j] > 0.0)) active[j] = false;
    for (size_t i = 0; i < m; i++)
        for (size_t j = 0; j < w; j++) if (!active[j]) p[i * w + j] = 0.0;
    std::vector<std::array<double, WINDOW>> ring(w);
    for (auto& a : ring) a.fill(0.0);
    size_t k = 0;
    for (;;) {
        bool any = false;
        for (size_t j = 0; j < w; j++) any |= active[j];
        if (!any) break;
        if (out.iterations >= maxiter) { out.rc = 430; g_err = "convergence not achieved"; return out; }
        ops.apply(p.data(), w, q.data());
        dots(p.data(), q.data(), m, w, pq.data());
        for (size_t j = 0; j < w; j++) {
            gamma[j] = 0.0;
            if (active[j]) {
                if (pq[j] > 0.0 && std::isfinite(pq[j])) gamma[j] = rho[j] / pq[j];
                else active[j] = false;
            }
        }
        std::fill(xb.begin(), xb.end(), 0.0);
        std::fill(xr.begin(), xr.end(), 0.0);
        for (size_t i = 0; i < m; i++)
            for (size_t j = 0; j < w; j++) {
                double xv = x[i * w + j] + gamma[j] * p[i * w + j];
                double rv = r[i * w + j] - gamma[j] * q[i * w + j];
                x[i * w + j] = xv;
                r[i * w + j] = rv;
                xb[j] += xv * rhs[i * w + j];
                xr[j] += xv * rv;
            }
        pre.apply(ops.st, r.data(), z.data(), w);
        dots(r.data(), z.data(), m, w, rho_new.data());
        out.iterations++;
        k++;
        for (size_t j = 0; j < w; j++) {
            if (!active[j]) continue;
            ring[j][(k - 1) % WINDOW] = gamma[j] * rho[j];
            double ssk = ss1[j] - (xb[j] + xr[j]);
            thr[j] = std::max(tol * tol * ssk, floor_[j]);
            double sum = 0;
            for (double v : ring[j]) sum += v;
            bool done = k >= WINDOW && sum <= thr[j];
            bool at_roundoff = rho_new[j] <= floor_[j];
            if (done || at_roundoff || !(rho_new[j] > 0.0)) active[j] = false;
        }
        for (size_t i = 0; i < m; i++)
            for (size_t j = 0; j < w; j++) {
                double beta = active[j] ? rho_new[j] / rho[j] : 0.0;
                p[i * w + j] = active[j] ? z[i * w + j] + beta * p[i * w + j] : 0.0;
            }
        rho = rho_new;
    }
    return out;
}

// ---------------------------------------------------------------------------------------------
// solve.rs:351 FeSolver (Absorber implementation) with :1141-1311 residualize.
struct Absorber {
    Structure st;
    WeightState ws;
    Precond pre;
    bool pre_fresh = false;
    int norm_fe1 = -1;

    void ensure_pre() {
        if (pre_fresh) return;
        pre.inv_diag.resize(st.m);
        for (size_t i = 0; i < st.m; i++)  // jacobi.rs:7
            pre.inv_diag[i] = (ws.redundant[i] || !(ws.diag[i] > 0.0)) ? 0.0 : 1.0 / ws.diag[i];
        pre.has_small = st.m_small > 0;
        if (pre.has_small) {
            Ops ops{st, ws};
            Vec a = ops.assemble_small();
            pre.small.factor(a, st.m_small, std::vector<uint8_t>(ws.redundant.begin(), ws.redundant.begin() + st.m_small));
        }
        pre_fresh = true;
    }

    // The reduced system is solved exactly when every block is in the dense small factor
    // (solve.rs:923-930).
    bool exact_pre() const { return st.m > 0 && st.m_small == st.m && pre.has_small; }

    int residualize(double* z, size_t r, double tol, size_t maxiter, bool want_coefs, const double* warm,
                    double* coefs, size_t* iters, int* exact) {
        size_t m = st.m, g1 = st.g1;
        if (r == 0) { if (iters) *iters = 1; if (exact) *exact = 1; return 0; }
        ensure_pre();
        Ops ops{st, ws};
        Vec rhs(m * r), b1(size_t(g1) * r), wsq(r), wsum(r);
        ops.rhs(z, r, rhs.data(), b1.data(), wsq.data(), wsum.data());
        Vec ss0(r), ss1(r);
        for (size_t j = 0; j < r; j++) {  // solve.rs:1210-1217
            double s = wsq[j] - wsum[j] * wsum[j] / ws.sw;
            ss0[j] = s > 1e-15 * wsq[j] ? s : 0.0;
            double b1sq = 0;
            for (u32 s1 = 0; s1 < g1; s1++) b1sq += b1[size_t(s1) * r + j] * b1[size_t(s1) * r + j] / ws.n1[s1];
            ss1[j] = wsq[j] - b1sq;
        }
        Vec buf((m + g1) * r, 0.0);
        if (warm) std::copy(warm, warm + m * r, buf.begin());
        for (size_t j = 0; j < r; j++)
            if (ss0[j] == 0.0) for (size_t i = 0; i < m; i++) buf[i * r + j] = 0.0;
        size_t it = 1;
        int ex = 1;
        if (m > 0) {
            PcgOut o = pcg(ops, pre, exact_pre(), rhs.data(), buf.data(), r, ss1, ss0, tol, maxiter);
            if (o.rc) return o.rc;
            it = std::max<size_t>(o.iterations, 1);
            bool all0 = true;
            for (double s : ss0) all0 &= s == 0.0;
            ex = o.exact || all0;
        }
        ops.residualize_rows(z, r, buf.data(), b1.data(), want_coefs ? buf.data() + m * r : nullptr);
        if (want_coefs && coefs) std::copy(buf.begin(), buf.end(), coefs);
        if (iters) *iters = it;
        if (exact) *exact = ex;
        return 0;
    }
};

// ---------------------------------------------------------------------------------------------
// stats.rs:40-176 col_stats (pass A) and :195 gram (pass B).
struct ColStats { Vec sumsq, sd, wmean, wss, wss_unc; };

static ColStats col_stats(const double* rows, size_t n, size_t r, const double* w) {
    ColStats cs;
    cs.sumsq.assign(r, 0); cs.sd.assign(r, 0); cs.wmean.assign(r, 0); cs.wss.assign(r, 0); cs.wss_unc.assign(r, 0);
    Vec mean(r, 0), m2(r, 0);
    double sw = 0;
    for (size_t i = 0; i < n; i++) sw += w ? w[i] : 1.0;
    for (size_t j = 0; j < r; j++) {
        double s = 0, ws_ = 0;
        for (size_t i = 0; i < n; i++) {
            double x = rows[i * r + j];
            s += x;
            ws_ += (w ? w[i] : 1.0) * x;
            cs.sumsq[j] += x * x;
            cs.wss_unc[j] += (w ? w[i] : 1.0) * x * x;
        }
        mean[j] = s / double(n);
        cs.wmean[j] = ws_ / sw;
        for (size_t i = 0; i < n; i++) {
            double x = rows[i * r + j];
            m2[j] += (x - mean[j]) * (x - mean[j]);
            cs.wss[j] += (w ? w[i] : 1.0) * (x - cs.wmean[j]) * (x - cs.wmean[j]);
        }
        cs.sd[j] = std::max(std::sqrt(m2[j] / (double(n) - 1.0)), 1e-3);
    }
    return cs;
}

static void gram(const double* rows, size_t n, size_t r, const double* w, Vec& g, Vec& ss) {
    g.assign(r * r, 0.0);
    ss.assign(r, 0.0);
    for (size_t i = 0; i < n; i++) {
        const double* row = rows + i * r;
        double wi = w ? w[i] : 1.0;
        for (size_t a = 0; a < r; a++) {
            ss[a] += row[a] * row[a];
            double wa = wi * row[a];
            for (size_t b = a; b < r; b++) g[a * r + b] += wa * row[b];
        }
    }
    for (size_t a = 0; a < r; a++) for (size_t b = 0; b < a; b++) g[a * r + b] = g[b * r + a];
}

// ---------------------------------------------------------------------------------------------
// vcov.rs:17-64 invsym (sweep in column order), :70 invsym_greedy, :220 inv_ext, :236 matmul,
// :254 sandwich, :292 robust_meat, :320 cluster_meat, :480-560 multiway_meat, :602-720 fix_psd.
constexpr double INVSYM_TOL = 1e-13;

static void sweep_pivot(Vec& m_, size_t k, size_t p, double d) {
    for (size_t j = 0; j < k; j++) m_[p * k + j] /= d;
    for (size_t i = 0; i < k; i++) {
        if (i == p) continue;
        double b = m_[i * k + p];
        if (b == 0.0) continue;
        for (size_t j = 0; j < k; j++) m_[i * k + j] -= b * m_[p * k + j];
        m_[i * k + p] = -b / d;
    }
    m_[p * k + p] = 1.0 / d;
}

static void symmetrize_avg(Vec& m_, size_t k) {
    for (size_t i = 0; i < k; i++)
        for (size_t j = 0; j < i; j++) {
            double v = 0.5 * (m_[i * k + j] + m_[j * k + i]);
            m_[i * k + j] = m_[j * k + i] = v;
        }
}

static Vec invsym(const Vec& a, size_t k, double tol, std::vector<bool>& dropped) {
    Vec m_ = a;
    dropped.assign(k, false);
    for (size_t p = 0; p < k; p++) {
        double d = m_[p * k + p];
        if (std::isnan(d) || d <= tol * a[p * k + p] || d <= 0.0) {
            dropped[p] = true;
            for (size_t j = 0; j < k; j++) m_[p * k + j] = m_[j * k + p] = 0.0;
            continue;
        }
        sweep_pivot(m_, k, p, d);
    }
    symmetrize_avg(m_, k);
    return m_;
}

static Vec invsym_greedy(const Vec& a, size_t k, double tol, std::vector<bool>& dropped) {
    Vec m_ = a;
    std::vector<bool> visited(k, false);
    dropped.assign(k, false);
    for (size_t it = 0; it < k; it++) {
        size_t p = SIZE_MAX;
        for (size_t i = 0; i < k; i++)
            if (!visited[i] && (p == SIZE_MAX || m_[i * k + i] > m_[p * k + p])) p = i;
        visited[p] = true;
        double d = m_[p * k + p];
        if (std::isnan(d) || d <= tol * a[p * k + p] || d <= 0.0) {
            dropped[p] = true;
            for (size_t j = 0; j < k; j++) m_[p * k + j] = m_[j * k + p] = 0.0;
            continue;
        }
        sweep_pivot(m_, k, p, d);
    }
    symmetrize_avg(m_, k);
    return m_;
}

static Vec inv_ext(const Vec& inv, size_t k, const Vec& means, double n_c) {
    size_t k1 = k + 1;
    Vec out(k1 * k1, 0.0), side(k);
    for (size_t j = 0; j < k; j++) {
        double s = 0;
        for (size_t i = 0; i < k; i++) s += means[i] * inv[i * k + j];
        side[j] = -s;
    }
    double corner = 1.0 / n_c;
    for (size_t j = 0; j < k; j++) corner -= side[j] * means[j];
    for (size_t i = 0; i < k; i++) {
        for (size_t j = 0; j < k; j++) out[i * k1 + j] = inv[i * k + j];
        out[i * k1 + k] = out[k * k1 + i] = side[i];
    }
    out[k * k1 + k] = corner;
    return out;
}

static Vec matmul(const Vec& a, const Vec& b, size_t k) {
    Vec out(k * k, 0.0);
    for (size_t i = 0; i < k; i++)
        for (size_t l = 0; l < k; l++) {
            double x = a[i * k + l];
            if (x == 0.0) continue;
            for (size_t j = 0; j < k; j++) out[i * k + j] += x * b[l * k + j];
        }
    return out;
}

static Vec sandwich(const Vec& d, const Vec& meat, size_t k, double scale) {
    Vec v = matmul(matmul(d, meat, k), d, k);
    symmetrize_avg(v, k);
    for (auto& x : v) x *= scale;
    return v;
}

static void add_outer(Vec& acc, const double* a, double s, size_t m) {
    for (size_t i = 0; i < m; i++) {
        double ai = a[i] * s;
        if (ai == 0.0) continue;
        for (size_t j = i; j < m; j++) acc[i * m + j] += ai * a[j];
    }
}
static void mirror(Vec& acc, size_t m) {
    for (size_t i = 0; i < m; i++) for (size_t j = 0; j < i; j++) acc[i * m + j] = acc[j * m + i];
}

// Cluster score sums grouped by code (row-order codes), then sum_g s_g s_g^T.
template <class RowF>
static Vec cluster_meat(const std::vector<u32>& codes, u32 g, size_t msz, RowF row) {
    Vec sums(size_t(g) * msz, 0.0), a(msz);
    for (size_t i = 0; i < codes.size(); i++) {
        double s = row(i, a.data());
        double* o = sums.data() + size_t(codes[i]) * msz;
        for (size_t p = 0; p < msz; p++) o[p] += s * a[p];
    }
    Vec meat(msz * msz, 0.0);
    for (u32 c = 0; c < g; c++) add_outer(meat, sums.data() + size_t(c) * msz, 1.0, msz);
    mirror(meat, msz);
    return meat;
}

static void sym_eigen(const Vec& a, size_t k, Vec& lam, Vec& v) {
    Vec m_ = a;
    v.assign(k * k, 0.0);
    for (size_t i = 0; i < k; i++) v[i * k + i] = 1.0;
    const double eps = 2.220446049250313e-16;
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0, total = 0;
        for (size_t i = 0; i < k; i++)
            for (size_t j = 0; j < k; j++) { if (i != j) off += m_[i * k + j] * m_[i * k + j]; total += m_[i * k + j] * m_[i * k + j]; }
        if (off <= eps * eps * total * 1e-4 || off == 0.0) break;
        for (size_t p = 0; p < k; p++)
            for (size_t q = p + 1; q < k; q++) {
                double apq = m_[p * k + q];
                if (apq == 0.0) continue;
                double theta = (m_[q * k + q] - m_[p * k + p]) / (2.0 * apq);
                double t = (theta > 0 ? 1.0 : (theta < 0 ? -1.0 : 0.0)) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                if (theta == 0.0) t = 1.0;
                double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (size_t r = 0; r < k; r++) {
                    double mrp = m_[r * k + p], mrq = m_[r * k + q];
                    m_[r * k + p] = c * mrp - s * mrq;
                    m_[r * k + q] = s * mrp + c * mrq;
                }
                for (size_t r = 0; r < k; r++) {
                    double mpr = m_[p * k + r], mqr = m_[q * k + r];
                    m_[p * k + r] = c * mpr - s * mqr;
                    m_[q * k + r] = s * mpr + c * mqr;
                }
                for (size_t r = 0; r < k; r++) {
                    double vrp = v[r * k + p], vrq = v[r * k + q];
                    v[r * k + p] = c * vrp - s * vrq;
                    v[r * k + q] = s * vrp + c * vrq;
                }
            }
    }
    lam.resize(k);
    for (size_t i = 0; i < k; i++) lam[i] = m_[i * k + i];
}

static bool clip_psd(const Vec& v, size_t k, Vec& out) {
    Vec lam, u;
    sym_eigen(v, k, lam, u);
    bool neg = false;
    for (double l : lam) neg |= l < 0.0;
    if (!neg) return false;
    out.assign(k * k, 0.0);
    for (size_t e = 0; e < k; e++) {
        if (lam[e] <= 0.0) continue;
        for (size_t i = 0; i < k; i++) {
            double ui = u[i * k + e] * lam[e];
            for (size_t j = 0; j <= i; j++) out[i * k + j] += ui * u[j * k + e];
        }
    }
    for (size_t i = 0; i < k; i++) for (size_t j = 0; j < i; j++) out[j * k + i] = out[i * k + j];
    return true;
}

static bool fix_psd(Vec& v, size_t k, bool report_constant) {
    symmetrize_avg(v, k);
    size_t kb = report_constant ? k - 1 : k;
    Vec backup(kb * kb);
    for (size_t i = 0; i < kb; i++) for (size_t j = 0; j < kb; j++) backup[i * kb + j] = v[i * k + j];
    Vec fixed;
    if (!clip_psd(v, k, fixed)) return false;
    v = fixed;
    if (report_constant) {
        Vec sub;
        if (!clip_psd(backup, kb, sub)) sub = backup;
        for (size_t i = 0; i < kb; i++) for (size_t j = 0; j < kb; j++) v[i * k + j] = sub[i * kb + j];
    }
    return true;
}

}  // namespace orc

// =============================================================================================
// C ABI (ctypes) — the oracle's entry points.
using namespace orc;

struct OrcAbsorber { Absorber a; };

extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

void orc_set_threads(int t) { if (t > 0) omp_set_num_threads(t); }
int orc_max_threads() { return omp_get_max_threads(); }

void orc_splitmix_fill_u64(uint64_t seed, uint64_t index, int use_stream, uint64_t* out, size_t n) {
    SplitMix64 s = use_stream ? SplitMix64::stream(seed, index) : SplitMix64(seed);
    for (size_t i = 0; i < n; i++) out[i] = s.next_u64();
}

int orc_factorize_f64(const double* x, size_t n, uint32_t* codes, uint32_t* nlevels) {
    std::vector<u32> c;
    u32 g = 0;
    int rc = factorize_f64(x, n, c, g);
    if (rc) return rc;
    std::copy(c.begin(), c.end(), codes);
    *nlevels = g;
    return 0;
}

int orc_combine(const uint32_t* const* parts, const uint32_t* nl, int np, size_t n, uint32_t* out, uint32_t* nlevels) {
    std::vector<std::vector<u32>> own(np);
    std::vector<const std::vector<u32>*> ptrs;
    std::vector<u32> g(nl, nl + np);
    for (int p = 0; p < np; p++) { own[p].assign(parts[p], parts[p] + n); ptrs.push_back(&own[p]); }
    std::vector<u32> o;
    u32 nn = 0;
    combine(ptrs, g, o, nn);
    std::copy(o.begin(), o.end(), out);
    *nlevels = nn;
    return 0;
}

uint64_t orc_drop_singletons(const uint32_t* const* codes, const uint32_t* g, int nterms, size_t n,
                             const double* fw, uint8_t* alive) {
    std::vector<std::vector<u32>> c(nterms);
    for (int t = 0; t < nterms; t++) c[t].assign(codes[t], codes[t] + n);
    std::vector<u32> gg(g, g + nterms);
    std::vector<uint8_t> al(alive, alive + n);
    u64 d = drop_singletons(c, gg, fw, al);
    std::copy(al.begin(), al.end(), alive);
    return d;
}

uint64_t orc_mobility_groups(const uint32_t* a, uint32_t ga, const uint32_t* b, uint32_t gb, size_t n, uint32_t* gv) {
    std::vector<u32> va(a, a + n), vb(b, b + n), out;
    u64 k = mobility_groups(va, ga, vb, gb, gv ? &out : nullptr);
    if (gv) std::copy(out.begin(), out.end(), gv);
    return k;
}

void* orc_absorber_create(const uint32_t* const* codes, const uint32_t* g, int nterms, const double* w, size_t n) {
    auto* h = new OrcAbsorber();
    std::vector<std::vector<u32>> c(nterms);
    for (int t = 0; t < nterms; t++) c[t].assign(codes[t], codes[t] + n);
    std::vector<u32> gg(g, g + nterms);
    h->a.st = build_structure(c, gg, n, SMALL_LIMIT);
    h->a.norm_fe1 = fe1_index(gg);
    refresh_weights(h->a.st, h->a.ws, w);
    return h;
}

void orc_absorber_destroy(void* h) { delete static_cast<OrcAbsorber*>(h); }

// info: n, m, g1, ncells, nb, m_small, fe1, small_work
void orc_absorber_info(void* h, uint64_t* out) {
    auto& st = static_cast<OrcAbsorber*>(h)->a.st;
    out[0] = st.n; out[1] = st.m; out[2] = st.g1; out[3] = st.ncells; out[4] = st.nb; out[5] = st.m_small;
    out[6] = uint64_t(int64_t(st.fe1)); out[7] = st.small_work;
}

void orc_absorber_row_order(void* h, uint32_t* out) {
    auto& st = static_cast<OrcAbsorber*>(h)->a.st;
    std::copy(st.pi.begin(), st.pi.end(), out);
}

// structure arrays: seg_off (g1+1), cell_codes (M*nb), cell_obs_off (M+1 or empty), block info
// (term, g, off, small) x nb.
void orc_absorber_structure(void* h, uint32_t* seg_off, uint32_t* cell_codes, uint32_t* cell_obs_off, uint64_t* blocks) {
    auto& st = static_cast<OrcAbsorber*>(h)->a.st;
    if (seg_off) std::copy(st.seg_off.begin(), st.seg_off.end(), seg_off);
    if (cell_codes) std::copy(st.cell_codes.begin(), st.cell_codes.end(), cell_codes);
    if (cell_obs_off && !st.cell_obs_off.empty()) std::copy(st.cell_obs_off.begin(), st.cell_obs_off.end(), cell_obs_off);
    if (blocks)
        for (size_t b = 0; b < st.nb; b++) {
            blocks[4 * b] = st.blocks[b].term; blocks[4 * b + 1] = st.blocks[b].g;
            blocks[4 * b + 2] = st.blocks[b].off; blocks[4 * b + 3] = st.blocks[b].small;
        }
}

// weight state: n1 (g1), nr (m), diag (m), redundant (m), sw
void orc_absorber_weight_state(void* h, double* n1, double* nr, double* diag, uint8_t* red, double* sw) {
    auto& ws = static_cast<OrcAbsorber*>(h)->a.ws;
    if (n1) std::copy(ws.n1.begin(), ws.n1.end(), n1);
    if (nr) std::copy(ws.nr.begin(), ws.nr.end(), nr);
    if (diag) std::copy(ws.diag.begin(), ws.diag.end(), diag);
    if (red) std::copy(ws.redundant.begin(), ws.redundant.end(), red);
    if (sw) *sw = ws.sw;
}

int orc_absorber_set_weights(void* h, const double* w) {
    auto& a = static_cast<OrcAbsorber*>(h)->a;
    if (w)
        for (size_t i = 0; i < a.st.n; i++)
            if (!(std::isfinite(w[i]) && w[i] > 0.0)) { g_err = "weights must be positive and finite"; return 198; }
    // weights arrive in row order (Absorber::set_weights); the state keeps kept order for rows
    std::vector<double> kept;
    if (w) {
        kept.resize(a.st.n);
        for (size_t r = 0; r < a.st.n; r++) kept[a.st.pi[r]] = w[r];
    }
    refresh_weights(a.st, a.ws, w ? kept.data() : nullptr);
    a.pre_fresh = false;
    return 0;
}

int orc_absorber_residualize(void* h, double* z, size_t r, double tol, size_t maxiter, int want_coefs,
                             const double* warm, double* coefs, uint64_t* iters, int* exact) {
    size_t it = 0;
    int rc = static_cast<OrcAbsorber*>(h)->a.residualize(z, r, tol, maxiter, want_coefs != 0, warm, coefs, &it, exact);
    if (iters) *iters = it;
    return rc;
}

// Operator pieces, for kernel-level parity tests.
void orc_absorber_apply(void* h, const double* p, size_t r, double* y) {
    auto& a = static_cast<OrcAbsorber*>(h)->a;
    Ops{a.st, a.ws}.apply(p, r, y);
}
void orc_absorber_rhs(void* h, const double* rows, size_t r, double* y, double* b1, double* wsq, double* wsum) {
    auto& a = static_cast<OrcAbsorber*>(h)->a;
    Ops{a.st, a.ws}.rhs(rows, r, y, b1, wsq, wsum);
}
void orc_absorber_precond(void* h, const double* rr, size_t w, double* z) {
    auto& a = static_cast<OrcAbsorber*>(h)->a;
    a.ensure_pre();
    a.pre.apply(a.st, rr, z, w);
}
void orc_absorber_fit_rows(void* h, const double* coefs, size_t r, size_t col, double* out) {
    auto& a = static_cast<OrcAbsorber*>(h)->a;
    size_t m = a.st.m, g1 = a.st.g1;
    std::vector<double> x(m), al(g1);
    for (size_t i = 0; i < m; i++) x[i] = coefs[i * r + col];
    for (size_t s = 0; s < g1; s++) al[s] = coefs[(m + s) * r + col];
    Ops{a.st, a.ws}.fit_rows(x.data(), al.data(), out);
}

// solve.rs:1319-1343 term_values: values per session term, normalised so every term but the
// most-levels one has weighted mean 0. `out` holds sum_q g_q values, terms in session order.
int orc_absorber_term_values(void* h, const double* coefs, size_t r, size_t col, const uint32_t* g, int nterms, double* out) {
    auto& a = static_cast<OrcAbsorber*>(h)->a;
    auto& st = a.st;
    if (st.fe1 < 0 || a.norm_fe1 < 0) return 0;
    std::vector<std::vector<double>> vals(nterms), lw(nterms);
    vals[st.fe1].resize(st.g1);
    for (size_t s = 0; s < st.g1; s++) vals[st.fe1][s] = coefs[(st.m + s) * r + col];
    lw[st.fe1] = a.ws.n1;
    for (auto& b : st.blocks) {
        vals[b.term].resize(b.g);
        lw[b.term].resize(b.g);
        for (size_t l = 0; l < b.g; l++) { vals[b.term][l] = coefs[(b.off + l) * r + col]; lw[b.term][l] = a.ws.nr[b.off + l]; }
    }
    double shift = 0;
    for (int t = 0; t < nterms; t++) {
        if (t == a.norm_fe1) continue;
        double mean = 0;
        for (size_t l = 0; l < vals[t].size(); l++) mean += vals[t][l] * lw[t][l];
        mean /= a.ws.sw;
        for (auto& v : vals[t]) v -= mean;
        shift += mean;
    }
    for (auto& v : vals[a.norm_fe1]) v += shift;
    size_t o = 0;
    for (int t = 0; t < nterms; t++) { for (size_t l = 0; l < g[t]; l++) out[o + l] = vals[t][l]; o += g[t]; }
    return 0;
}

// ------------------------------------------------------------------------------------------
// Full OLS call with reghdfe conventions (session.rs:458-560 prepare + ols.rs:234-470).
struct OrcOlsSpec {
    size_t n_input;
    int nfactors;
    const double* const* factors;   // factor value columns (n_input each)
    int nterms;
    const int* term_nf;             // factors per absorb term
    const int* term_f;              // flattened factor indices
    int ncl;
    const int* cl_nf;               // factors per cluster dimension
    const int* cl_f;
    const double* y;
    int nx;
    const double* const* x;
    const double* w;                // raw weights or null
    int weight_kind;                // 0 none, 1 aweight, 2 fweight, 3 pweight
    int vce;                        // 0 unadjusted, 1 robust, 2 cluster
    int drop_singletons;
    int noconstant;
    int firstpair;
    double tol;
    size_t maxiter;
    int threads;
};

struct OrcOlsOut {
    // sizes: b (nx+1), V ((nx+1)^2), status (nx), sample (n_input), resid (n_input), d (n_input),
    // groupvar (n_input), dof_table (5 * nslots max 64)
    double* b;
    double* V;
    uint8_t* status;
    uint8_t* sample;
    double* resid;        // kept order, optional
    double* d;            // kept order, optional
    double* groupvar;     // kept order, optional
    double* dof_table;
    int nslots;
    int k_all;
    // scalars
    double N, rank, df_r, df_m, df_a, df_a_initial, df_a_redundant, df_a_nested;
    double N_clust, N_clustervars, N_clust1, N_clust2, num_singletons, N_full, report_constant;
    double rss, tss, tss_within, mss, rmse, r2, r2_a, r2_within, r2_a_within, ll, ll_0, F, sumweights;
    double ic, y_absorbed;
};

static double nanv() { return std::nan(""); }

// A prepared session: kept-order term and cluster codes, raw kept-order weights and their kind,
// and the absorber built on the terms (session.rs).
struct OrcSession {
    Absorber ab;
    std::vector<std::vector<u32>> tcodes, ccodes;
    std::vector<u32> tg, cg;
    std::vector<double> wk;
    int kind = 0;
    size_t n = 0;
    u64 nsing = 0;
};

static void session_build(OrcSession& s) {
    s.ab.st = build_structure(s.tcodes, s.tg, s.n, SMALL_LIMIT);
    s.ab.norm_fe1 = fe1_index(s.tg);
    refresh_weights(s.ab.st, s.ab.ws, s.wk.empty() ? nullptr : s.wk.data());
}

// The OLS call on a prepared session (ols.rs:263-470): rows (n x (1 + nx), row order) are
// residualized in place; outputs in kept order.
struct OlsArgs {
    int vce, noconstant, firstpair;
    double tol;
    size_t maxiter;
};

static int session_ols(OrcSession& s, std::vector<double>& rows, size_t nx, const OlsArgs& a, OrcOlsOut* out) {
    Absorber& ab = s.ab;
    const size_t n = s.n, r = 1 + nx;
    const auto& pi = ab.st.pi;
    const auto& tcodes = s.tcodes;
    const auto& tg = s.tg;
    const auto& ccodes = s.ccodes;
    const auto& cg = s.cg;
    const u64 nsing = s.nsing;
    // weights (ols.rs:77-108)
    int kind = s.kind;
    std::vector<double> raw, wv;
    double sumw = double(n);
    if (!s.wk.empty()) {
        raw.resize(n);
        sumw = 0;
        for (size_t i = 0; i < n; i++) { raw[i] = s.wk[pi[i]]; sumw += raw[i]; }
        if (kind == 1 || kind == 3) { wv.resize(n); for (size_t i = 0; i < n; i++) wv[i] = raw[i] * double(n) / sumw; }
        else if (kind == 2) wv = raw;
    }
    double bigN = kind == 2 ? sumw : double(n);
    auto wvf = [&](size_t i) { return wv.empty() ? 1.0 : wv[i]; };
    int vce = a.vce;
    if (vce == 0 && kind == 3) vce = 1;  // ols.rs:150 pweight + unadjusted -> robust
    bool has_intercept = true;  // intercept-only absorb terms (or noabsorb) contain the constant
    bool report_constant = has_intercept && !a.noconstant;

    // dof (needs cluster codes in kept order)
    Dof dof = estimate_dof(tcodes, tg, vce == 2 ? ccodes : std::vector<std::vector<u32>>{}, n, a.firstpair != 0, out->groupvar != nullptr);

    ColStats cs = col_stats(rows.data(), n, r, raw.empty() ? nullptr : raw.data());
    Vec tss_all(r);
    double tscale = (kind == 1 || kind == 3) ? double(n) / sumw : 1.0;
    for (size_t j = 0; j < r; j++) tss_all[j] = (has_intercept ? cs.wss[j] : cs.wss_unc[j]) * tscale;
    const Vec& sd = cs.sd;

    bool want_coefs = out->d != nullptr;
    size_t m = ab.st.m, g1 = ab.st.g1;
    std::vector<double> coefs((m + g1) * r);
    size_t iters = 0;
    int exact = 0;
    int rc = ab.residualize(rows.data(), r, a.tol, a.maxiter, want_coefs, nullptr, coefs.data(), &iters, &exact);
    if (rc) return rc;

    Vec g, ss_res;
    gram(rows.data(), n, r, wv.empty() ? nullptr : wv.data(), g, ss_res);
    double ctol = std::min(1e-6, a.tol / 10.0);
    std::vector<bool> absorbed(r);
    for (size_t j = 0; j < r; j++) absorbed[j] = ss_res[j] / cs.sumsq[j] <= ctol;
    std::vector<uint8_t> status(nx, 0);
    bool y_abs = nx >= 1 && absorbed[0];
    if (y_abs) {
        for (size_t i = 0; i < n; i++) rows[i * r] = 0.0;
        for (size_t j = 0; j < r; j++) g[j] = g[j * r] = 0.0;
    }
    for (size_t j = 1; j < r; j++) if (absorbed[j]) status[j - 1] = 2;
    std::vector<size_t> cand;
    for (size_t j = 1; j < r; j++) if (status[j - 1] == 0) cand.push_back(j);
    size_t kc = cand.size();
    Vec gs(kc * kc);
    for (size_t a = 0; a < kc; a++) for (size_t b = 0; b < kc; b++) gs[a * kc + b] = g[cand[a] * r + cand[b]] / (sd[cand[a]] * sd[cand[b]]);
    std::vector<bool> dropped;
    Vec inv_c = invsym(gs, kc, INVSYM_TOL, dropped);
    std::vector<size_t> keep_pos, kept_cols;
    for (size_t c = 0; c < kc; c++) {
        if (dropped[c]) status[cand[c] - 1] = 3;
        else { keep_pos.push_back(c); kept_cols.push_back(cand[c]); }
    }
    size_t k = kept_cols.size();
    Vec inv_s(k * k);
    for (size_t a = 0; a < k; a++) for (size_t b = 0; b < k; b++) inv_s[a * k + b] = inv_c[keep_pos[a] * kc + keep_pos[b]];
    double sd_y = sd[0];
    Vec xy_s(k), b_s(k, 0.0), beta(k);
    for (size_t a = 0; a < k; a++) xy_s[a] = g[kept_cols[a] * r] / (sd[kept_cols[a]] * sd_y);
    for (size_t a = 0; a < k; a++) for (size_t b = 0; b < k; b++) b_s[a] += inv_s[a * k + b] * xy_s[b];
    for (size_t a = 0; a < k; a++) beta[a] = b_s[a] * sd_y / sd[kept_cols[a]];

    std::vector<double> e(n);
    for (size_t i = 0; i < n; i++) {
        double v = rows[i * r];
        for (size_t a = 0; a < k; a++) v -= beta[a] * rows[i * r + kept_cols[a]];
        e[i] = v;
    }
    double rss = 0;
    for (size_t i = 0; i < n; i++) rss += wvf(i) * e[i] * e[i];
    double rss_s = rss / (sd_y * sd_y);

    Vec means_s(k), xbar(k);
    for (size_t a = 0; a < k; a++) { means_s[a] = cs.wmean[kept_cols[a]] / sd[kept_cols[a]]; xbar[a] = cs.wmean[kept_cols[a]]; }
    double ybar_s = cs.wmean[0] / sd_y;
    double b0_s = ybar_s;
    for (size_t a = 0; a < k; a++) b0_s -= means_s[a] * b_s[a];
    size_t msz = k + (report_constant ? 1 : 0);
    double n_const = (kind == 1 || kind == 3) ? double(n) : sumw;
    Vec bread = report_constant ? inv_ext(inv_s, k, means_s, n_const) : inv_s;
    Vec b_full_s = b_s;
    if (report_constant) b_full_s.push_back(b0_s);

    double df_a = double(dof.df_a), df_m = double(k);
    double df_r = bigN - df_a - df_m;
    Vec v_s(msz * msz, 0.0);
    double g_min = 0;
    if (!ccodes.empty()) { g_min = cg[0]; for (u32 x : cg) g_min = std::min<double>(g_min, x); }
    double nested_adj = dof.df_a_nested > 0 ? 1.0 : 0.0;
    double q_cluster = (bigN - 1.0) / (bigN - nested_adj - df_m - df_a) * g_min / (g_min - 1.0);
    Vec sc(msz);
    for (size_t a = 0; a < k; a++) sc[a] = sd[kept_cols[a]];
    if (report_constant) sc[k] = 1.0;
    auto fill_row = [&](size_t i, double* a) {
        for (size_t p = 0; p < k; p++) a[p] = rows[i * r + kept_cols[p]] + (report_constant ? xbar[p] : 0.0);
        if (report_constant) a[k] = 1.0;
    };
    auto standardize = [&](Vec& mt) {
        for (size_t a = 0; a < msz; a++) for (size_t b = 0; b < msz; b++) mt[a * msz + b] /= sc[a] * sc[b] * sd_y * sd_y;
    };
    if (msz > 0) {
        if (vce == 0) {
            double adj = bigN / df_r;
            for (size_t i = 0; i < msz * msz; i++) v_s[i] = (rss_s / bigN) * adj * bread[i];
        } else if (vce == 1) {
            Vec meat(msz * msz, 0.0), a(msz);
            for (size_t i = 0; i < n; i++) {
                fill_row(i, a.data());
                double mult;
                if (kind == 0) mult = e[i] * e[i];
                else if (kind == 2) mult = e[i] * e[i] * wvf(i);
                else { double x = e[i] * wvf(i); mult = x * x; }
                add_outer(meat, a.data(), mult, msz);
            }
            mirror(meat, msz);
            standardize(meat);
            v_s = sandwich(bread, meat, msz, bigN / (bigN - df_a - df_m));
        } else {
            // vcov.rs:480-560 multiway meat: inclusion-exclusion over non-empty subsets
            size_t q = ccodes.size();
            Vec meat(msz * msz, 0.0);
            std::vector<std::vector<size_t>> subs;
            for (size_t size = 1; size <= q; size++) {
                std::vector<size_t> cur;
                std::function<void(size_t)> rec = [&](size_t start) {
                    if (cur.size() == size) { subs.push_back(cur); return; }
                    for (size_t i = start; i < q; i++) { cur.push_back(i); rec(i + 1); cur.pop_back(); }
                };
                rec(0);
            }
            for (auto& sub : subs) {
                double sign = sub.size() % 2 == 1 ? 1.0 : -1.0;
                std::vector<u32> kc_;
                u32 gsub;
                if (sub.size() == 1) { kc_ = ccodes[sub[0]]; gsub = cg[sub[0]]; }
                else {
                    std::vector<const std::vector<u32>*> ptrs;
                    std::vector<u32> gs2;
                    for (size_t d : sub) { ptrs.push_back(&ccodes[d]); gs2.push_back(cg[d]); }
                    combine(ptrs, gs2, kc_, gsub);
                }
                std::vector<u32> rc_(n);
                for (size_t i = 0; i < n; i++) rc_[i] = kc_[pi[i]];
                Vec part = cluster_meat(rc_, gsub, msz, [&](size_t i, double* a) { fill_row(i, a); return e[i] * wvf(i); });
                for (size_t i = 0; i < msz * msz; i++) meat[i] += sign * part[i];
            }
            standardize(meat);
            v_s = sandwich(bread, meat, msz, q_cluster);
            if (ccodes.size() > 1) fix_psd(v_s, msz, report_constant);
        }
    }
    if (vce == 2) df_r = std::min(df_r, g_min - 1.0);
    for (size_t i = 0; i < msz; i++) for (size_t j = 0; j < i; j++) v_s[j * msz + i] = v_s[i * msz + j];

    double f_stat = nanv();
    if (k > 0) {
        Vec vkk(k * k);
        for (size_t a = 0; a < k; a++) for (size_t b = 0; b < k; b++) vkk[a * k + b] = v_s[a * msz + b];
        std::vector<bool> dv;
        Vec iv = invsym_greedy(vkk, k, 1e-9, dv);
        bool anyd = false;
        for (bool x : dv) anyd |= x;
        if (!anyd) {
            double qf = 0;
            for (size_t a = 0; a < k; a++) for (size_t b = 0; b < k; b++) qf += b_s[a] * iv[a * k + b] * b_s[b];
            f_stat = qf / df_m;
            if (!std::isfinite(f_stat)) f_stat = nanv();
        }
    }
    bool anynan = false;
    for (double x : v_s) anynan |= std::isnan(x);
    if (anynan) std::fill(v_s.begin(), v_s.end(), 0.0);
    Vec sx(msz);
    for (size_t a = 0; a < msz; a++) sx[a] = sc[a] / sd_y;
    Vec b_raw(msz), v_raw(msz * msz);
    for (size_t a = 0; a < msz; a++) b_raw[a] = b_full_s[a] / sx[a];
    for (size_t a = 0; a < msz; a++) for (size_t b = 0; b < msz; b++) v_raw[a * msz + b] = v_s[a * msz + b] / (sx[a] * sx[b]);
    double b0 = report_constant ? b_raw[k] : 0.0;

    size_t k_all = nx + (report_constant ? 1 : 0);
    std::vector<size_t> pos;
    for (size_t c : kept_cols) pos.push_back(c - 1);
    if (report_constant) pos.push_back(nx);
    std::fill(out->b, out->b + k_all, 0.0);
    std::fill(out->V, out->V + k_all * k_all, 0.0);
    for (size_t a = 0; a < pos.size(); a++) {
        out->b[pos[a]] = b_raw[a];
        for (size_t b = 0; b < pos.size(); b++) out->V[pos[a] * k_all + pos[b]] = v_raw[a * msz + b];
    }
    out->k_all = int(k_all);
    std::copy(status.begin(), status.end(), out->status);

    double tss = tss_all[0], tss_within = g[0];
    double used_df_r = bigN - df_a - df_m - double(dof.df_a_nested);
    double hi = has_intercept ? 1.0 : 0.0;
    double ln2pi = std::log(2.0 * M_PI);
    auto fin = [](double x) { return std::isfinite(x) ? x : nanv(); };
    out->N = bigN; out->rank = df_m; out->df_r = df_r; out->df_m = df_m;
    out->df_a = df_a; out->df_a_initial = double(dof.df_a_initial); out->df_a_redundant = double(dof.df_a_redundant);
    out->df_a_nested = double(dof.df_a_nested);
    out->N_clust = vce == 2 ? g_min : nanv();
    out->N_clustervars = vce == 2 ? double(ccodes.size()) : nanv();
    out->N_clust1 = vce == 2 && ccodes.size() > 0 ? double(cg[0]) : nanv();
    out->N_clust2 = vce == 2 && ccodes.size() > 1 ? double(cg[1]) : nanv();
    out->num_singletons = double(nsing);
    out->N_full = bigN + double(nsing);
    out->report_constant = report_constant;
    out->rss = fin(rss); out->tss = fin(tss); out->tss_within = fin(tss_within); out->mss = fin(tss - rss);
    out->rmse = fin(used_df_r != 0.0 ? std::sqrt(rss / used_df_r) : std::sqrt(rss));
    out->r2 = fin(1.0 - rss / tss);
    out->r2_a = fin(1.0 - (rss / used_df_r) / (tss / (bigN - hi)));
    out->r2_within = fin(1.0 - rss / tss_within);
    out->r2_a_within = fin(1.0 - (rss / used_df_r) / (tss_within / (used_df_r + df_m)));
    out->ll = fin(-0.5 * bigN * (1.0 + ln2pi + std::log(rss / bigN)));
    out->ll_0 = fin(-0.5 * bigN * (1.0 + ln2pi + std::log(tss_within / bigN)));
    out->F = f_stat;
    out->sumweights = sumw;
    out->ic = double(iters);
    out->y_absorbed = y_abs;
    out->nslots = int(dof.slots.size());
    for (size_t i = 0; i < dof.slots.size() && i < 64; i++) {
        auto& s = dof.slots[i];
        double* t = out->dof_table + 5 * i;
        t[0] = double(s.k); t[1] = double(s.m); t[2] = double(s.k - s.m); t[3] = s.exact ? 0.0 : 1.0; t[4] = s.nested ? 1.0 : 0.0;
    }
    if (out->resid) for (size_t i = 0; i < n; i++) out->resid[pi[i]] = e[i];
    if (out->d && want_coefs) {
        // fe_recovery: d = fit of alpha_y - sum beta_j alpha_xj, plus b0 (the constant)
        Vec comb((m + g1), 0.0), cvec(r, 0.0);
        cvec[0] = 1.0;
        for (size_t a = 0; a < k; a++) cvec[kept_cols[a]] = -beta[a];
        for (size_t i = 0; i < m + g1; i++) for (size_t j = 0; j < r; j++) comb[i] += coefs[i * r + j] * cvec[j];
        std::vector<double> fr(n);
        Ops{ab.st, ab.ws}.fit_rows(comb.data(), comb.data() + m, fr.data());
        for (size_t i = 0; i < n; i++) out->d[pi[i]] = fr[i] - b0;
    }
    if (out->groupvar) {
        for (size_t i = 0; i < n; i++) out->groupvar[i] = dof.has_groupvar ? double(dof.groupvar[i]) : nanv();
    }
    return 0;
}

int orc_ols(const OrcOlsSpec* sp, OrcOlsOut* out) {
    if (sp->threads > 0) omp_set_num_threads(sp->threads);
    size_t n0 = sp->n_input;
    // factorize
    std::vector<std::vector<u32>> fcodes(sp->nfactors);
    std::vector<u32> fg(sp->nfactors);
    for (int f = 0; f < sp->nfactors; f++) {
        int rc = factorize_f64(sp->factors[f], n0, fcodes[f], fg[f]);
        if (rc) return rc;
    }
    auto interact = [&](const int* fs, int nf, std::vector<u32>& out_, u32& g_) {
        std::vector<const std::vector<u32>*> ptrs;
        std::vector<u32> gs;
        for (int i = 0; i < nf; i++) { ptrs.push_back(&fcodes[fs[i]]); gs.push_back(fg[fs[i]]); }
        combine(ptrs, gs, out_, g_);
    };
    std::vector<std::vector<u32>> tcodes(sp->nterms);
    std::vector<u32> tg(sp->nterms);
    {
        int o = 0;
        for (int t = 0; t < sp->nterms; t++) { interact(sp->term_f + o, sp->term_nf[t], tcodes[t], tg[t]); o += sp->term_nf[t]; }
    }
    std::vector<std::vector<u32>> ccodes(sp->ncl);
    std::vector<u32> cg(sp->ncl);
    {
        int o = 0;
        for (int c = 0; c < sp->ncl; c++) { interact(sp->cl_f + o, sp->cl_nf[c], ccodes[c], cg[c]); o += sp->cl_nf[c]; }
    }
    // singletons
    std::vector<uint8_t> alive(n0, 1);
    const double* fw = sp->weight_kind == 2 ? sp->w : nullptr;
    u64 nsing = sp->drop_singletons ? drop_singletons(tcodes, tg, fw, alive) : 0;
    std::vector<u32> kept;
    for (size_t i = 0; i < n0; i++) if (alive[i]) kept.push_back(u32(i));
    size_t n = kept.size();
    if (n < 2) { g_err = "insufficient observations"; return 2001; }
    for (int t = 0; t < sp->nterms; t++) { std::vector<u32> c; u32 g; restrict_codes(tcodes[t], tg[t], kept, c, g); tcodes[t] = c; tg[t] = g; }
    for (int c = 0; c < sp->ncl; c++) { std::vector<u32> cc; u32 g; restrict_codes(ccodes[c], cg[c], kept, cc, g); ccodes[c] = cc; cg[c] = g; }
    std::vector<double> wk;
    if (sp->w) { wk.resize(n); for (size_t i = 0; i < n; i++) wk[i] = sp->w[kept[i]]; }

    OrcSession sess;
    sess.tcodes = tcodes;
    sess.tg = tg;
    sess.ccodes = ccodes;
    sess.cg = cg;
    sess.n = n;
    sess.nsing = nsing;
    sess.kind = sp->w ? sp->weight_kind : 0;
    sess.wk = wk;
    session_build(sess);
    const auto& pi = sess.ab.st.pi;

    // rows [y, x...] in row order
    size_t nx = sp->nx, r = 1 + nx;
    std::vector<double> rows(n * r);
    for (size_t i = 0; i < n; i++) {
        size_t o = kept[pi[i]];
        rows[i * r] = sp->y[o];
        for (size_t j = 0; j < nx; j++) rows[i * r + 1 + j] = sp->x[j][o];
    }
    int rc = session_ols(sess, rows, nx, OlsArgs{sp->vce, sp->noconstant, sp->firstpair, sp->tol, sp->maxiter}, out);
    if (rc) return rc;
    for (size_t i = 0; i < n0; i++) out->sample[i] = alive[i];
    return 0;
}

// Session entry points (the bench's CPU arm): a prepared session reused across OLS calls.
int orc_session_create(const uint32_t* const* codes, const uint32_t* g, int nterms, const uint32_t* const* cl,
                       const uint32_t* cl_g, int ncl, const double* w, int kind, size_t n, uint64_t nsing,
                       void** out) {
    auto* s = new OrcSession();
    for (int q = 0; q < nterms; q++) {
        s->tcodes.emplace_back(codes[q], codes[q] + n);
        s->tg.push_back(g[q]);
    }
    for (int c = 0; c < ncl; c++) {
        s->ccodes.emplace_back(cl[c], cl[c] + n);
        s->cg.push_back(cl_g[c]);
    }
    if (w) s->wk.assign(w, w + n);
    s->kind = w ? kind : 0;
    s->n = n;
    s->nsing = nsing;
    session_build(*s);
    *out = s;
    return 0;
}

void orc_session_destroy(void* s) { delete static_cast<OrcSession*>(s); }

void orc_session_row_order(const void* s, uint32_t* out) {
    const auto& pi = static_cast<const OrcSession*>(s)->ab.st.pi;
    std::copy(pi.begin(), pi.end(), out);
}

int orc_session_ols(void* s, double* rows, size_t nx, int vce, int noconstant, int firstpair, double tol,
                    size_t maxiter, OrcOlsOut* out) {
    auto* ss = static_cast<OrcSession*>(s);
    std::vector<double> v(rows, rows + ss->n * (1 + nx));
    int rc = session_ols(*ss, v, nx, OlsArgs{vce, noconstant, firstpair, tol, maxiter}, out);
    std::copy(v.begin(), v.end(), rows);
    return rc;
}

}  // extern "C"
