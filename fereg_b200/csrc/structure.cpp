// Cell structure of the intercept-only FE design, built on the host once per sample.
//
// Follows the reference's structure::build (crates/fereg-core/src/structure.rs:247-527): the
// eliminated term (FE1) minimises the assembly work E with three or more terms, the other terms
// are blocks (small ones first while their levels total at most SMALL_LIMIT), rows are sorted by
// (FE1 code, block codes in block order, observation) and cut into cells and segments. The sort
// is a stable LSD counting sort, so equal keys keep observation order; the result is unique and
// therefore identical to the reference's (which sorts per segment in parallel).

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <numeric>

#include "common.h"

namespace fereg {

static thread_local std::string g_last_error;
void set_last_error(const std::string& msg) { g_last_error = msg; }
const char* last_error() { return g_last_error.c_str(); }

void check_codes_host(const std::vector<const u32*>& codes, const std::vector<u32>& g, size_t n) {
    for (size_t q = 0; q < codes.size(); q++) {
        const u32* c = codes[q];
        const u32 gq = g[q];
        int bad = 0;
#pragma omp parallel for reduction(| : bad) schedule(static) if (n > (size_t(1) << 20))
        for (long long i = 0; i < (long long)n; i++) bad |= c[i] >= gq;
        if (bad) throw Error(RC_INVALID_INPUT, "term code out of range of its level count");
    }
}

void check_weights_host(const double* w, size_t n) {
    int bad = 0;
#pragma omp parallel for reduction(| : bad) schedule(static) if (n > (size_t(1) << 20))
    for (long long i = 0; i < (long long)n; i++) bad |= !(std::isfinite(w[i]) && w[i] > 0.0);
    if (bad) throw Error(RC_INVALID_INPUT, "weights must be positive and finite");
}

// absorber.rs:100-108: the intercept-only term with the most levels, first on ties.
int fe1_index(const std::vector<u32>& g) {
    int best = -1;
    for (size_t q = 0; q < g.size(); q++)
        if (best < 0 || g[q] > g[size_t(best)]) best = int(q);
    return best;
}

// Stable counting sort of `ids` by key(id) < g. Above 2^18 ids it runs in parallel: thread t
// counts its contiguous range, then writes it from its own offset in every bucket (after the
// lower-ranked threads' ids), which keeps the order of one sequential pass.
template <class Key>
static void counting_pass(std::vector<u32>& ids, std::vector<u32>& tmp, u32 g, Key key) {
    const size_t n = ids.size();
    const size_t cap = std::max<size_t>(1, (size_t(128) << 20) / (4 * (size_t(g) + 1)));
    const int T = n < (size_t(1) << 18) ? 1 : int(std::min<size_t>({16, size_t(omp_get_max_threads()), cap}));
    std::vector<u32> pos(size_t(T) * g, 0);
    auto lo = [&](int th) { return size_t(n * size_t(th) / size_t(T)); };
#pragma omp parallel num_threads(T)
    {
        const int th = omp_get_thread_num();
        u32* p = pos.data() + size_t(th) * g;
        for (size_t i = lo(th); i < lo(th + 1); i++) p[key(ids[i])]++;
    }
    u32 acc = 0;
    for (u32 k = 0; k < g; k++)
        for (int th = 0; th < T; th++) {
            const u32 v = pos[size_t(th) * g + k];
            pos[size_t(th) * g + k] = acc;
            acc += v;
        }
    tmp.resize(n);
#pragma omp parallel num_threads(T)
    {
        const int th = omp_get_thread_num();
        u32* p = pos.data() + size_t(th) * g;
        for (size_t i = lo(th); i < lo(th + 1); i++) tmp[p[key(ids[i])]++] = ids[i];
    }
    ids.swap(tmp);
}

// structure.rs:256-352 choose_elimination (E = sum over the other terms o and the levels s of
// the candidate of d_{s,o}^2, d the distinct levels of o within s).
static int choose_elimination(const std::vector<const u32*>& codes, const std::vector<u32>& g, size_t n) {
    const int f0 = fe1_index(g);
    if (f0 < 0 || codes.size() < 3) return f0;
    std::vector<size_t> cands;
    for (size_t q = 0; q < g.size(); q++)
        if (size_t(g[q]) * 4 >= g[size_t(f0)]) cands.push_back(q);
    if (cands.size() < 2) return f0;
    std::vector<u64> size(g[size_t(f0)], 0);
    for (size_t i = 0; i < n; i++) size[codes[size_t(f0)][i]]++;
    u64 bound = 0;
    for (u64 s : size) bound += s * s;
    bound *= u64(codes.size() - 1);
    if (bound <= 64 * u64(n)) return f0;
    bool have = false;
    u64 best_e = 0;
    u32 best_g = 0;
    size_t best_f = 0;
    for (size_t f : cands) {
        std::vector<u32> off(size_t(g[f]) + 1, 0), ids(n);
        for (size_t i = 0; i < n; i++) off[codes[f][i] + 1]++;
        for (u32 k = 0; k < g[f]; k++) off[k + 1] += off[k];
        {
            std::vector<u32> cur(off.begin(), off.end() - 1);
            for (size_t i = 0; i < n; i++) ids[cur[codes[f][i]]++] = u32(i);
        }
        u64 e = 0;
        for (size_t o = 0; o < codes.size(); o++) {
            if (o == f) continue;
            std::vector<u32> stamp(g[o], 0);
            for (u32 s = 0; s < g[f]; s++) {
                u64 d = 0;
                for (u32 p = off[s]; p < off[s + 1]; p++) {
                    u32 c = codes[o][ids[p]];
                    if (stamp[c] != s + 1) { stamp[c] = s + 1; d++; }
                }
                e += d * d;
            }
        }
        bool better = !have || e < best_e || (e == best_e && (g[f] > best_g || (g[f] == best_g && f < best_f)));
        if (better) { have = true; best_e = e; best_g = g[f]; best_f = f; }
    }
    return int(best_f);
}

HostStructure plan_structure(const std::vector<const u32*>& codes, const std::vector<u32>& g, size_t n,
                             size_t small_limit) {
    HostStructure st;
    st.n = n;
    st.fe1 = choose_elimination(codes, g, n);
    st.g1 = st.fe1 >= 0 ? g[size_t(st.fe1)] : 1;

    // Small/large classification: ascending G (term index on ties) while the total stays within
    // small_limit (structure.rs:366-378); small blocks first, then large, each in term order.
    std::vector<size_t> others;
    for (size_t q = 0; q < g.size(); q++)
        if (int(q) != st.fe1) others.push_back(q);
    std::vector<size_t> by_g = others;
    std::stable_sort(by_g.begin(), by_g.end(), [&](size_t a, size_t b) { return g[a] < g[b]; });
    std::vector<bool> small(g.size(), false);
    size_t total = 0;
    for (size_t q : by_g) {
        if (total + g[q] > small_limit) break;
        total += g[q];
        small[q] = true;
    }
    u32 off = 0;
    for (int pass = 0; pass < 2; pass++)
        for (size_t q : others)
            if (small[q] == (pass == 0)) {
                st.blocks.push_back({u32(q), g[q], off, bool(small[q])});
                off += g[q];
            }
    st.m = off;
    for (auto& b : st.blocks)
        if (b.small) st.m_small += b.g;
    return st;
}

HostStructure build_structure(const std::vector<const u32*>& codes, const std::vector<u32>& g, size_t n,
                              size_t small_limit) {
    HostStructure st = plan_structure(codes, g, n, small_limit);
    const size_t nb = st.blocks.size();

    // Rows by (FE1, block codes, obs): check the order first (panels usually arrive sorted).
    auto key_less_eq = [&](u32 a, u32 b) {  // key(a) <= key(b), ignoring obs
        if (st.fe1 >= 0) {
            u32 ca = codes[size_t(st.fe1)][a], cb = codes[size_t(st.fe1)][b];
            if (ca != cb) return ca < cb;
        }
        for (size_t k = 0; k < nb; k++) {
            u32 ca = codes[st.blocks[k].term][a], cb = codes[st.blocks[k].term][b];
            if (ca != cb) return ca < cb;
        }
        return true;
    };
    const int T = n < (size_t(1) << 18) ? 1 : std::min(16, omp_get_max_threads());
    auto lo = [&](int th) { return size_t(n * size_t(th) / size_t(T)); };
    int unsorted = 0;
#pragma omp parallel for num_threads(T) reduction(| : unsorted) schedule(static)
    for (long long i = 1; i < (long long)n; i++)
        if (!key_less_eq(u32(i - 1), u32(i))) unsorted = 1;
    st.pi.resize(n);
    std::iota(st.pi.begin(), st.pi.end(), 0u);
    if (unsorted) {
        std::vector<u32> tmp;
        for (size_t k = nb; k-- > 0;) {
            const u32* c = codes[st.blocks[k].term];
            counting_pass(st.pi, tmp, st.blocks[k].g, [c](u32 i) { return c[i]; });
        }
        if (st.fe1 >= 0) {
            const u32* c = codes[size_t(st.fe1)];
            counting_pass(st.pi, tmp, st.g1, [c](u32 i) { return c[i]; });
        }
    }

    // Cells and segments: a row opens a cell when its key differs from the previous row's. Thread
    // t cuts its own range of rows (the first compared with the row before the range), then
    // writes its cells at the offset of the cells of the lower-ranked threads.
    const u32* c1 = st.fe1 >= 0 ? codes[size_t(st.fe1)] : nullptr;
    auto opens = [&](size_t r) {
        if (r == 0) return true;
        const u32 o = st.pi[r], p = st.pi[r - 1];
        if (c1 && c1[o] != c1[p]) return true;
        for (size_t k = 0; k < nb; k++)
            if (codes[st.blocks[k].term][o] != codes[st.blocks[k].term][p]) return true;
        return false;
    };
    std::vector<size_t> tcells(size_t(T) + 1, 0);
#pragma omp parallel num_threads(T)
    {
        const int th = omp_get_thread_num();
        size_t cnt = 0;
        for (size_t r = lo(th); r < lo(th + 1); r++) cnt += opens(r) ? 1 : 0;
        tcells[size_t(th) + 1] = cnt;
    }
    for (int th = 0; th < T; th++) tcells[size_t(th) + 1] += tcells[size_t(th)];
    st.ncells = tcells[size_t(T)];
    const size_t M = st.ncells;
    std::vector<u32> starts(M);
    st.coord.resize(nb * M);
    std::vector<u32> cseg(M);  // FE1 level of every cell
#pragma omp parallel num_threads(T)
    {
        const int th = omp_get_thread_num();
        size_t c = tcells[size_t(th)];
        for (size_t r = lo(th); r < lo(th + 1); r++)
            if (opens(r)) {
                const u32 o = st.pi[r];
                starts[c] = u32(r);
                cseg[c] = c1 ? c1[o] : 0;
                for (size_t k = 0; k < nb; k++) st.coord[k * M + c] = st.blocks[k].off + codes[st.blocks[k].term][o];
                c++;
            }
    }
    st.seg_off.assign(size_t(st.g1) + 1, 0);
    for (size_t c = 0; c < M; c++) st.seg_off[size_t(cseg[c]) + 1]++;
    for (u32 s = 0; s < st.g1; s++) st.seg_off[s + 1] += st.seg_off[s];
    if (M != n) {
        st.cell_row = std::move(starts);
        st.cell_row.push_back(u32(n));
    }

    // Dense small-block work sum_s (distinct small coordinates)^2 (structure.rs:521-525).
    if (st.m_small > 0) {
        u64 work = 0;
#pragma omp parallel num_threads(T) reduction(+ : work)
        {
            std::vector<u32> mark(st.m_small, 0);
#pragma omp for schedule(static)
            for (long long s = 0; s < (long long)st.g1; s++) {
                u64 d = 0;
                for (u32 c = st.seg_off[size_t(s)]; c < st.seg_off[size_t(s) + 1]; c++)
                    for (size_t k = 0; k < nb; k++) {
                        if (!st.blocks[k].small) continue;
                        u32 x = st.coord[k * st.ncells + c];
                        if (mark[x] != u32(s) + 1) {
                            mark[x] = u32(s) + 1;
                            d++;
                        }
                    }
                work += d * d;
            }
        }
        st.small_work = work;
        if (work > 64 * u64(st.ncells)) {
            for (auto& b : st.blocks) b.small = false;
            st.m_small = 0;
        }
    }
    return st;
}

// A stable parallel counting sort: thread t takes a contiguous range of cells, counts its
// entries per coordinate, and writes them from its own offset in every list (the entries of
// lower-ranked threads, hence of earlier cells, come first), so every list is in cell order
// exactly as in one pass over the cells.
PullTable build_pull_table(const HostStructure& st) {
    PullTable t;
    const size_t nb = st.nb(), M = st.ncells, m = st.m;
    const size_t E = M * nb, no = nb > 0 ? nb - 1 : 0;
    t.off.assign(m + 1, 0);
    t.cell.resize(E);
    t.seg.resize(E);
    t.other.resize(E * no);
    if (E == 0) return t;
    std::vector<u32> cseg(M);  // segment of every cell
#pragma omp parallel for schedule(static)
    for (long long s = 0; s < (long long)st.g1; s++)
        for (u32 c = st.seg_off[size_t(s)]; c < st.seg_off[size_t(s) + 1]; c++) cseg[c] = u32(s);
    const size_t cap = std::max<size_t>(1, (size_t(128) << 20) / (4 * std::max<size_t>(1, m)));
    const int T = E < (size_t(1) << 20) ? 1 : int(std::min<size_t>({16, size_t(omp_get_max_threads()), cap}));
    std::vector<u32> pos(size_t(T) * m, 0);  // per thread: count, then first write position per list
    auto lo = [&](int th) { return size_t(M * size_t(th) / size_t(T)); };
#pragma omp parallel num_threads(T)
    {
        const int th = omp_get_thread_num();
        u32* p = pos.data() + size_t(th) * m;
        for (size_t c = lo(th); c < lo(th + 1); c++)
            for (size_t k = 0; k < nb; k++) p[st.coord[k * M + c]]++;
    }
    for (size_t x = 0; x < m; x++) {
        u32 acc = 0;
        for (int th = 0; th < T; th++) {
            const u32 v = pos[size_t(th) * m + x];
            pos[size_t(th) * m + x] = acc;
            acc += v;
        }
        t.off[x + 1] = acc;
    }
    for (size_t x = 0; x < m; x++) t.off[x + 1] += t.off[x];
#pragma omp parallel num_threads(T)
    {
        const int th = omp_get_thread_num();
        u32* p = pos.data() + size_t(th) * m;
        for (size_t c = lo(th); c < lo(th + 1); c++)
            for (size_t k = 0; k < nb; k++) {
                const u32 x = st.coord[k * M + c];
                const u32 e = t.off[x] + p[x]++;
                t.cell[e] = u32(c);
                t.seg[e] = cseg[c];
                size_t o = 0;
                for (size_t k2 = 0; k2 < nb; k2++)
                    if (k2 != k) t.other[size_t(e) * no + o++] = st.coord[k2 * M + c];
            }
    }
    return t;
}

TileList build_tiles(const std::vector<u32>& off, u32 k_begin, u32 k_end, u32 cap, u32 min_len) {
    TileList it;
    u32 k = k_begin;
    while (k < k_end) {
        const u32 cnt = off[k + 1] - off[k];
        if (cnt <= min_len) {  // left to the one-thread-per-list kernels
            k++;
            continue;
        }
        if (cnt > cap) {
            const u32 np = (cnt + cap - 1) / cap;
            const int32_t f = int32_t(it.fix_k.size());
            it.fix_k.push_back(k);
            it.fix_p0.push_back(it.nparts);
            it.fix_np.push_back(np);
            for (u32 p = 0; p < np; p++) {
                it.k0.push_back(k);
                it.k1.push_back(k + 1);
                it.e0.push_back(off[k] + p * cap);
                it.e1.push_back(std::min(off[k] + (p + 1) * cap, off[k + 1]));
                it.part.push_back(int32_t(it.nparts + p));
                it.fixidx.push_back(f);
            }
            it.nparts += np;
            k++;
            continue;
        }
        u32 k1 = k, tot = 0;
        while (k1 < k_end) {
            const u32 c = off[k1 + 1] - off[k1];
            if (c <= min_len || c > cap || (tot + c > cap && k1 > k)) break;
            tot += c;
            k1++;
        }
        it.k0.push_back(k);
        it.k1.push_back(k1);
        it.e0.push_back(off[k]);
        it.e1.push_back(off[k1]);
        it.part.push_back(-1);
        it.fixidx.push_back(-1);
        k = k1;
    }
    return it;
}

}  // namespace fereg

namespace fereg {

void split_tiles(const std::vector<u32>& off, const std::vector<u32>* weight, u32 k_begin, u32 k_end, u32 warp_max,
                 u32 pack, u32 max_lists, u32 cta_cap, WarpTileList& wt, TileList& ct) {
    auto wgt = [&](u32 k) { return weight ? (*weight)[k] : off[k + 1] - off[k]; };
    // warp tiles: consecutive lists of weight <= warp_max, packed while the total stays <= pack
    u32 k = k_begin;
    while (k < k_end) {
        if (wgt(k) > warp_max) {
            k++;
            continue;
        }
        u32 k1 = k, tot = 0;
        while (k1 < k_end) {
            const u32 w = wgt(k1);
            if (w > warp_max || (k1 > k && (tot + w > pack || k1 - k >= max_lists))) break;
            tot += w;
            k1++;
        }
        wt.k0.push_back(k);
        wt.k1.push_back(k1);
        wt.e0.push_back(off[k]);
        wt.e1.push_back(off[k1]);
        k = k1;
    }
    // CTA tiles over the others (lists longer than warp_max by weight)
    k = k_begin;
    while (k < k_end) {
        if (wgt(k) <= warp_max) {
            k++;
            continue;
        }
        const u32 cnt = off[k + 1] - off[k];
        if (cnt > cta_cap) {
            const u32 np = (cnt + cta_cap - 1) / cta_cap;
            const int32_t f = int32_t(ct.fix_k.size());
            ct.fix_k.push_back(k);
            ct.fix_p0.push_back(ct.nparts);
            ct.fix_np.push_back(np);
            for (u32 p = 0; p < np; p++) {
                ct.k0.push_back(k);
                ct.k1.push_back(k + 1);
                ct.e0.push_back(off[k] + p * cta_cap);
                ct.e1.push_back(std::min(off[k] + (p + 1) * cta_cap, off[k + 1]));
                ct.part.push_back(int32_t(ct.nparts + p));
                ct.fixidx.push_back(f);
            }
            ct.nparts += np;
            k++;
            continue;
        }
        u32 k1 = k, tot = 0;
        while (k1 < k_end) {
            const u32 c = off[k1 + 1] - off[k1];
            if (wgt(k1) <= warp_max || c > cta_cap || (tot + c > cta_cap && k1 > k)) break;
            tot += c;
            k1++;
        }
        ct.k0.push_back(k);
        ct.k1.push_back(k1);
        ct.e0.push_back(off[k]);
        ct.e1.push_back(off[k1]);
        ct.part.push_back(-1);
        ct.fixidx.push_back(-1);
        k = k1;
    }
}

}  // namespace fereg
