// Smoothed-aggregation multigrid hierarchy of an escalated large block (see amg.h). Host setup;
// the V-cycle runs on the device (amg.cuh).
#include "amg.h"

#include <algorithm>
#include <cmath>

namespace fereg {

namespace {

// CSR rows produced by parallel row passes: row i's ascending (column, value) pairs.
struct RowLists {
    std::vector<std::vector<u32>> c;
    std::vector<std::vector<double>> v;
    explicit RowLists(size_t n) : c(n), v(n) {}
    Csr to_csr(u32 ncols) const {
        Csr M;
        M.nr = u32(c.size());
        M.nc = ncols;
        M.ptr.assign(c.size() + 1, 0);
        for (size_t i = 0; i < c.size(); i++) M.ptr[i + 1] = M.ptr[i] + u32(c[i].size());
        M.col.resize(M.ptr.back());
        M.val.resize(M.ptr.back());
        for (size_t i = 0; i < c.size(); i++) {
            std::copy(c[i].begin(), c[i].end(), M.col.begin() + M.ptr[i]);
            std::copy(v[i].begin(), v[i].end(), M.val.begin() + M.ptr[i]);
        }
        return M;
    }
};

// Sparse accumulator of one row: the touched columns ascending with their values, then reset.
void flush_row(std::vector<double>& acc, std::vector<u32>& touched, std::vector<char>& seen, std::vector<u32>& cols,
               std::vector<double>& vals, double scale) {
    std::sort(touched.begin(), touched.end());
    for (u32 l : touched) {
        cols.push_back(l);
        vals.push_back(scale * acc[l]);
        acc[l] = 0.0;
        seen[l] = 0;
    }
    touched.clear();
}

// C = A B (row by row, sparse accumulator per thread).
Csr spgemm(const Csr& A, const Csr& B) {
    RowLists rl(A.nr);
#pragma omp parallel
    {
        std::vector<double> acc(B.nc, 0.0);
        std::vector<char> seen(B.nc, 0);
        std::vector<u32> touched;
#pragma omp for schedule(dynamic, 64)
        for (long long ii = 0; ii < (long long)A.nr; ii++) {
            const u32 i = u32(ii);
            for (u32 e = A.ptr[i]; e < A.ptr[i + 1]; e++) {
                const u32 k = A.col[e];
                const double a = A.val[e];
                for (u32 f = B.ptr[k]; f < B.ptr[k + 1]; f++) {
                    const u32 j = B.col[f];
                    if (!seen[j]) {
                        seen[j] = 1;
                        touched.push_back(j);
                    }
                    acc[j] += a * B.val[f];
                }
            }
            flush_row(acc, touched, seen, rl.c[i], rl.v[i], 1.0);
        }
    }
    return rl.to_csr(B.nc);
}

Csr transpose(const Csr& A) {
    Csr T;
    T.nr = A.nc;
    T.nc = A.nr;
    T.ptr.assign(size_t(A.nc) + 1, 0);
    for (u32 c : A.col) T.ptr[c + 1]++;
    for (u32 j = 0; j < A.nc; j++) T.ptr[j + 1] += T.ptr[j];
    T.col.resize(A.col.size());
    T.val.resize(A.col.size());
    std::vector<u32> pos(T.ptr.begin(), T.ptr.end() - 1);
    for (u32 i = 0; i < A.nr; i++)
        for (u32 e = A.ptr[i]; e < A.ptr[i + 1]; e++) {
            const u32 t = pos[A.col[e]]++;
            T.col[t] = i;
            T.val[t] = A.val[e];
        }
    return T;
}

std::vector<double> diagonal(const Csr& A) {
    std::vector<double> d(A.nr, 0.0);
    for (u32 i = 0; i < A.nr; i++)
        for (u32 e = A.ptr[i]; e < A.ptr[i + 1]; e++)
            if (A.col[e] == i) d[i] = A.val[e];
    return d;
}

void set_dinv(AmgLevel& L, const std::vector<bool>& out) {
    const std::vector<double> d = diagonal(L.A);
    L.dinv.assign(L.n, 0.0);
    for (u32 i = 0; i < L.n; i++)
        if (!out[i] && d[i] > 0.0) L.dinv[i] = AMG_OMEGA / d[i];
}

// S_bb of block b (operator.rs:2054 assemble_block): for each level k, the cells of k, their
// segments, and every cell of those segments; off-diagonal -c_k c_l / n1, the diagonal from the
// weight state.
AmgLevel assemble_block(const HostStructure& hs, size_t b, const double* cw, const double* n1, const double* diag,
                        const uint8_t* red) {
    const Block& B = hs.blocks[b];
    const u32 g = B.g, off = B.off;
    const size_t M = hs.ncells;
    const u32* coord = hs.coord.data() + b * M;
    std::vector<u32> seg(M);
    for (u32 s = 0; s < hs.g1; s++)
        for (u32 c = hs.seg_off[s]; c < hs.seg_off[s + 1]; c++) seg[c] = s;
    std::vector<u32> loff(size_t(g) + 1, 0), lcell(M);
    for (size_t c = 0; c < M; c++) loff[coord[c] - off + 1]++;
    for (u32 k = 0; k < g; k++) loff[k + 1] += loff[k];
    {
        std::vector<u32> pos(loff.begin(), loff.end() - 1);
        for (size_t c = 0; c < M; c++) lcell[pos[coord[c] - off]++] = u32(c);
    }
    std::vector<bool> out(g);
    for (u32 k = 0; k < g; k++) out[k] = red[off + k] || !(diag[off + k] > 0.0);
    RowLists rl(g);
#pragma omp parallel
    {
        std::vector<double> acc(g, 0.0);
        std::vector<char> seen(g, 0);
        std::vector<u32> touched;
#pragma omp for schedule(dynamic, 64)
        for (long long kk = 0; kk < (long long)g; kk++) {
            const u32 k = u32(kk);
            if (out[k]) continue;  // a left-out coordinate: an empty row
            for (u32 e = loff[k]; e < loff[k + 1]; e++) {
                const u32 c = lcell[e], s = seg[c];
                const double f = (cw ? cw[c] : 1.0) / n1[s];
                for (u32 c2 = hs.seg_off[s]; c2 < hs.seg_off[s + 1]; c2++) {
                    const u32 l = coord[c2] - off;
                    if (l == k || out[l]) continue;
                    if (!seen[l]) {
                        seen[l] = 1;
                        touched.push_back(l);
                    }
                    acc[l] -= f * (cw ? cw[c2] : 1.0);
                }
            }
            seen[k] = 1;
            touched.push_back(k);
            acc[k] = diag[off + k];
            flush_row(acc, touched, seen, rl.c[k], rl.v[k], 1.0);
        }
    }
    AmgLevel L;
    L.n = g;
    L.A = rl.to_csr(g);
    set_dinv(L, out);
    return L;
}

// Plain aggregation: roots in node order whose strong neighbours are all free take up to 7 of
// them (strongest first); free nodes then join the aggregate of their strongest aggregated
// neighbour; nodes left over start aggregates of their own. Left-out nodes (dinv 0) get -1.
u32 aggregate(const AmgLevel& L, std::vector<int>& agg) {
    const Csr& A = L.A;
    const u32 n = L.n;
    constexpr int FREE = -2;
    agg.assign(n, FREE);
    std::vector<double> smax(n, 0.0);
    for (u32 i = 0; i < n; i++) {
        if (L.dinv[i] == 0.0) {
            agg[i] = -1;
            continue;
        }
        for (u32 e = A.ptr[i]; e < A.ptr[i + 1]; e++)
            if (A.col[e] != i) smax[i] = std::max(smax[i], std::fabs(A.val[e]));
    }
    u32 nc = 0;
    std::vector<std::pair<double, u32>> cand;
    for (u32 i = 0; i < n; i++) {
        if (agg[i] != FREE) continue;
        bool ok = true;
        cand.clear();
        for (u32 e = A.ptr[i]; e < A.ptr[i + 1] && ok; e++) {
            const u32 j = A.col[e];
            if (j == i || std::fabs(A.val[e]) < 0.25 * smax[i]) continue;
            if (agg[j] >= 0) ok = false;
            else if (agg[j] == FREE) cand.push_back({-std::fabs(A.val[e]), j});
        }
        if (!ok) continue;
        std::sort(cand.begin(), cand.end());
        agg[i] = int(nc);
        for (size_t t = 0; t < cand.size() && t < 7; t++) agg[cand[t].second] = int(nc);
        nc++;
    }
    const std::vector<int> snap(agg);
    for (u32 i = 0; i < n; i++) {
        if (agg[i] != FREE) continue;
        double best = 0.0;
        int to = FREE;
        for (u32 e = A.ptr[i]; e < A.ptr[i + 1]; e++) {
            const u32 j = A.col[e];
            if (j == i || snap[j] < 0) continue;
            if (std::fabs(A.val[e]) > best) {
                best = std::fabs(A.val[e]);
                to = snap[j];
            }
        }
        agg[i] = to;
    }
    for (u32 i = 0; i < n; i++)
        if (agg[i] == FREE) agg[i] = int(nc++);
    return nc;
}

// P = (I - (2/3) D^-1 A) P0 for the piecewise-constant P0 of `agg` (rows of left-out nodes empty).
Csr smoothed_prolongation(const AmgLevel& L, const std::vector<int>& agg, u32 nc) {
    Csr P0;
    P0.nr = L.n;
    P0.nc = nc;
    P0.ptr.assign(size_t(L.n) + 1, 0);
    for (u32 i = 0; i < L.n; i++) {
        P0.ptr[i + 1] = P0.ptr[i];
        if (agg[i] >= 0) {
            P0.col.push_back(u32(agg[i]));
            P0.val.push_back(1.0);
            P0.ptr[i + 1]++;
        }
    }
    Csr AP = spgemm(L.A, P0);
    const std::vector<double> d = diagonal(L.A);
    RowLists rl(L.n);
#pragma omp parallel
    {
        std::vector<double> acc(nc, 0.0);
        std::vector<char> seen(nc, 0);
        std::vector<u32> touched;
#pragma omp for schedule(dynamic, 256)
        for (long long ii = 0; ii < (long long)L.n; ii++) {
            const u32 i = u32(ii);
            if (agg[i] < 0 || !(d[i] > 0.0)) continue;
            const double f = (2.0 / 3.0) / d[i];
            for (u32 e = AP.ptr[i]; e < AP.ptr[i + 1]; e++) {
                const u32 j = AP.col[e];
                if (!seen[j]) {
                    seen[j] = 1;
                    touched.push_back(j);
                }
                acc[j] -= f * AP.val[e];
            }
            const u32 a = u32(agg[i]);
            if (!seen[a]) {
                seen[a] = 1;
                touched.push_back(a);
            }
            acc[a] += 1.0;
            flush_row(acc, touched, seen, rl.c[i], rl.v[i], 1.0);
        }
    }
    return rl.to_csr(nc);
}

}  // namespace

AmgHierarchy amg_build(const HostStructure& hs, size_t block, const double* cell_w, const double* n1,
                       const double* diag, const uint8_t* red) {
    AmgHierarchy H;
    H.block = u32(block);
    H.levels.push_back(assemble_block(hs, block, cell_w, n1, diag, red));
    while (H.levels.back().n > AMG_COARSE) {
        AmgLevel& fine = H.levels.back();
        std::vector<int> agg;
        const u32 nc = aggregate(fine, agg);
        if (nc == 0 || size_t(nc) * 10 > size_t(fine.n) * 9) break;  // aggregation stalled: stop here
        fine.P = smoothed_prolongation(fine, agg, nc);
        fine.Pt = transpose(fine.P);
        AmgLevel C;
        C.n = nc;
        C.A = spgemm(fine.Pt, spgemm(fine.A, fine.P));
        std::vector<bool> out(nc, false);
        set_dinv(C, out);
        H.levels.push_back(std::move(C));
    }
    // the coarsest level as a dense matrix (its generalized inverse is formed on the device)
    const AmgLevel& L = H.levels.back();
    H.coarse.assign(size_t(L.n) * L.n, 0.0);
    for (u32 i = 0; i < L.n; i++)
        for (u32 e = L.A.ptr[i]; e < L.A.ptr[i + 1]; e++) H.coarse[size_t(i) * L.n + L.A.col[e]] = L.A.val[e];
    return H;
}

}  // namespace fereg
