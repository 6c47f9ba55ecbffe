// Warp-tile kernels for the short lists: segments of at most WT cells (and WT rows) and
// coordinate lists of at most PULL_WARP_MAX entries. Longer lists go to the CTA tiles
// (tiles.cuh).
//
// A warp takes one warp tile at a time (whole consecutive segments with at most WT cells and WT
// rows in all, or whole consecutive coordinate lists): lanes first load the tile's indices (one
// lane per cell or entry, coalesced) and, in the row passes, the tile's rows (flat, coalesced)
// into the warp's shared memory; then lanes (group, column) gather the reduced vectors with all
// gathers of a round in flight, and sums run per column in list order. Warps never wait on each
// other inside the loop. Column blocks wider than WCOLS are launched per column chunk.
//
// The small coordinates (when summed in the segment passes) accumulate in the warp's shared
// memory with each column owned by one lane; at the end the CTA adds its warps in warp order into
// its own partial row. All sums have a fixed order: results do not depend on timing.
#pragma once

#include "tiles.cuh"

namespace fereg {

constexpr int WT = 32;                 // cells (rows) per warp tile
constexpr int WCOLS = 32;              // columns per launch of the warp kernels
constexpr int WPB = 8;                 // warps per CTA
constexpr u32 PULL_WARP_MAX = 8192;    // entries of one coordinate list walked by one warp
constexpr int LMAX = WT;               // segments up to this many cells use the warp tiles
constexpr u32 PULL_THR_MAX = PULL_WARP_MAX;

// Warp tiles over short lists.
struct WarpTiles {
    u32 n;
    const u32* k0;
    const u32* k1;
    const u32* e0;
    const u32* e1;
};

__device__ __forceinline__ u32 wlane() { return threadIdx.x & 31u; }
__device__ __forceinline__ u32 wid_in_cta() { return threadIdx.x >> 5; }

// Lane layout over (group, column) for a chunk of Rc <= 32 columns: G = 32 / Rc groups.
struct GMap {
    int Rc, G, g, j;
    bool on;
};
__device__ __forceinline__ GMap gmap(int Rc) {
    const int G = 32 / Rc;
    const int l = int(wlane());
    return {Rc, G, l / Rc, l % Rc, l < G * Rc};
}

// Sum of v over the groups holding the same column, groups in order (all lanes get the sum;
// inactive lanes must hold 0).
template <class T>
__device__ __forceinline__ T group_sum(T v, const GMap& m) {
    if (m.G == 1) return v;
    T s = T(0);
    for (int g = 0; g < m.G; g++) s += __shfl_sync(FULL, v, g * m.Rc + m.j);
    return s;
}

// Per-warp shared memory, laid out for a column chunk of Rc columns (sizes in bytes, 16-byte
// aligned parts): the per-cell vectors first, then the per-cell indices.
__host__ __device__ constexpr size_t al16(size_t b) { return (b + 15) / 16 * 16; }
__host__ __device__ constexpr size_t idx_bytes() { return al16(WT * 8) + al16(4 * WT * 4) + al16(WT * 4) + al16((WT + 1) * 4); }
// segment kernels: u (per-cell, T)
__host__ __device__ constexpr size_t wseg_bytes(int Rc, size_t tsz) { return al16(WT * Rc * tsz) + idx_bytes(); }
// row kernels: v (the tile's rows), u (per cell), both double, + row weights
__host__ __device__ constexpr size_t wrows_bytes(int Rc) { return 2 * al16(WT * Rc * 8) + al16(WT * 8) + idx_bytes(); }

template <class T>
struct WSeg {
    T* u;
    double* cw;
    u32* code;
    u32* segl;
    u32* row0;
};

template <class T>
__device__ __forceinline__ WSeg<T> wseg_at(unsigned char* base, int Rc) {
    unsigned char* p = base + size_t(wid_in_cta()) * wseg_bytes(Rc, sizeof(T));
    WSeg<T> w;
    w.u = reinterpret_cast<T*>(p);
    p += al16(WT * Rc * sizeof(T));
    w.cw = reinterpret_cast<double*>(p);
    p += al16(WT * 8);
    w.code = reinterpret_cast<u32*>(p);
    p += al16(4 * WT * 4);
    w.segl = reinterpret_cast<u32*>(p);
    p += al16(WT * 4);
    w.row0 = reinterpret_cast<u32*>(p);
    return w;
}

// CTA end: adds the warps' small-coordinate accumulators (wacc, ms_acc x Rc per warp) in warp
// order into the CTA's partial row.
template <class T>
__device__ __forceinline__ void flush_wacc(const T* wacc_all, u32 ms_acc, int Rc, int j0, int R, T* cta_small) {
    __syncthreads();
    T* mine = cta_small + size_t(blockIdx.x) * ms_acc * R;
    for (u32 i = threadIdx.x; i < ms_acc * u32(Rc); i += blockDim.x) {
        T s = T(0);
        for (int w = 0; w < WPB; w++) s += wacc_all[size_t(w) * ms_acc * Rc + i];
        mine[size_t(i / Rc) * R + j0 + i % Rc] = s;
    }
}

// Loads the tile's per-cell indices into the warp's shared memory (lane = cell).
template <class T>
__device__ __forceinline__ void load_cells(const DevStruct& S, const DevWeights& W, u32 c0, u32 c1, u32 s0,
                                           const WSeg<T>& sm) {
    const u32 lane = wlane();
    const u32 c = c0 + lane;
    if (c < c1) {
        sm.cw[lane] = cellw(W, c);
        for (u32 b = 0; b < S.nb && b < 4; b++) sm.code[b * WT + lane] = __ldcs(S.coord + size_t(b) * S.M + c);
        u32 s = s0;
        while (S.seg_off[s + 1] <= c) s++;
        sm.segl[lane] = s - s0;
    }
    __syncwarp();
}

// ---------------------------------------------------------------------------------------------
// Operator pass 1 (operator.rs:894-948) on short segments: t_s = sum_c W_c u_c / n1_s with
// u_c = sum_b P[coord_b(c)]; small coordinates: sum of W_c (u_c - t_s) per small code.
template <class T>
__global__ void __launch_bounds__(WPB * 32) k_wseg_apply(DevStruct S, DevWeights W, WarpTiles wt, const T* __restrict__ P,
                                                         int R, int j0, int Rc, T* __restrict__ t,
                                                         T* __restrict__ cta_small) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const WSeg<T> sm = wseg_at<T>(smem_raw, Rc);
    T* wacc_all = reinterpret_cast<T*>(smem_raw + WPB * wseg_bytes(Rc, sizeof(T)));
    T* wacc = wacc_all + size_t(wid_in_cta()) * S.ms_acc * Rc;
    const bool acc = cta_small != nullptr;
    const u32 lane = wlane();
    if (acc)
        for (u32 i = lane; i < S.ms_acc * u32(Rc); i += 32) wacc[i] = T(0);
    const GMap gm = gmap(Rc);
    const u32 wid = blockIdx.x * WPB + wid_in_cta(), nw = gridDim.x * WPB;
    for (u32 tile = wid; tile < wt.n; tile += nw) {
        const u32 s0 = wt.k0[tile], s1 = wt.k1[tile], c0 = wt.e0[tile], c1 = wt.e1[tile];
        const u32 nc = c1 - c0;
        load_cells(S, W, c0, c1, s0, sm);
        // gathers: lane (g, j) over cells i = g, g+G, ...
        if (gm.on) {
#pragma unroll 4
            for (u32 i = gm.g; i < nc; i += gm.G) {
                T v = T(0);
                for (u32 b = 0; b < S.nb; b++) v += P[size_t(sm.code[b * WT + i]) * R + j0 + gm.j];
                sm.u[i * Rc + gm.j] = T(sm.cw[i]) * v;
            }
        }
        __syncwarp();
        // per segment, column sums in cell order (lane = column)
        for (u32 jj = lane; jj < u32(Rc); jj += 32) {
            u32 i = 0;
            for (u32 s = s0; s < s1; s++) {
                const u32 e = S.seg_off[s + 1] - c0;
                T sum = T(0);
                const u32 ib = i;
                for (; i < e; i++) sum += sm.u[i * Rc + jj];
                const T tsv = sum * T(W.n1inv[s]);
                t[size_t(s) * R + j0 + jj] = tsv;
                if (acc)
                    for (u32 q = ib; q < e; q++) {
                        const T z = sm.u[q * Rc + jj] - T(sm.cw[q]) * tsv;
                        for (u32 b = 0; b < S.ns_acc; b++) wacc[sm.code[b * WT + q] * Rc + jj] += z;
                    }
            }
        }
        __syncwarp();
    }
    if (acc) flush_wacc(wacc_all, S.ms_acc, Rc, j0, R, cta_small);
}

// Operator pass 2 on short coordinate lists (k >= ms_acc): Y[k] = nr_k P[k] + sum over the cells
// c of k of W_c (sum_{other b} P[coord_b(c)] - t_{s(c)}). Lanes (g, j) walk the entries of a
// round (indices prefetched by lane = entry), groups combined in order per coordinate.
template <class T>
__global__ void __launch_bounds__(WPB * 32) k_wpull_apply(DevStruct S, DevWeights W, WarpTiles wt,
                                                          const T* __restrict__ P, const T* __restrict__ t, int R,
                                                          int j0, int Rc, T* __restrict__ Y) {
    __shared__ u32 seg_s[WPB][32];
    __shared__ u32 oth_s[WPB][3 * 32];
    __shared__ double w_s[WPB][32];
    const u32 wi = wid_in_cta(), lane = wlane();
    const GMap gm = gmap(Rc);
    const u32 no = S.nb - 1;
    const u32 wid = blockIdx.x * WPB + wi, nw = gridDim.x * WPB;
    for (u32 tile = wid; tile < wt.n; tile += nw) {
        const u32 k0 = wt.k0[tile], k1 = wt.k1[tile];
        for (u32 k = k0; k < k1; k++) {
            const u32 a = S.pl_off[k], b = S.pl_off[k + 1];
            T acc = T(0);
            for (u32 base = a; base < b; base += 32) {
                const u32 e = base + lane;
                if (e < b) {
                    seg_s[wi][lane] = __ldcs(S.pl_seg + e);
                    for (u32 o = 0; o < no && o < 3; o++) oth_s[wi][o * 32 + lane] = __ldcs(S.pl_other + size_t(e) * no + o);
                    w_s[wi][lane] = W.cell_w ? W.cell_w[__ldcs(S.pl_cell + e)] : 1.0;
                }
                __syncwarp();
                const u32 cnt = min(32u, b - base);
                if (gm.on) {
#pragma unroll 8
                    for (u32 i = gm.g; i < cnt; i += gm.G) {
                        T u = -__ldcg(t + size_t(seg_s[wi][i]) * R + j0 + gm.j);
                        for (u32 o = 0; o < no; o++) u += P[size_t(oth_s[wi][o * 32 + i]) * R + j0 + gm.j];
                        acc += T(w_s[wi][i]) * u;
                    }
                }
                __syncwarp();
            }
            acc = group_sum(acc, gm);
            if (gm.on && gm.g == 0) {
                const size_t o = size_t(k) * R + j0 + gm.j;
                Y[o] = T(W.nr[k]) * P[o] + acc;
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Per-warp shared memory of the row passes (wrows_bytes(Rc) per warp).
struct WRows {
    double* v;
    double* u;
    double* wr;
    double* cw;
    u32* code;
    u32* segl;
    u32* row0;
};

__device__ __forceinline__ WRows wrows_at(unsigned char* base, int Rc) {
    unsigned char* p = base + size_t(wid_in_cta()) * wrows_bytes(Rc);
    WRows w;
    w.v = reinterpret_cast<double*>(p);
    p += al16(WT * Rc * 8);
    w.u = reinterpret_cast<double*>(p);
    p += al16(WT * Rc * 8);
    w.wr = reinterpret_cast<double*>(p);
    p += al16(WT * 8);
    w.cw = reinterpret_cast<double*>(p);
    p += al16(WT * 8);
    w.code = reinterpret_cast<u32*>(p);
    p += al16(4 * WT * 4);
    w.segl = reinterpret_cast<u32*>(p);
    p += al16(WT * 4);
    w.row0 = reinterpret_cast<u32*>(p);
    return w;
}

// Flat coalesced load of rows [r0, r1) x columns [j0, j0 + Rc) into v.
__device__ __forceinline__ void load_rows(const double* __restrict__ rows, int R, int j0, int Rc, u32 r0, u32 r1,
                                          const double* w_rows, const WRows& sm) {
    const u32 lane = wlane();
    const u32 ne = (r1 - r0) * u32(Rc);
#pragma unroll 4
    for (u32 f = lane; f < ne; f += 32) sm.v[f] = __ldcs(rows + size_t(r0 + f / Rc) * R + j0 + f % Rc);
    if (w_rows && lane < r1 - r0) sm.wr[lane] = w_rows[r0 + lane];
}

__device__ __forceinline__ void load_cells_rows(const DevStruct& S, const DevWeights& W, u32 c0, u32 c1, u32 s0,
                                                const WRows& sm) {
    const u32 lane = wlane();
    const u32 c = c0 + lane;
    if (c < c1) {
        sm.cw[lane] = cellw(W, c);
        for (u32 b = 0; b < S.nb && b < 4; b++) sm.code[b * WT + lane] = __ldcs(S.coord + size_t(b) * S.M + c);
        u32 s = s0;
        while (S.seg_off[s + 1] <= c) s++;
        sm.segl[lane] = s - s0;
        sm.row0[lane] = row0_of(S, c);
        if (c == c1 - 1) sm.row0[lane + 1] = row1_of(S, c);
    }
}

// Right-hand side pass 1 (operator.rs:969-1066) on short segments: b1_s = sum over the rows of s
// of w v; per-CTA partials of [sum w v^2, sum w v] (cta_part[blockIdx][2R], this chunk's
// columns); small coordinates' sums of s_c - W_c b1_s / n1_s into cta_small.
__global__ void __launch_bounds__(WPB * 32) k_wseg_rhs(DevStruct S, DevWeights W, WarpTiles wt,
                                                       const double* __restrict__ rows, int R, int j0, int Rc,
                                                       double* __restrict__ b1, double* __restrict__ cta_part,
                                                       double* __restrict__ cta_small) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const WRows sm = wrows_at(smem_raw, Rc);
    double* wacc_all = reinterpret_cast<double*>(smem_raw + WPB * wrows_bytes(Rc));
    double* colsum = wacc_all + size_t(WPB) * S.ms_acc * Rc;  // WPB x 2 x Rc
    double* wacc = wacc_all + size_t(wid_in_cta()) * S.ms_acc * Rc;
    const bool acc = cta_small != nullptr;
    const u32 lane = wlane();
    if (acc)
        for (u32 i = lane; i < S.ms_acc * u32(Rc); i += 32) wacc[i] = 0.0;
    double q = 0.0, ws = 0.0;  // column lane's totals (lane < Rc)
    const u32 wid = blockIdx.x * WPB + wid_in_cta(), nw = gridDim.x * WPB;
    for (u32 tile = wid; tile < wt.n; tile += nw) {
        const u32 s0 = wt.k0[tile], s1 = wt.k1[tile], c0 = wt.e0[tile], c1 = wt.e1[tile];
        const u32 r0 = row0_of(S, c0), r1 = row0_of(S, c1);
        load_rows(rows, R, j0, Rc, r0, r1, W.w_rows, sm);
        load_cells_rows(S, W, c0, c1, s0, sm);
        __syncwarp();
        for (u32 jj = lane; jj < u32(Rc); jj += 32) {
            u32 i = 0;
            for (u32 s = s0; s < s1; s++) {
                const u32 e = S.seg_off[s + 1] - c0;
                double sum = 0.0;
                for (u32 ci = i; ci < e; ci++) {
                    double sc = 0.0;
                    for (u32 rr = sm.row0[ci] - r0; rr < sm.row0[ci + 1] - r0; rr++) {
                        const double x = sm.v[rr * Rc + jj];
                        const double wx = W.w_rows ? sm.wr[rr] * x : x;
                        sc += wx;
                        q += wx * x;
                    }
                    sm.u[ci * Rc + jj] = sc;
                    sum += sc;
                }
                ws += sum;
                b1[size_t(s) * R + j0 + jj] = sum;
                if (acc) {
                    const double bt = sum * W.n1inv[s];
                    for (u32 ci = i; ci < e; ci++) {
                        const double z = sm.u[ci * Rc + jj] - sm.cw[ci] * bt;
                        for (u32 b = 0; b < S.ns_acc; b++) wacc[sm.code[b * WT + ci] * Rc + jj] += z;
                    }
                }
                i = e;
            }
        }
        __syncwarp();
    }
    for (u32 jj = lane; jj < u32(Rc); jj += 32) {
        colsum[(size_t(wid_in_cta()) * 2) * Rc + jj] = q;
        colsum[(size_t(wid_in_cta()) * 2 + 1) * Rc + jj] = ws;
    }
    __syncthreads();
    for (u32 i = threadIdx.x; i < 2 * u32(Rc); i += blockDim.x) {
        double s = 0.0;
        for (int w = 0; w < WPB; w++) s += colsum[size_t(w) * 2 * Rc + i];
        const u32 half = i / Rc, jj = i % Rc;
        cta_part[size_t(blockIdx.x) * 2 * R + half * R + j0 + jj] = s;
    }
    if (acc) flush_wacc(wacc_all, S.ms_acc, Rc, j0, R, cta_small);
}

// Right-hand side pass 2 on short coordinate lists (k >= ms_acc): rhs[k] = sum over the cells c
// of k of (s_c - W_c b1_{s(c)} / n1_{s(c)}).
__global__ void __launch_bounds__(WPB * 32) k_wpull_rhs(DevStruct S, DevWeights W, WarpTiles wt,
                                                        const double* __restrict__ rows, const double* __restrict__ b1,
                                                        int R, int j0, int Rc, double* __restrict__ Y) {
    __shared__ u32 cell_s[WPB][32];
    __shared__ u32 seg_s[WPB][32];
    const u32 wi = wid_in_cta(), lane = wlane();
    const GMap gm = gmap(Rc);
    const u32 wid = blockIdx.x * WPB + wi, nw = gridDim.x * WPB;
    for (u32 tile = wid; tile < wt.n; tile += nw) {
        const u32 k0 = wt.k0[tile], k1 = wt.k1[tile];
        for (u32 k = k0; k < k1; k++) {
            const u32 a = S.pl_off[k], b = S.pl_off[k + 1];
            double acc = 0.0;
            for (u32 base = a; base < b; base += 32) {
                const u32 e = base + lane;
                if (e < b) {
                    cell_s[wi][lane] = __ldcs(S.pl_cell + e);
                    seg_s[wi][lane] = __ldcs(S.pl_seg + e);
                }
                __syncwarp();
                const u32 cnt = min(32u, b - base);
                if (gm.on) {
#pragma unroll 8
                    for (u32 i = gm.g; i < cnt; i += gm.G) {
                        const u32 c = cell_s[wi][i], s = seg_s[wi][i];
                        double sc = 0.0;
                        const u32 re = row1_of(S, c);
                        for (u32 row = row0_of(S, c); row < re; row++) {
                            const double x = rows[size_t(row) * R + j0 + gm.j];
                            sc += W.w_rows ? W.w_rows[row] * x : x;
                        }
                        acc += sc - cellw(W, c) * __ldcg(b1 + size_t(s) * R + j0 + gm.j) * W.n1inv[s];
                    }
                }
                __syncwarp();
            }
            acc = group_sum(acc, gm);
            if (gm.on && gm.g == 0) Y[size_t(k) * R + j0 + gm.j] = acc;
        }
    }
}

// Residualization of short segments (operator.rs:1107-1179): alpha_s = (b1_s - sum W_c u_c) / n1_s,
// u_c = sum_b x[coord_b(c)]; every row of cell c loses alpha_s + u_c.
__global__ void __launch_bounds__(WPB * 32) k_wresid(DevStruct S, DevWeights W, WarpTiles wt, double* __restrict__ rows,
                                                     int R, int j0, int Rc, const double* __restrict__ x,
                                                     const double* __restrict__ b1, double* __restrict__ alpha) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const WRows sm = wrows_at(smem_raw, Rc);
    const u32 lane = wlane();
    const GMap gm = gmap(Rc);
    const u32 wid = blockIdx.x * WPB + wid_in_cta(), nw = gridDim.x * WPB;
    for (u32 tile = wid; tile < wt.n; tile += nw) {
        const u32 s0 = wt.k0[tile], s1 = wt.k1[tile], c0 = wt.e0[tile], c1 = wt.e1[tile];
        const u32 nc = c1 - c0;
        const u32 r0 = row0_of(S, c0), r1 = row0_of(S, c1);
        load_rows(rows, R, j0, Rc, r0, r1, nullptr, sm);
        load_cells_rows(S, W, c0, c1, s0, sm);
        __syncwarp();
        if (gm.on) {
#pragma unroll 4
            for (u32 i = gm.g; i < nc; i += gm.G) {
                double v = 0.0;
                for (u32 b = 0; b < S.nb; b++) v += x[size_t(sm.code[b * WT + i]) * R + j0 + gm.j];
                sm.u[i * Rc + gm.j] = v;
            }
        }
        __syncwarp();
        // per segment (lane = column): alpha, then the segment's rows lose alpha + u_c in place
        for (u32 jj = lane; jj < u32(Rc); jj += 32) {
            u32 i = 0;
            for (u32 s = s0; s < s1; s++) {
                const u32 e = S.seg_off[s + 1] - c0;
                double sum = 0.0;
                for (u32 ci = i; ci < e; ci++) sum += sm.cw[ci] * sm.u[ci * Rc + jj];
                const double al = (b1[size_t(s) * R + j0 + jj] - sum) * W.n1inv[s];
                if (alpha) alpha[size_t(s) * R + j0 + jj] = al;
                for (; i < e; i++) {
                    const double f = al + sm.u[i * Rc + jj];
                    for (u32 rr = sm.row0[i] - r0; rr < sm.row0[i + 1] - r0; rr++) sm.v[rr * Rc + jj] -= f;
                }
            }
        }
        __syncwarp();
        // coalesced store of the tile's rows
        const u32 ne = (r1 - r0) * u32(Rc);
#pragma unroll 4
        for (u32 f = lane; f < ne; f += 32) __stcs(rows + size_t(r0 + f / Rc) * R + j0 + f % Rc, sm.v[f]);
        __syncwarp();
    }
}

}  // namespace fereg
