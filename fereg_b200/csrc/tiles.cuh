// Tile kernels over the cell structure: the segment passes (per FE1 level) and the coordinate
// pulls (per reduced coordinate) of the rhs, operator and residualize steps.
//
// A CTA takes one tile at a time: up to TILE consecutive cells of whole segments (or TILE
// consecutive entries of the coordinate-sorted lists), or a TILE-sized slice of one long list.
//   phase A  thread (slot, column) over the tile's cells/entries: independent gathers, the
//            per-cell value goes to shared memory;
//   phase B  thread (segment or coordinate, column): the sum over its cells in list order.
// Slices of long lists write partial sums that k_fix adds in slice order. Column blocks wider
// than RC_MAX are walked in chunks.
//
// Small blocks (at most SACC_MAX coordinates in all) are summed inside the segment passes: after
// phase B every cell's value is known, and one thread per (small block, column) walks the tile's
// cells in order into a per-tile accumulator that is added to the CTA's own partial row; the
// rows of all CTAs are summed in CTA order afterwards. The coordinate pulls then cover the large
// coordinates only. All sums have a fixed order: results do not depend on timing.
#pragma once

#include "device.cuh"

namespace fereg {

constexpr int TB = 256;       // threads per tile CTA
constexpr int TILE = 128;     // cells or entries per tile
constexpr int PULL_SLICE = 2048;  // entries per coordinate-list tile
constexpr int RC_MAX = 16;    // columns per chunk
constexpr int SACC_MAX = 16;  // small coordinates summed in the segment passes
constexpr int SACC_BLOCKS = 4;

// Tiles over a CSR-like list (segments -> cells, or coordinates -> entries).
struct TileSet {
    u32 n;
    const u32* k0;
    const u32* k1;
    const u32* e0;
    const u32* e1;
    const int* part;     // partial slot of a slice of a long list, -1 otherwise
    const int* fixidx;   // index into the fix lists for slices, -1 otherwise
    u32 nfix;
    const u32* fix_k;
    const u32* fix_p0;
    const u32* fix_np;
    u32 nparts;
};

struct DevStruct {
    u32 M, g1, nb, m, ms;
    u32 ms_acc;           // small coordinates summed in the segment passes (0: none)
    u32 ns_acc;           // small blocks summed there (blocks 0..ns_acc-1)
    const u32* seg_off;
    const u32* coord;     // nb x M block-major global coordinates
    const u32* cell_row;  // M+1 (null: cell c is row c)
    const u32* pl_off;    // m+1
    const u32* pl_cell;
    const u32* pl_seg;
    const u32* pl_other;  // E x (nb-1)
    TileSet seg;          // tiles over segments
    TileSet pull;         // tiles over the pulled coordinates [ms_acc, m)
};

struct DevWeights {
    const double* w_rows;  // null: unweighted
    const double* cell_w;  // null: every cell weight is 1
    const double* n1inv;
    const double* nr;
};

__device__ __forceinline__ double cellw(const DevWeights& W, u32 c) { return W.cell_w ? W.cell_w[c] : 1.0; }
__device__ __forceinline__ u32 row0_of(const DevStruct& S, u32 c) { return S.cell_row ? S.cell_row[c] : c; }
__device__ __forceinline__ u32 row1_of(const DevStruct& S, u32 c) { return S.cell_row ? S.cell_row[c + 1] : c + 1; }

struct ColMap {
    int Rc, nslot, slot, col;
    bool on;
};

// Threads of a TB-thread CTA over (slot, column) for the column chunk starting at j0.
__device__ __forceinline__ ColMap colmap(int R, int j0) {
    const int Rc = min(R - j0, RC_MAX);
    const int nslot = TB / Rc;
    const int slot = int(threadIdx.x) / Rc;
    return {Rc, nslot, slot, int(threadIdx.x) % Rc, slot < nslot};
}

// Per-tile scratch of the segment passes.
template <class T>
struct SegSmem {
    T vals[TILE * RC_MAX];   // per-cell values
    T sval[TILE * RC_MAX];   // per-segment values (t_s, b1_s n1inv_s or alpha_s)
    T tacc[SACC_MAX * RC_MAX];
    u32 cellseg[TILE];
    u32 scode[SACC_BLOCKS * TILE];
};

// Loads the tile's cell -> local segment map and the small-block coordinates of its cells.
__device__ __forceinline__ void seg_maps(const DevStruct& S, u32 s0, u32 s1, u32 c0, u32 c1, u32* cellseg, u32* scode) {
    for (u32 s = s0 + threadIdx.x; s < s1; s += TB) {
        const u32 a = max(S.seg_off[s], c0), b = min(S.seg_off[s + 1], c1);
        for (u32 c = a; c < b; c++) cellseg[c - c0] = s - s0;
    }
    for (u32 i = threadIdx.x; i < S.ns_acc * (c1 - c0); i += TB) {
        const u32 b = i / (c1 - c0), c = c0 + i % (c1 - c0);
        scode[b * TILE + (c - c0)] = __ldcs(S.coord + size_t(b) * S.M + c);
    }
}

// vals holds the tile's per-cell values z_c (chunk j0): adds sum_{c in tile with small code k} z_c
// to the CTA's partial row (cta_small[blockIdx][k*R + j]).
template <class T>
__device__ __forceinline__ void small_accumulate(const DevStruct& S, SegSmem<T>& sm, u32 ncell, const ColMap& cm,
                                                 int j0, int R, T* __restrict__ cta_small) {
    const u32 nk = S.ms_acc * u32(cm.Rc);
    for (u32 i = threadIdx.x; i < nk; i += TB) sm.tacc[i] = T(0);
    __syncthreads();
    if (threadIdx.x < S.ns_acc * u32(cm.Rc)) {
        const u32 b = threadIdx.x / cm.Rc;
        const int col = int(threadIdx.x % cm.Rc);
        for (u32 i = 0; i < ncell; i++) sm.tacc[sm.scode[b * TILE + i] * cm.Rc + col] += sm.vals[i * cm.Rc + col];
    }
    __syncthreads();
    T* mine = cta_small + size_t(blockIdx.x) * S.ms_acc * R;
    for (u32 i = threadIdx.x; i < nk; i += TB) {
        const u32 k = i / cm.Rc;
        const int col = int(i % cm.Rc);
        mine[size_t(k) * R + j0 + col] += sm.tacc[i];
    }
}

template <class T>
__device__ __forceinline__ void zero_cta_row(T* __restrict__ cta_small, u32 len) {
    if (!cta_small) return;
    T* mine = cta_small + size_t(blockIdx.x) * len;
    for (u32 i = threadIdx.x; i < len; i += TB) mine[i] = T(0);
}

// ---------------------------------------------------------------------------------------------
// Operator pass 1 (operator.rs:894-948): t_s = sum_c W_c u_c / n1_s with u_c = sum_b P[coord_b(c)],
// and the small coordinates' Y_k = sum over the cells c of k of W_c (u_c - t_s) into the CTA
// rows of cta_small. Slices of long segments write partial W u sums (`part`). With
// `slices_only` only the slices run (the W u partials of the residualize pass).
template <class T>
__global__ void __launch_bounds__(TB) k_seg_apply(DevStruct S, DevWeights W, const T* __restrict__ P, int R,
                                                  T* __restrict__ t, T* __restrict__ part, bool slices_only,
                                                  T* __restrict__ cta_small) {
    __shared__ SegSmem<T> sm;
    const TileSet& ts = S.seg;
    const bool acc = cta_small && S.ms_acc > 0;
    if (acc) zero_cta_row(cta_small, S.ms_acc * u32(R));
    for (u32 tile = blockIdx.x; tile < ts.n; tile += gridDim.x) {
        const u32 s0 = ts.k0[tile], s1 = ts.k1[tile], c0 = ts.e0[tile], c1 = ts.e1[tile];
        const int pslot = ts.part[tile];
        if (slices_only && pslot < 0) continue;
        __syncthreads();
        if (acc && pslot < 0) seg_maps(S, s0, s1, c0, c1, sm.cellseg, sm.scode);
        for (int j0 = 0; j0 < R; j0 += RC_MAX) {
            const ColMap cm = colmap(R, j0);
            if (cm.on) {
#pragma unroll 4
                for (u32 c = c0 + cm.slot; c < c1; c += cm.nslot) {
                    T u = T(0);
                    for (u32 b = 0; b < S.nb; b++) u += P[size_t(__ldcs(S.coord + size_t(b) * S.M + c)) * R + j0 + cm.col];
                    sm.vals[(c - c0) * cm.Rc + cm.col] = T(cellw(W, c)) * u;
                }
            }
            __syncthreads();
            const u32 nk = (s1 - s0) * u32(cm.Rc);
            for (u32 idx = threadIdx.x; idx < nk; idx += TB) {
                const u32 s = s0 + idx / cm.Rc;
                const int col = int(idx % cm.Rc);
                const u32 a = max(S.seg_off[s], c0), b = min(S.seg_off[s + 1], c1);
                T sum = T(0);
                for (u32 c = a; c < b; c++) sum += sm.vals[(c - c0) * cm.Rc + col];
                if (pslot < 0) {
                    const T ts_ = sum * T(W.n1inv[s]);
                    t[size_t(s) * R + j0 + col] = ts_;
                    sm.sval[(s - s0) * cm.Rc + col] = ts_;
                } else {
                    part[size_t(pslot) * R + j0 + col] = sum;
                }
            }
            if (acc && pslot < 0) {
                __syncthreads();
                // z_c = W_c (u_c - t_s)
                for (u32 i = threadIdx.x; i < (c1 - c0) * u32(cm.Rc); i += TB) {
                    const u32 c = i / cm.Rc;
                    const int col = int(i % cm.Rc);
                    sm.vals[i] -= T(cellw(W, c0 + c)) * sm.sval[sm.cellseg[c] * cm.Rc + col];
                }
                __syncthreads();
                small_accumulate(S, sm, c1 - c0, cm, j0, R, cta_small);
            }
            __syncthreads();
        }
    }
}

// Sum over the slots of a CTA of red[slot * Rc + col] into red[col] (slot 0), by a pairwise tree
// over the slot indices: the same order every call. Every thread of the CTA calls it.
template <class T>
__device__ __forceinline__ void slot_tree(T* red, const ColMap& cm) {
    for (int s = 1; s < cm.nslot; s *= 2) {
        __syncthreads();
        if (cm.on && cm.slot % (2 * s) == 0 && cm.slot + s < cm.nslot)
            red[cm.slot * cm.Rc + cm.col] += red[(cm.slot + s) * cm.Rc + cm.col];
    }
    __syncthreads();
}

// Operator pass 2: Y[k] = nr_k P[k] + sum over the cells c of k of W_c (sum_{other b} P - t_{s(c)})
// for the pulled coordinates. A tile holds whole lists or a slice of one long list (its partial
// goes to k_fix); per list, thread (slot, column) sums the entries slot, slot + nslot, ... in a
// register and the slots are combined by slot_tree.
template <class T>
__global__ void __launch_bounds__(TB) k_pull_apply(DevStruct S, DevWeights W, const T* __restrict__ P,
                                                   const T* __restrict__ t, int R, T* __restrict__ Y,
                                                   T* __restrict__ part) {
    __shared__ T red[TB];
    const TileSet& ts = S.pull;
    const u32 no = S.nb - 1;
    for (u32 tile = blockIdx.x; tile < ts.n; tile += gridDim.x) {
        const u32 k0 = ts.k0[tile], k1 = ts.k1[tile], e0 = ts.e0[tile], e1 = ts.e1[tile];
        const int pslot = ts.part[tile];
        for (int j0 = 0; j0 < R; j0 += RC_MAX) {
            const ColMap cm = colmap(R, j0);
            for (u32 k = k0; k < k1; k++) {
                const u32 a = max(S.pl_off[k], e0), b = min(S.pl_off[k + 1], e1);
                T acc = T(0);
                if (cm.on) {
#pragma unroll 4
                    for (u32 e = a + cm.slot; e < b; e += cm.nslot) {
                        T u = -__ldcg(t + size_t(__ldcs(S.pl_seg + e)) * R + j0 + cm.col);
                        for (u32 o = 0; o < no; o++)
                            u += P[size_t(__ldcs(S.pl_other + size_t(e) * no + o)) * R + j0 + cm.col];
                        acc += W.cell_w ? T(W.cell_w[__ldcs(S.pl_cell + e)]) * u : u;
                    }
                    red[cm.slot * cm.Rc + cm.col] = acc;
                }
                slot_tree(red, cm);
                if (cm.on && cm.slot == 0) {
                    const size_t o = size_t(k) * R + j0 + cm.col;
                    if (pslot < 0) Y[o] = T(W.nr[k]) * P[o] + red[cm.col];
                    else part[size_t(pslot) * R + j0 + cm.col] = red[cm.col];
                }
                __syncthreads();
            }
        }
    }
}

// Long lists: out[key] = sum of the partials in slice order, plus nr_key P[key] (mode 0), or
// times 1/n1_key (mode 1), or as is (mode 2). One CTA per list.
template <class T>
__global__ void __launch_bounds__(TB) k_fix(TileSet ts, DevWeights W, const T* __restrict__ P,
                                            const T* __restrict__ part, int R, int mode, T* __restrict__ out) {
    __shared__ T red[TB];
    for (u32 f = blockIdx.x; f < ts.nfix; f += gridDim.x) {
        const u32 key = ts.fix_k[f], p0 = ts.fix_p0[f], np = ts.fix_np[f];
        for (int j0 = 0; j0 < R; j0 += RC_MAX) {
            const ColMap cm = colmap(R, j0);
            T acc = T(0);
            if (cm.on) {
#pragma unroll 8
                for (u32 p = cm.slot; p < np; p += cm.nslot) acc += part[size_t(p0 + p) * R + j0 + cm.col];
            }
            red[threadIdx.x] = acc;
            __syncthreads();
            if (int(threadIdx.x) < cm.Rc) {
                T s = T(0);
                for (int sl = 0; sl < cm.nslot; sl++) s += red[sl * cm.Rc + threadIdx.x];
                const size_t o = size_t(key) * R + j0 + threadIdx.x;
                if (mode == 0) out[o] = T(W.nr[key]) * P[o] + s;
                else if (mode == 1) out[o] = s * T(W.n1inv[key]);
                else out[o] = s;
            }
            __syncthreads();
        }
    }
}

// Y[i] (i < ms_acc * R) = sum over the CTA partial rows of up to three kernels (null arrays are
// skipped): one warp per element, lane l sums rows l, l+32, ... of each array in turn, then a
// fixed butterfly.
template <class T>
__global__ void k_small_reduce(const T* __restrict__ a, int na, const T* __restrict__ b, int nb_,
                               const T* __restrict__ c, int nc, u32 len, T* __restrict__ Y) {
    const int lane = int(threadIdx.x & 31);
    const u32 w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (u32 i = w0; i < len; i += nw) {
        T s = T(0);
        if (a)
            for (int p = lane; p < na; p += 32) s += a[size_t(p) * len + i];
        if (b)
            for (int p = lane; p < nb_; p += 32) s += b[size_t(p) * len + i];
        if (c)
            for (int p = lane; p < nc; p += 32) s += c[size_t(p) * len + i];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
        if (lane == 0) Y[i] = s;
    }
}

// ---------------------------------------------------------------------------------------------
// Right-hand side pass 1 (operator.rs:969-1066): b1_s = sum over the rows of s of w v (partials
// for slices of long segments); per-CTA partial sums of [sum w v^2, sum w v] per column
// (cta_part, grid x 2R, accumulated over the CTA's tiles in tile order); and the small
// coordinates' rhs_k = sum over the cells c of k of (s_c - W_c b1_s / n1_s) into cta_small.
__global__ void __launch_bounds__(TB) k_seg_rhs(DevStruct S, DevWeights W, const double* __restrict__ rows, int R,
                                                double* __restrict__ b1, double* __restrict__ part,
                                                double* __restrict__ cta_part, double* __restrict__ cta_small) {
    __shared__ SegSmem<double> sm;
    __shared__ double red[2 * TB];
    const TileSet& ts = S.seg;
    const bool acc = cta_small && S.ms_acc > 0;
    double* mine = cta_part + size_t(blockIdx.x) * 2 * R;
    for (int j = threadIdx.x; j < 2 * R; j += TB) mine[j] = 0.0;
    if (acc) zero_cta_row(cta_small, S.ms_acc * u32(R));
    for (u32 tile = blockIdx.x; tile < ts.n; tile += gridDim.x) {
        const u32 s0 = ts.k0[tile], s1 = ts.k1[tile], c0 = ts.e0[tile], c1 = ts.e1[tile];
        const int pslot = ts.part[tile];
        __syncthreads();
        if (acc && pslot < 0) seg_maps(S, s0, s1, c0, c1, sm.cellseg, sm.scode);
        for (int j0 = 0; j0 < R; j0 += RC_MAX) {
            const ColMap cm = colmap(R, j0);
            double q = 0.0, a1 = 0.0;
            if (cm.on) {
#pragma unroll 4
                for (u32 c = c0 + cm.slot; c < c1; c += cm.nslot) {
                    double a = 0.0;
                    const u32 r1 = row1_of(S, c);
                    for (u32 row = row0_of(S, c); row < r1; row++) {
                        const double v = __ldcs(rows + size_t(row) * R + j0 + cm.col);
                        const double wv = W.w_rows ? W.w_rows[row] * v : v;
                        a += wv;
                        q += wv * v;
                    }
                    a1 += a;
                    sm.vals[(c - c0) * cm.Rc + cm.col] = a;
                }
            }
            red[threadIdx.x] = q;
            red[TB + threadIdx.x] = a1;
            __syncthreads();
            const u32 nk = (s1 - s0) * u32(cm.Rc);
            for (u32 idx = threadIdx.x; idx < nk; idx += TB) {
                const u32 s = s0 + idx / cm.Rc;
                const int col = int(idx % cm.Rc);
                const u32 a = max(S.seg_off[s], c0), b = min(S.seg_off[s + 1], c1);
                double sum = 0.0;
                for (u32 c = a; c < b; c++) sum += sm.vals[(c - c0) * cm.Rc + col];
                if (pslot < 0) {
                    b1[size_t(s) * R + j0 + col] = sum;
                    sm.sval[(s - s0) * cm.Rc + col] = sum * W.n1inv[s];
                } else {
                    part[size_t(pslot) * R + j0 + col] = sum;
                }
            }
            // tile totals per column, slots in order
            if (int(threadIdx.x) < cm.Rc) {
                double tq = 0.0, tw = 0.0;
                for (int sl = 0; sl < cm.nslot; sl++) {
                    tq += red[sl * cm.Rc + threadIdx.x];
                    tw += red[TB + sl * cm.Rc + threadIdx.x];
                }
                mine[j0 + threadIdx.x] += tq;
                mine[R + j0 + threadIdx.x] += tw;
            }
            if (acc && pslot < 0) {
                __syncthreads();
                for (u32 i = threadIdx.x; i < (c1 - c0) * u32(cm.Rc); i += TB) {
                    const u32 c = i / cm.Rc;
                    const int col = int(i % cm.Rc);
                    sm.vals[i] -= cellw(W, c0 + c) * sm.sval[sm.cellseg[c] * cm.Rc + col];
                }
                __syncthreads();
                small_accumulate(S, sm, c1 - c0, cm, j0, R, cta_small);
            }
            __syncthreads();
        }
    }
}

// Small coordinates of the slices of long segments, once b1 is complete.
__global__ void __launch_bounds__(TB) k_rhs_small_slices(DevStruct S, DevWeights W, const double* __restrict__ rows,
                                                         const double* __restrict__ b1, int R,
                                                         double* __restrict__ cta_small) {
    __shared__ SegSmem<double> sm;
    const TileSet& ts = S.seg;
    zero_cta_row(cta_small, S.ms_acc * u32(R));
    for (u32 tile = blockIdx.x; tile < ts.n; tile += gridDim.x) {
        const u32 s0 = ts.k0[tile], c0 = ts.e0[tile], c1 = ts.e1[tile];
        if (ts.part[tile] < 0) continue;
        __syncthreads();
        seg_maps(S, s0, s0 + 1, c0, c1, sm.cellseg, sm.scode);
        for (int j0 = 0; j0 < R; j0 += RC_MAX) {
            const ColMap cm = colmap(R, j0);
            if (cm.on)
                for (u32 c = c0 + cm.slot; c < c1; c += cm.nslot) {
                    double a = 0.0;
                    const u32 r1 = row1_of(S, c);
                    for (u32 row = row0_of(S, c); row < r1; row++) {
                        const double v = rows[size_t(row) * R + j0 + cm.col];
                        a += W.w_rows ? W.w_rows[row] * v : v;
                    }
                    sm.vals[(c - c0) * cm.Rc + cm.col] = a - cellw(W, c) * b1[size_t(s0) * R + j0 + cm.col] * W.n1inv[s0];
                }
            __syncthreads();
            small_accumulate(S, sm, c1 - c0, cm, j0, R, cta_small);
            __syncthreads();
        }
    }
}

// Right-hand side pass 2: rhs[k] = sum over the cells c of k of (s_c - W_c b1_{s(c)} / n1_{s(c)})
// for the pulled coordinates, with the tiles and the slot sums of k_pull_apply.
__global__ void __launch_bounds__(TB) k_pull_rhs(DevStruct S, DevWeights W, const double* __restrict__ rows,
                                                 const double* __restrict__ b1, int R, double* __restrict__ Y,
                                                 double* __restrict__ part) {
    __shared__ double red[TB];
    const TileSet& ts = S.pull;
    for (u32 tile = blockIdx.x; tile < ts.n; tile += gridDim.x) {
        const u32 k0 = ts.k0[tile], k1 = ts.k1[tile], e0 = ts.e0[tile], e1 = ts.e1[tile];
        const int pslot = ts.part[tile];
        for (int j0 = 0; j0 < R; j0 += RC_MAX) {
            const ColMap cm = colmap(R, j0);
            for (u32 k = k0; k < k1; k++) {
                const u32 a = max(S.pl_off[k], e0), b = min(S.pl_off[k + 1], e1);
                double acc = 0.0;
                if (cm.on) {
#pragma unroll 4
                    for (u32 e = a + cm.slot; e < b; e += cm.nslot) {
                        const u32 c = __ldcs(S.pl_cell + e), s = __ldcs(S.pl_seg + e);
                        double sc = 0.0;
                        const u32 r1 = row1_of(S, c);
                        for (u32 row = row0_of(S, c); row < r1; row++) {
                            const double v = __ldcs(rows + size_t(row) * R + j0 + cm.col);
                            sc += W.w_rows ? W.w_rows[row] * v : v;
                        }
                        acc += sc - cellw(W, c) * __ldcg(b1 + size_t(s) * R + j0 + cm.col) * W.n1inv[s];
                    }
                    red[cm.slot * cm.Rc + cm.col] = acc;
                }
                slot_tree(red, cm);
                if (cm.on && cm.slot == 0) {
                    if (pslot < 0) Y[size_t(k) * R + j0 + cm.col] = red[cm.col];
                    else part[size_t(pslot) * R + j0 + cm.col] = red[cm.col];
                }
                __syncthreads();
            }
        }
    }
}

// sum_s b1_s^2 / n1_s per column (solve.rs:648-658) as per-CTA partials (grid x R).
__global__ void __launch_bounds__(TB) k_b1sq(u32 g1, const double* __restrict__ b1, const double* __restrict__ n1inv,
                                             int R, double* __restrict__ cta_part) {
    __shared__ double red[TB];
    for (int j0 = 0; j0 < R; j0 += RC_MAX) {
        const ColMap cm = colmap(R, j0);
        double acc = 0.0;
        if (cm.on) {
            // four segments' loads in flight together, the sum in segment order
            const u32 step = gridDim.x * u32(cm.nslot);
            u32 s = blockIdx.x * u32(cm.nslot) + u32(cm.slot);
            const double* col = b1 + j0 + cm.col;
            for (; size_t(s) + 3 * size_t(step) < g1; s += 4 * step) {
                const double v0 = col[size_t(s) * R], v1 = col[size_t(s + step) * R];
                const double v2 = col[size_t(s + 2 * step) * R], v3 = col[size_t(s + 3 * step) * R];
                const double n0 = n1inv[s], n1 = n1inv[s + step], n2 = n1inv[s + 2 * step], n3 = n1inv[s + 3 * step];
                acc += v0 * v0 * n0;
                acc += v1 * v1 * n1;
                acc += v2 * v2 * n2;
                acc += v3 * v3 * n3;
            }
            for (; s < g1; s += step) {
                const double v = col[size_t(s) * R];
                acc += v * v * n1inv[s];
            }
        }
        red[threadIdx.x] = acc;
        __syncthreads();
        if (int(threadIdx.x) < cm.Rc) {
            double s = 0.0;
            for (int sl = 0; sl < cm.nslot; sl++) s += red[sl * cm.Rc + threadIdx.x];
            cta_part[size_t(blockIdx.x) * R + j0 + threadIdx.x] = s;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------
// Residualization (operator.rs:1107-1179): alpha_s = (b1_s - sum_c W_c u_c) / n1_s with
// u_c = sum_b x[coord_b(c)], then every row of cell c loses alpha_s + u_c. Slices of long
// segments take alpha from `along` (fix index x R), filled beforehand by k_seg_apply on x and
// k_fix_alpha. With one row per cell, each thread's row elements are loaded first so their
// latency overlaps the gathers of x.
constexpr int PF = TILE / (TB / RC_MAX);  // row elements per thread and chunk (one row per cell)

__global__ void __launch_bounds__(TB, 4) k_residualize(DevStruct S, DevWeights W, double* __restrict__ rows, int R,
                                                    const double* __restrict__ x, const double* __restrict__ b1,
                                                    const double* __restrict__ along, double* __restrict__ alpha) {
    __shared__ double vals[TILE * RC_MAX];
    __shared__ double aseg[TILE * RC_MAX];
    __shared__ u32 cellseg[TILE];
    const TileSet& ts = S.seg;
    for (u32 tile = blockIdx.x; tile < ts.n; tile += gridDim.x) {
        const u32 s0 = ts.k0[tile], s1 = ts.k1[tile], c0 = ts.e0[tile], c1 = ts.e1[tile];
        const int fidx = ts.fixidx[tile];
        __syncthreads();
        for (u32 s = s0 + threadIdx.x; s < s1; s += TB) {
            const u32 a = max(S.seg_off[s], c0), b = min(S.seg_off[s + 1], c1);
            for (u32 c = a; c < b; c++) cellseg[c - c0] = s - s0;
        }
        for (int j0 = 0; j0 < R; j0 += RC_MAX) {
            const ColMap cm = colmap(R, j0);
            double rv[PF];
            const bool pre = S.cell_row == nullptr;
            if (pre && cm.on) {
#pragma unroll
                for (int k = 0; k < PF; k++) {
                    const u32 c = c0 + cm.slot + u32(k * cm.nslot);
                    rv[k] = c < c1 ? __ldcs(rows + size_t(c) * R + j0 + cm.col) : 0.0;
                }
            }
            if (cm.on) {
#pragma unroll 4
                for (u32 c = c0 + cm.slot; c < c1; c += cm.nslot) {
                    double u = 0.0;
                    for (u32 b = 0; b < S.nb; b++) u += x[size_t(__ldcs(S.coord + size_t(b) * S.M + c)) * R + j0 + cm.col];
                    vals[(c - c0) * cm.Rc + cm.col] = u;
                }
            }
            __syncthreads();
            const u32 nk = (s1 - s0) * u32(cm.Rc);
            for (u32 idx = threadIdx.x; idx < nk; idx += TB) {
                const u32 s = s0 + idx / cm.Rc;
                const int col = int(idx % cm.Rc);
                double a;
                if (fidx < 0) {
                    const u32 ca = S.seg_off[s], cb = S.seg_off[s + 1];
                    double acc = 0.0;
                    for (u32 c = ca; c < cb; c++) acc += cellw(W, c) * vals[(c - c0) * cm.Rc + col];
                    a = (b1[size_t(s) * R + j0 + col] - acc) * W.n1inv[s];
                    if (alpha) alpha[size_t(s) * R + j0 + col] = a;
                } else {
                    a = along[size_t(fidx) * R + j0 + col];
                }
                aseg[(s - s0) * cm.Rc + col] = a;
            }
            __syncthreads();
            if (cm.on) {
                if (pre) {
#pragma unroll
                    for (int k = 0; k < PF; k++) {
                        const u32 c = c0 + cm.slot + u32(k * cm.nslot);
                        if (c < c1) {
                            const double f = aseg[cellseg[c - c0] * cm.Rc + cm.col] + vals[(c - c0) * cm.Rc + cm.col];
                            __stcs(rows + size_t(c) * R + j0 + cm.col, rv[k] - f);
                        }
                    }
                } else {
#pragma unroll 4
                    for (u32 c = c0 + cm.slot; c < c1; c += cm.nslot) {
                        const double f = aseg[cellseg[c - c0] * cm.Rc + cm.col] + vals[(c - c0) * cm.Rc + cm.col];
                        const u32 r1 = row1_of(S, c);
                        for (u32 row = row0_of(S, c); row < r1; row++) rows[size_t(row) * R + j0 + cm.col] -= f;
                    }
                }
            }
            __syncthreads();
        }
    }
}

// alpha of the long segments: along[f] = (b1_s - sum of the W u partials) / n1_s; also written
// to alpha (g1 x R) when requested. One CTA per long segment.
__global__ void __launch_bounds__(TB) k_fix_alpha(TileSet ts, DevWeights W, const double* __restrict__ part,
                                                  const double* __restrict__ b1, int R, double* __restrict__ along,
                                                  double* __restrict__ alpha) {
    __shared__ double red[TB];
    for (u32 f = blockIdx.x; f < ts.nfix; f += gridDim.x) {
        const u32 s = ts.fix_k[f], p0 = ts.fix_p0[f], np = ts.fix_np[f];
        for (int j0 = 0; j0 < R; j0 += RC_MAX) {
            const ColMap cm = colmap(R, j0);
            double acc = 0.0;
            if (cm.on)
                for (u32 p = cm.slot; p < np; p += cm.nslot) acc += part[size_t(p0 + p) * R + j0 + cm.col];
            red[threadIdx.x] = acc;
            __syncthreads();
            if (int(threadIdx.x) < cm.Rc) {
                double sum = 0.0;
                for (int sl = 0; sl < cm.nslot; sl++) sum += red[sl * cm.Rc + threadIdx.x];
                const int j = j0 + int(threadIdx.x);
                const double a = (b1[size_t(s) * R + j] - sum) * W.n1inv[s];
                along[size_t(f) * R + j] = a;
                if (alpha) alpha[size_t(s) * R + j] = a;
            }
            __syncthreads();
        }
    }
}

}  // namespace fereg
