// Device refresh of the weight state (operator.rs:211-338 refresh_weights, :344-570
// level_weights): cell weights W_c = sum of the cell's row weights, n1_s = sum of the segment's
// W_c, and for every reduced coordinate k: n_k = sum of W_c over the cells of k, and
// diag_k = n_k - sum_s c_{s,k}^2 / n1_s with c_{s,k} the weight of k's cells in segment s; k is
// redundant when diag_k <= 1e-12 n_k (operator.rs:21), and the Jacobi factor is 1 / diag_k
// otherwise. The coordinate-sorted lists hold each coordinate's cells in cell order, hence in
// segment order, so c_{s,k} are the sums over runs of equal segment: warps walk chunks of the
// lists 32 entries at a time with a segmented scan, and a per-coordinate pass stitches the runs
// that cross chunk boundaries. All sums have a fixed order.
#pragma once

#include "device.cuh"

namespace fereg {

// flag = 1 when a weight is not positive and finite.
__global__ void k_check_weights(const double* __restrict__ w, size_t n, int* flag) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const double x = w[i];
        if (!(x > 0.0 && x <= 1.7976931348623157e308)) atomicExch(flag, 1);
    }
}

// W_c = sum of the row weights of cell c (rows cell_row[c] .. cell_row[c+1]).
__global__ void k_cell_weights(const double* __restrict__ w, const u32* __restrict__ cell_row, u32 M,
                               double* __restrict__ cw) {
    for (u32 c = blockIdx.x * blockDim.x + threadIdx.x; c < M; c += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (u32 r = cell_row[c]; r < cell_row[c + 1]; r++) s += w[r];
        cw[c] = s;
    }
}

// out[r] = in[pi[r]]: kept-order values in row order.
__global__ void k_gather_rows_f64(const double* __restrict__ in, const u32* __restrict__ pi, size_t n,
                                  double* __restrict__ out) {
    for (size_t r = size_t(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += size_t(gridDim.x) * blockDim.x)
        out[r] = in[pi[r]];
}

// W_c = the number of rows of cell c (unit row weights).
__global__ void k_cell_counts(const u32* __restrict__ cell_row, u32 M, double* __restrict__ cw) {
    for (u32 c = blockIdx.x * blockDim.x + threadIdx.x; c < M; c += gridDim.x * blockDim.x)
        cw[c] = double(cell_row[c + 1] - cell_row[c]);
}

// n1_s = sum of W_c over the segment's cells (cw null: 1 per cell); n1inv = 1 / n1.
__global__ void k_seg_weights(const double* __restrict__ cw, const u32* __restrict__ seg_off, u32 g1,
                              double* __restrict__ n1, double* __restrict__ n1inv) {
    for (u32 s = blockIdx.x * blockDim.x + threadIdx.x; s < g1; s += gridDim.x * blockDim.x) {
        double a = 0.0;
        for (u32 c = seg_off[s]; c < seg_off[s + 1]; c++) a += cw ? cw[c] : 1.0;
        n1[s] = a;
        n1inv[s] = 1.0 / a;
    }
}

// n_k, diag_k, redundant_k and the Jacobi factor of every coordinate, in two passes so that a
// long list (a 10-level year block holds n/10 entries per list) does not serialize on one warp.
//
// Pass 1, a warp per chunk of at most CW_CHUNK entries of one list: the chunk's sum of weights,
// its sum of squared runs as if the chunk were the whole list (dq_iso = sum_runs x^2 / n1_s), and
// its first and last runs (segment, partial sum). A segment's entries are contiguous in a list
// (lists are in cell order, cells in segment order), so the first run is every entry of the
// first entry's segment, and likewise for the last.
constexpr u32 CW_CHUNK = 512;

struct CwChunk {
    double nr, dq, xf, xl;
    u32 sf, sl;
};

__global__ void k_coord_chunks(const u32* __restrict__ chunk_e0, const u32* __restrict__ chunk_e1, u32 nchunks,
                               const u32* __restrict__ pl_cell, const u32* __restrict__ pl_seg,
                               const double* __restrict__ cw, const double* __restrict__ n1inv,
                               CwChunk* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const size_t gw = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5, nw = (size_t(gridDim.x) * blockDim.x) >> 5;
    constexpr u32 NONE = 0xffffffffu;
    for (size_t c = gw; c < nchunks; c += nw) {
        const u32 e0 = chunk_e0[c], e1 = chunk_e1[c];
        const u32 sf = pl_seg[e0], sl = pl_seg[e1 - 1];
        double nr_acc = 0.0, dq_acc = 0.0, xf = 0.0, xl = 0.0;
        u32 carry_s = NONE;
        double carry = 0.0;
        for (u32 base = e0; base < e1; base += 32) {
            const u32 e = base + u32(lane);
            const bool valid = e < e1;
            const double wv = valid ? (cw ? cw[pl_cell[e]] : 1.0) : 0.0;
            const u32 s = valid ? pl_seg[e] : NONE;
            nr_acc += wv;
            if (s == sf) xf += wv;
            if (s == sl) xl += wv;
            // the run carried from the previous sub-chunk ends here unless this one continues it
            const u32 s0 = __shfl_sync(FULL, s, 0);
            if (lane == 0 && carry_s != NONE && s0 != carry_s) dq_acc += carry * carry * n1inv[carry_s];
            // inclusive scan of wv over the lane's run (runs are contiguous)
            double x = wv;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const double y = __shfl_up_sync(FULL, x, d);
                const u32 sy = __shfl_up_sync(FULL, s, d);
                if (lane >= d && sy == s) x += y;
            }
            if (valid && s == carry_s) x += carry;  // the run left open by the previous sub-chunk
            const u32 s_next = __shfl_down_sync(FULL, s, 1);
            const bool tail = valid && (lane == 31 || s_next != s);
            const int last = int(min(31u, e1 - 1 - base));
            const u32 s_last = __shfl_sync(FULL, s, last);
            const double x_last = __shfl_sync(FULL, x, last);
            const bool final_sub = base + 32 >= e1;
            if (tail && (final_sub || s != s_last)) dq_acc += x * x * n1inv[s];
            carry_s = s_last;
            carry = x_last;
        }
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
            nr_acc += __shfl_down_sync(FULL, nr_acc, d);
            dq_acc += __shfl_down_sync(FULL, dq_acc, d);
            xf += __shfl_down_sync(FULL, xf, d);
            xl += __shfl_down_sync(FULL, xl, d);
        }
        if (lane == 0) out[c] = CwChunk{nr_acc, dq_acc, xf, xl, sf, sl};
    }
}

// Pass 2, a thread per coordinate: the chunks of its list in order. Sums of nr and dq_iso; a run
// that spans chunks (its parts x_i) contributes (sum x_i)^2 - sum x_i^2 more. Then diag_k =
// n_k - dq_k, redundant when diag_k <= 1e-12 n_k (operator.rs:21), Jacobi factor 1 / diag_k.
__global__ void k_coord_combine(const u32* __restrict__ list_chunk_off, u32 m, const CwChunk* __restrict__ ch,
                                const double* __restrict__ n1inv, double* __restrict__ nr, double* __restrict__ diag,
                                uint8_t* __restrict__ red, double* __restrict__ inv_diag) {
    constexpr u32 NONE = 0xffffffffu;
    for (u32 k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        double n_acc = 0.0, dq = 0.0, X = 0.0, Q = 0.0;
        u32 cs = NONE;
        for (u32 c = list_chunk_off[k]; c < list_chunk_off[k + 1]; c++) {
            const CwChunk h = ch[c];
            n_acc += h.nr;
            dq += h.dq;
            if (h.sf == cs) {
                X += h.xf;
                Q += h.xf * h.xf;
            } else {
                if (cs != NONE) dq += (X * X - Q) * n1inv[cs];
                cs = h.sf;
                X = h.xf;
                Q = h.xf * h.xf;
            }
            if (h.sl != h.sf) {  // the chunk holds more runs: the carried run ends at its first
                dq += (X * X - Q) * n1inv[cs];
                cs = h.sl;
                X = h.xl;
                Q = h.xl * h.xl;
            }
        }
        if (cs != NONE) dq += (X * X - Q) * n1inv[cs];
        const double dg = n_acc - dq;
        const bool r = dg <= 1e-12 * n_acc;
        nr[k] = n_acc;
        diag[k] = dg;
        red[k] = r ? 1 : 0;
        inv_diag[k] = (r || !(dg > 0.0)) ? 0.0 : 1.0 / dg;
    }
}

// Dense small super-block S_SS (ms x ms, the first ms coordinates, ns small blocks) for the current
// cell weights, on the device (operator.rs:1457-1523, as the host assembly of the dense factor):
//   S_SS[k][l] = sum_c W_c [k in c][l in c] - sum_s c_{s,k} c_{s,l} / n1_s,
// by rows: one warp per work item (row k, a run of k's coordinate-list entries that never splits a segment),
// accumulating the item's dense partial row in shared memory. Per entry (cell c of segment s):
// S[k][l] += W_c for the small codes l of c; once per segment of the run, with
// c_{s,k} = sum over the segment's cells and small blocks of W [code == k] (a warp sum in fixed
// order), S[k][l] -= c_{s,k} W_c' / n1_s for the small codes l of every cell c' of s. Lane 0
// applies the updates in entry and cell order, so the row does not depend on timing;
// k_small_rows_sum adds a row's items in item order.
__global__ void __launch_bounds__(256) k_small_rows(const u32* __restrict__ seg_off, const u32* __restrict__ coord,
                                                    u32 M, int ns, u32 ms, const double* __restrict__ cw,
                                                    const double* __restrict__ n1inv, const u32* __restrict__ pl_cell,
                                                    const u32* __restrict__ pl_seg, const u32* __restrict__ item_k,
                                                    const u32* __restrict__ item_a, const u32* __restrict__ item_b,
                                                    u32 nitems, double* __restrict__ part) {
    extern __shared__ double rows_s[];
    const u32 w = threadIdx.x / 32, lane = threadIdx.x % 32;
    const u32 it = blockIdx.x * 8 + w;
    if (it >= nitems) return;  // whole warps
    double* row = rows_s + size_t(w) * ms;
    for (u32 l = lane; l < ms; l += 32) row[l] = 0.0;
    __syncwarp();
    const u32 k = item_k[it];
    u32 prev = 0xffffffffu;
    for (u32 e = item_a[it]; e < item_b[it]; e++) {
        const u32 c = pl_cell[e], s = pl_seg[e];
        if (lane == 0) {
            const double wc = cw ? cw[c] : 1.0;
            for (int b = 0; b < ns; b++) row[coord[size_t(b) * M + c]] += wc;
        }
        if (s != prev) {
            prev = s;
            const u32 c0 = seg_off[s], c1 = seg_off[s + 1];
            double ck = 0.0;
            for (u32 cc = c0 + lane; cc < c1; cc += 32) {
                const double wc = cw ? cw[cc] : 1.0;
                for (int b = 0; b < ns; b++)
                    if (coord[size_t(b) * M + cc] == k) ck += wc;
            }
#pragma unroll
            for (int o = 16; o > 0; o /= 2) ck += __shfl_xor_sync(FULL, ck, o);
            const double f = ck * n1inv[s];
            if (lane == 0)
                for (u32 cc = c0; cc < c1; cc++) {
                    const double v = f * (cw ? cw[cc] : 1.0);
                    for (int b = 0; b < ns; b++) row[coord[size_t(b) * M + cc]] -= v;
                }
        }
        __syncwarp();
    }
    for (u32 l = lane; l < ms; l += 32) part[size_t(it) * ms + l] = row[l];
}

// Row k of S_SS: the partial rows of k's items (first[k] .. first[k+1]) added in item order.
__global__ void k_small_rows_sum(const double* __restrict__ part, const u32* __restrict__ first, u32 ms,
                                 double* __restrict__ out) {
    const u32 k = blockIdx.x;
    for (u32 l = threadIdx.x; l < ms; l += blockDim.x) {
        double v = 0.0;
        for (u32 it = first[k]; it < first[k + 1]; it++) v += part[size_t(it) * ms + l];
        out[size_t(k) * ms + l] = v;
    }
}


// ak (k x k) = the kept rows / columns of a (ms x ms), scaled to unit diagonal.
__global__ void k_small_gather(const double* __restrict__ a, u32 ms, const u32* __restrict__ keep,
                               const double* __restrict__ scale, int k, double* __restrict__ ak) {
    const size_t total = size_t(k) * k;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += size_t(gridDim.x) * blockDim.x) {
        const int r = int(i / k), c = int(i % k);
        ak[i] = a[size_t(keep[r]) * ms + keep[c]] * scale[r] * scale[c];
    }
}

// Sum of a vector into per-CTA partials (fixed tree); the host adds the partials in CTA order.
__global__ void __launch_bounds__(256) k_vec_sum(const double* __restrict__ v, size_t n, double* __restrict__ part) {
    __shared__ double red[256];
    double s = 0.0;
    for (size_t i = size_t(blockIdx.x) * 256 + threadIdx.x; i < n; i += size_t(gridDim.x) * 256) s += v[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// ---------------------------------------------------------------------------------------------
// The rows of S on the small coordinates, for the operator (operator.rs:894-948 restated as a
// product): with at most SACC_MAX small coordinates (blocks 0..ns-1, coordinates 0..ms-1),
//   S[k][f] = sum_{c containing k and f} W_c - sum_s c_{s,k} c_{s,f} / n1_s,
// with c_{s,k} the weight of the cells of segment s that hold k. The operator then takes
// Y[k] = sum_f S[k][f] P[f] for the small k from this dense ms x m block (stored transposed,
// srow[f * ms + k], f over every coordinate) instead of accumulating per cell in the segment
// pass. srow depends on the weights: it is rebuilt with every weight state.

// c_{s,k} for every segment s and small coordinate k < ms: one thread per (segment, k), the
// segment's cells in order.
__global__ void k_seg_small_w(const u32* __restrict__ seg_off, const u32* __restrict__ coord, u32 M, u32 g1, int ns,
                              u32 ms, const double* __restrict__ cw, double* __restrict__ csk) {
    const size_t total = size_t(g1) * ms;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += size_t(gridDim.x) * blockDim.x) {
        const u32 s = u32(i / ms), k = u32(i % ms);
        double a = 0.0;
        for (u32 c = seg_off[s]; c < seg_off[s + 1]; c++) {
            const double w = cw ? cw[c] : 1.0;
            for (int b = 0; b < ns; b++)
                if (coord[size_t(b) * M + c] == k) a += w;
        }
        csk[i] = a;
    }
}

// Partial rows of srow by work items: item i covers entries [item_a, item_b) of the coordinate
// list of f = item_f (whole runs of equal segment). One warp per item, lane k < ms holding
// S[k][f] over the item: for every entry (cell c of segment s) W_c when c holds k; at the end of
// each run of segment s, - c_{s,k} c_{s,f} / n1_s with c_{s,f} the run's weight sum. Every lane
// sums in entry order; k_srow_sum adds the items of a coordinate in item order.
__global__ void __launch_bounds__(256) k_srow_items(const u32* __restrict__ coord, u32 M, int ns, u32 ms,
                                                    const double* __restrict__ cw, const double* __restrict__ n1inv,
                                                    const u32* __restrict__ pl_cell, const u32* __restrict__ pl_seg,
                                                    const double* __restrict__ csk, const u32* __restrict__ item_a,
                                                    const u32* __restrict__ item_b, u32 nitems,
                                                    double* __restrict__ part) {
    const u32 lane = threadIdx.x & 31u;
    const u32 it = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (it >= nitems) return;  // whole warps
    const u32 b = item_b[it];
    double acc = 0.0, run = 0.0;
    for (u32 e = item_a[it]; e < b; e++) {
        const u32 c = pl_cell[e], s = pl_seg[e];
        const double w = cw ? cw[c] : 1.0;
        for (int bb = 0; bb < ns; bb++)
            if (coord[size_t(bb) * M + c] == lane) acc += w;
        run += w;
        if (e + 1 == b || pl_seg[e + 1] != s) {
            if (lane < ms) acc -= csk[size_t(s) * ms + lane] * run * n1inv[s];
            run = 0.0;
        }
    }
    if (lane < ms) part[size_t(it) * ms + lane] = acc;
}

// srow[f * ms + k] = the partial rows of f's items (first[f] .. first[f+1]) added in item order.
__global__ void k_srow_sum(const double* __restrict__ part, const u32* __restrict__ first, u32 m, u32 ms,
                           double* __restrict__ srow) {
    const size_t total = size_t(m) * ms;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += size_t(gridDim.x) * blockDim.x) {
        const u32 f = u32(i / ms), k = u32(i % ms);
        double v = 0.0;
        for (u32 it = first[f]; it < first[f + 1]; it++) v += part[size_t(it) * ms + k];
        srow[i] = v;
    }
}

// Exact leverage of the fixed-effect columns per row (leverage.rs:128 fe_hat, by block
// elimination of FE1): h_i = w_i (1 / W_s + v_c' G v_c) for row i of cell c in segment s, where
// v_c = b_c - t_s, b_c the indicator of c's reduced coordinates, t_s = sum_{c' in s} W_c' b_c' / W_s
// and G a generalized inverse of the reduced system S (any one: v_c lies in the range of
// S = sum_c W_c v_c v_c'). G: the dense m x m inverse. One thread per segment, cells in order.
__global__ void k_fe_leverage(DevStruct S, DevWeights W, const double* __restrict__ G, double* __restrict__ h) {
    const u32 m = S.m, M = S.M;
    for (u32 s = blockIdx.x * blockDim.x + threadIdx.x; s < S.g1; s += gridDim.x * blockDim.x) {
        const u32 c0 = S.seg_off[s], c1 = S.seg_off[s + 1];
        const double winv = W.n1inv[s];
        // B(c, c') = b_c' G b_c'
        auto B = [&](u32 c, u32 c2) {
            double v = 0.0;
            for (u32 k = 0; k < S.nb; k++)
                for (u32 l = 0; l < S.nb; l++)
                    v += G[size_t(S.coord[size_t(k) * M + c]) * m + S.coord[size_t(l) * M + c2]];
            return v;
        };
        double tau = 0.0;  // t' G t
        for (u32 c = c0; c < c1; c++) {
            double row = 0.0;
            for (u32 c2 = c0; c2 < c1; c2++) row += cellw(W, c2) * B(c, c2);
            tau += cellw(W, c) * row;
        }
        tau *= winv * winv;
        for (u32 c = c0; c < c1; c++) {
            double gt = 0.0;  // b_c' G t
            for (u32 c2 = c0; c2 < c1; c2++) gt += cellw(W, c2) * B(c, c2);
            const double q = m ? B(c, c) - 2.0 * gt * winv + tau : 0.0;
            for (u32 i = row0_of(S, c); i < row1_of(S, c); i++) h[i] = (W.w_rows ? W.w_rows[i] : 1.0) * (winv + q);
        }
    }
}

}  // namespace fereg
