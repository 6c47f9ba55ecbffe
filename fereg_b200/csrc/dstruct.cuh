// Kernels of the cell-structure build on the device (structure.rs:356-527, restated from the host
// build in structure.cpp): the row order, the cells and segments, and the coordinate-sorted cell
// lists. Every array is the host build's, element for element: the sorts are stable LSD radix
// sorts (prep.cuh), and every other step is a per-element map or an order-free integer count.
#pragma once

#include "device.cuh"

namespace fereg {

constexpr int DS_TB = 256;

// Code columns of the session's terms in device memory: FE1 (t[0], when present) then the blocks,
// with each block term's first reduced coordinate (off[q], q >= has_fe1).
struct TermCodes {
    const u32* const* t;
    const u32* off;
    int nt;       // terms in t (FE1 counted when present)
    int has_fe1;
};

__device__ __forceinline__ bool row_key_differs(const TermCodes& tc, u32 a, u32 b) {
    for (int q = 0; q < tc.nt; q++)
        if (tc.t[q][a] != tc.t[q][b]) return true;
    return false;
}
// true when the key of row a is above that of row b (FE1, then the blocks in order)
__device__ __forceinline__ bool row_key_greater(const TermCodes& tc, u32 a, u32 b) {
    for (int q = 0; q < tc.nt; q++) {
        const u32 x = tc.t[q][a], y = tc.t[q][b];
        if (x != y) return x > y;
    }
    return false;
}

// flag = 1 when a code is not below its term's level count.
__global__ void k_ds_check(const u32* __restrict__ c, size_t n, u32 g, int* flag) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        if (c[i] >= g) atomicExch(flag, 1);
}

// flag = 1 when some consecutive rows (identity order) are out of key order.
__global__ void k_ds_unsorted(TermCodes tc, size_t n, int* flag) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x + 1; i < n; i += size_t(gridDim.x) * blockDim.x)
        if (row_key_greater(tc, u32(i - 1), u32(i))) atomicExch(flag, 1);
}

__global__ void k_ds_iota(u32* __restrict__ v, size_t n) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        v[i] = u32(i);
}

// key[i] = codes[pi[i]] (the sort key of one term, in the current order).
__global__ void k_ds_gather_key(const u32* __restrict__ codes, const u32* __restrict__ pi, size_t n,
                                u64* __restrict__ key) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        key[i] = codes[pi[i]];
}

// flags[r] = 1 when row r opens a cell (its key differs from the previous row's).
__global__ void k_ds_cell_flags(TermCodes tc, const u32* __restrict__ pi, size_t n, u32* __restrict__ flags) {
    for (size_t r = size_t(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += size_t(gridDim.x) * blockDim.x)
        flags[r] = (r == 0 || row_key_differs(tc, pi[r - 1], pi[r])) ? 1u : 0u;
}

// The cells: first row, FE1 level (segment) and block coordinates (block-major coord[k * M + c]).
__global__ void k_ds_cells(TermCodes tc, const u32* __restrict__ pi, size_t n, const u32* __restrict__ flags,
                           const u32* __restrict__ cell_of, u32 M, u32* __restrict__ cell_row, u32* __restrict__ cseg,
                           u32* __restrict__ coord) {
    for (size_t r = size_t(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += size_t(gridDim.x) * blockDim.x) {
        if (!flags[r]) continue;
        const u32 c = cell_of[r], o = pi[r];
        if (cell_row) cell_row[c] = u32(r);
        cseg[c] = tc.has_fe1 ? tc.t[0][o] : 0u;
        for (int q = tc.has_fe1; q < tc.nt; q++) coord[size_t(q - tc.has_fe1) * M + c] = tc.off[q] + tc.t[q][o];
    }
}

// seg_off[s] = the first cell of segment s (cells are in segment order; every level up to the
// last cell's is covered, the levels after it start at M).
__global__ void k_ds_seg_off(const u32* __restrict__ cseg, u32 M, u32 g1, u32* __restrict__ seg_off) {
    for (size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x; c <= M; c += size_t(gridDim.x) * blockDim.x) {
        const long long prev = c == 0 ? -1 : (long long)cseg[c - 1];
        const long long cur = c == M ? (long long)g1 : (long long)cseg[c];
        for (long long s = prev + 1; s <= cur && s <= (long long)g1; s++) seg_off[s] = u32(c);
    }
}

// The entries of the coordinate lists before their sort: block k's entries are the cells in
// order, keyed by their coordinate in block k (key[k * M + c], value c).
__global__ void k_ds_entries(const u32* __restrict__ coord, u32 M, int nb, u64* __restrict__ key, u32* __restrict__ val) {
    const size_t E = size_t(M) * nb;
    for (size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x; e < E; e += size_t(gridDim.x) * blockDim.x) {
        key[e] = coord[e];
        val[e] = u32(e % M);
    }
}

// Entry counts per coordinate (integer atomics: the counts do not depend on the order).
__global__ void k_ds_count(const u32* __restrict__ coord, size_t E, u32* __restrict__ cnt) {
    for (size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x; e < E; e += size_t(gridDim.x) * blockDim.x)
        atomicAdd(&cnt[coord[e]], 1u);
}

// After the sort: each entry's segment and the cell's coordinates in the other blocks (block
// order, the entry's own block skipped). boff[k] is block k's first coordinate, boff[nb] = m.
__global__ void k_ds_pull_rest(const u64* __restrict__ skey, const u32* __restrict__ cell, size_t E,
                               const u32* __restrict__ cseg, const u32* __restrict__ coord, u32 M, int nb,
                               const u32* __restrict__ boff, u32* __restrict__ pl_seg, u32* __restrict__ pl_other) {
    const int no = nb - 1;
    for (size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x; e < E; e += size_t(gridDim.x) * blockDim.x) {
        const u32 c = cell[e], x = u32(skey[e]);
        pl_seg[e] = cseg[c];
        int kb = 0;
        while (kb + 1 < nb && x >= boff[kb + 1]) kb++;
        int o = 0;
        for (int k2 = 0; k2 < nb; k2++)
            if (k2 != kb) pl_other[e * no + o++] = coord[size_t(k2) * M + c];
    }
}

// Dense small-block work: d_s, the number of (segment, small coordinate) pairs, as the runs of
// equal segment in the small coordinates' lists: one thread per entry of those lists (the first
// es entries), counting the entries that open a run (integer counts, order free).
__global__ void k_ds_small_pairs(const u64* __restrict__ skey, const u32* __restrict__ pl_seg, size_t es,
                                 u32* __restrict__ d) {
    for (size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x; e < es; e += size_t(gridDim.x) * blockDim.x)
        if (e == 0 || skey[e] != skey[e - 1] || pl_seg[e] != pl_seg[e - 1]) atomicAdd(&d[pl_seg[e]], 1u);
}

// sum over segments of d_s^2 into per-CTA partials (u64, order free).
__global__ void k_ds_sq_sum(const u32* __restrict__ d, u32 g1, unsigned long long* __restrict__ total) {
    unsigned long long a = 0;
    for (u32 s = blockIdx.x * blockDim.x + threadIdx.x; s < g1; s += gridDim.x * blockDim.x)
        a += (unsigned long long)d[s] * d[s];
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(FULL, a, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(total, a);
}

}  // namespace fereg
